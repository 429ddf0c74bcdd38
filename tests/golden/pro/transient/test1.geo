// 2 points
Point(1) = { 0, 0, 0, 2.5 };
Point(2) = { 10, 0, 0, 2.5 };

// create a line
Line(1) = { 1, 2 };
