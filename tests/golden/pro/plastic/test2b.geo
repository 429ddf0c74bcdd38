// 2 points
Point(1) = { 0, 0, 0, 0.2 };
Point(2) = { 0, 1, 0, 0.2 };

// create a line
Line(1) = { 1, 2 };
