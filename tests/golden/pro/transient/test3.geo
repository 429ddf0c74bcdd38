// 3 points
Point(1) = { 0, 0, 0, 1 };
Point(2) = { 10, 0, 0, 1 };
Point(3) = { 10, -10, 0, 1 };

// create lines
Line(1) = { 1, 2 };
Line(2) = { 2, 3 };
