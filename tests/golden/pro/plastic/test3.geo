// 2 points
Point(1) = { 0, 0, 0, 3e-3 };
Point(2) = { 0, 100e-3, 0, 3e-3 };

// create a line
Line(1) = { 1, 2 };
