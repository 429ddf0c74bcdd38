// 4 points
Point(1) = { 4, 0, 1, .5 };
Point(2) = { 4, 10, 1, .5 };

Point(3) = { 0, 5, 0, .5 };
Point(4) = { 14, 5, 0, .5 };

// create a line
Line(1) = { 1, 2 };
Line(2) = { 3, 4 };
