*X_GRID_PARAMETERS
$ zones / lengths / control volumes / exponents
  3
  0.000216 0.000288 0.000216
  6 12 6
  -1.2 1 1.2
*Y_GRID_PARAMETERS
$ zones / lengths / control volumes / exponents
  3
  0.000126 0.000168 0.000126
  3 8 3
  -1.2 1 1.2
*Z_GRID_PARAMETERS
$ zones / lengths / control volumes / exponents
  2
  0.00015 0.00015
  3 5
  -1.2 1
