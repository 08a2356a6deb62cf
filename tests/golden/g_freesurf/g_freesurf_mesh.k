*X_GRID_PARAMETERS
$ zones / lengths / control volumes / exponents
  1
  0.00072
  24
  1
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
  4 6
  -1.2 1
