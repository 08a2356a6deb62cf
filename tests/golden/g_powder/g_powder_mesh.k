*X_GRID_PARAMETERS
$ zones / lengths / control volumes / exponents
  1
  0.00048
  16
  1
*Y_GRID_PARAMETERS
$ zones / lengths / control volumes / exponents
  3
  9e-05 0.00012 9e-05
  2 6 2
  -1.2 1 1.2
*Z_GRID_PARAMETERS
$ zones / lengths / control volumes / exponents
  2
  0.00015 0.00015
  3 5
  -1.2 1
