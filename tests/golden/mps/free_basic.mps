NAME          FREEBASIC
* a small LP in free layout: every row type, two pairs per line, all bound kinds
ROWS
 N  COST
 L  LIM1
 G  LIM2
 E  MYEQN
 L  LIM3
COLUMNS
    X1  COST  1.0  LIM1  1.0
    X1  LIM2  1.0
    X2  COST  2.0  LIM1  1.0
    X2  MYEQN  -1.0
    X3  COST  -1.0  MYEQN  1.0
    X4  COST  0.5  LIM3  2.5
    X5  LIM3  -3.25  LIM2  0.75
    X6  COST  1e-3  LIM1  4
    X7  LIM2  .5  MYEQN  -0.0
RHS
    RHS  LIM1  4.0  LIM2  1.0
    RHS  MYEQN  7.0
    RHS  LIM3  1e2
BOUNDS
 UP BND  X1  4.0
 LO BND  X2  -1.0
 UP BND  X2  1.0
 FX BND  X3  2.5
 FR BND  X4
 MI BND  X5
 PL BND  X5
 BV BND  X6
 UP BND  X7  -2
ENDATA
