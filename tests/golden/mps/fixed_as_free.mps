NAME          FIXEDFREE
ROWS
 N  COST
 L  LIM1
 G  LIM2
 E  MYEQN
 L  LIM3
COLUMNS
    XONE      COST      1.0            LIM1      1.0
    XONE      LIM2      1.0
    XTWO      COST      2.0            LIM1      1.0
    XTWO      MYEQN     -1.0
    XTHREE    COST      -1.0           MYEQN     1.0
    XFOUR     LIM3      2.5
RHS
              LIM1      4.0            LIM2      1.0
              MYEQN     7.0
              LIM3      3.0            MYEQN     8.0
    RHS       LIM2      2.0
BOUNDS
 UP BND       XONE      4.0
 UP           XTWO      5.0
ENDATA
