NAME          FIXEDNET
ROWS
 N  COST
 L  LIM 1
 G  LIM2
 E  EQ
COLUMNS
    X         COST      1.0            LIM 1     1.0
    X         LIM2      1.0
    Y         COST      2.0            LIM 1     1.0
    Y         EQ        -1.0
    Z         COST      -123456.78901  EQ                 1.0
    W         LIM2      0.5            EQ        2
RHS
              LIM 1     4.0            LIM2      1.0
    RHS       EQ        7.0
BOUNDS
 UP BND       X         4.0
 MI BND       W
ENDATA
