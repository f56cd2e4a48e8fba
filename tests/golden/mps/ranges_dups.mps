NAME RANGES
ROWS
 N  z
 L  r1
 G  r2
 E  r3
 E  r4
 L  r5
 l  r6
 L
COLUMNS
    x  z  1  r1  1
    x  r1  2
    x  r2  1  r3  1
    y  r2  -1  r4  1
    y  r2  1
    y  r5  0
    y  ghost  5
    x  r6  1  r4  3
    x  r3  1e-12
    x  r3  -1e-12
    x  r3  1
    y  c7  4
RHS
    rhs  r1  5  r2  1
    rhs  r3  2  r4  -3
    rhs  z  10
RANGES
    rng  r1  4  r2  2
    rng  r3  -1.5  r4  2
    rng  r5  -1
BOUNDS
 UP  x  4
 UP BND y 9
ENDATA
