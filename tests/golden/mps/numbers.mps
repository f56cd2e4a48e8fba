NAME NUMBERS
ROWS
 N obj
 L a
 L b
 L c
 L d
COLUMNS
    x1 obj 1e5 a .5
    x2 obj -0.0 a +3
    x3 obj 1E-2 b 00012.5
    x4 obj 1.5abc 2
    x5 obj 1e b 2
    x6 b 7. c -.25e+1
    x7 c 6 d 1e999
    x8 d 4.25 obj 0x10
    x9 d 1.25e-310 a 9
RHS
    rhs a 1 b 2
    rhs c 3 d 4
ENDATA
