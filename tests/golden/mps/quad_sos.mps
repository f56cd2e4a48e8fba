NAME QP
ROWS
 N obj
 L c1
COLUMNS
    x obj 1 c1 1
    y obj 1 c1 1
RHS
    r c1 2
BOUNDS
 UP b x 5
QUADOBJ
    x x 2
    x y 1
    y y 2
SOS
 S1 SOS
    s1 S1 x 1 0 y 2 1
ENDATA
