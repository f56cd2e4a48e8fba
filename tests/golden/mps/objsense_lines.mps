NAME          LINES
OBJSENSE
    MAXIMIZE
ROWS
 N  profit
 E  bal
COLUMNS
    a  profit  1.5  bal  1
    b  profit  -2  bal  1
RHS
    r  bal  3
ENDATA
