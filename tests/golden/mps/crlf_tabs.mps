NAME          CRLF
ROWS
 N  obj
 L  c1
	G  c2
COLUMNS
    x	obj	1	c1	1
    y  obj  2  c2  1
    y  c1  1
RHS
    rhs  c1  4  c2  1
BOUNDS
 UP bnd x 3
ENDATA
