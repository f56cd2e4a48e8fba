* no N row: the first unknown row referenced in COLUMNS becomes the objective
NAME IMPLICIT
ROWS
 L cap
 G dem
COLUMNS
    p  cost  3  cap  1
    q  cost  5  cap  1
    q  dem  1
    r  other  7  dem  2
RHS
    b  cap  8  dem  1
ENDATA
