NAME MIXED
OBJSENSE MAX
ROWS
 N obj
 L c1
 G c2
COLUMNS
    MARKER                 'MARKER'                 'INTORG'
    y1 obj 3 c1 1
    y2 obj 2 c1 1
    y2 c2 1
    MARKER                 'MARKER'                 'INTEND'
    z obj 1 c2 1
    MARK0001  'MARKER'  'INTORG'
    w obj 4 c1 2
    MARK0002  'MARKER'  'INTEND'
RHS
    rhs c1 10 c2 2
BOUNDS
 UP b y1 1
 UI b y2 7
 LI b z 2
 UP b w 1
 SC b z 3
ENDATA
