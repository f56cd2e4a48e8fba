\ objective with a name, constraints over two lines, all senses, bounds forms
Maximize
 obj: 3 x + 2 y - z + 0.5 w
Subject To
 c1: x + y + z <= 10
 c2: x - y
   >= -2
 3 x + 2 z = 5
 cap: 2 x + 4 y + w <= 12.5
Bounds
 0 <= x <= 4
 -inf <= y <= 8
 z >= 1
 w <= 3
 y = 2
General
 y
End
