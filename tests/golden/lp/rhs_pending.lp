\ a constraint whose right-hand side is on the next line
Minimize
 x + y
Subject To
 c1: x + y >=
 2
 c2: x <= 5
End
