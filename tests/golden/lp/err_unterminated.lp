Minimize
 x + y
Subject To
 c1: x + y
 c2: x - y <= 1
End
