Minimize
 x
Subject To
 c1: x + y < 3
End
