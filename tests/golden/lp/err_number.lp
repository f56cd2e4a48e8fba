Minimize
 . x + y
Subject To
 c1: x <= 3
End
