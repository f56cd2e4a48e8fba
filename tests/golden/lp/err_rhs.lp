Minimize
 x + y
Subject To
 c1: x + y >= abc
End
