Minimize
 obj: x + 2 y
Subject To
 c1: x + y >= 1
	c2: x - y <= 3
Bounds
 x <= 10
End
