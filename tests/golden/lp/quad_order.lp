\ variables first named in the quadratic groups of the objective come before
\ those first named in constraints
Minimize
 cost: a + 2 b + [ 2 c ^ 2 + 3 c * d - e * e ] / 2
 + 4 f
Subject To
 r1: a + b + f >= 1
 r2: g + a = 2
 r3: 2 h - b <= 4
QUADRATIC
 [ h * i + 2 j ^ 2 ]
Binaries
 g h
End
