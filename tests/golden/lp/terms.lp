MINIMIZE
\ coefficient forms: exponents, leading dots, implicit 1, repeated variables,
\ a constant term, names with digits and underscores
 obj: 1e2 x_1 + .5 x2 - 2.5E-1 x3 + x_1 + 7
SUBJECT TO
 k1: 2e3x_1 + 3 x2 + x2 - x3 <= 1e1
 k2: - x_1 - 2 x2 >= -1.5e0
 k3: 0 x3 + x_1 = 0
 k4: 2 3 x2 + 1.5.5 x3 <= 2
S.T.
 k5: x3 <= 4
BOUNDS
 x2 >= -1
 .5 <= x3
 x_1 <= 1e3
 y free
End
garbage after end is ignored
