** a comment line
max
 2 p + 3 q
st
 p + q <= 4
 p + 3 q <= 6
constraints
 named: p - q = 0
semi-continuous
 p
GENERALS
 p q
SOS
 s1: S1:: p:1 q:2
END
