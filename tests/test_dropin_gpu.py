"""GPU: the drop-in at the reference's own seam. The reference's unchanged
InteriorPointSolver::solve runs with InteriorPointOptions::compute_backend set
to the B200 backend through the maintainer-side adapter (oracle/dropin_adapter.cpp
compiled against the reference sources). It must reach the reference's status
and objective (golden, CPU backend) while its products run as GPU kernels."""
import ctypes as C
import os

import numpy as np
import pytest

import lpgen
import oracle as O

pytestmark = pytest.mark.gpu
LIB = os.path.join(os.path.dirname(O.REF_LIB), "libhnref_dropin.so")
GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "reference_golden.npz"))


@pytest.mark.skipif(not os.path.exists(LIB), reason="oracle/_ref drop-in library not built")
@pytest.mark.parametrize("name,args", [("ipm_60x150", (60, 150, 8, 3)), ("ipm_200x500", (200, 500, 8, 4))])
def test_reference_ipm_with_b200_backend(hn, name, args):
    lib = C.CDLL(LIB)
    f = lib.hnref_ipm_solve_b200
    f.restype = C.c_int
    lp = lpgen.lp_uniform(*args)
    rp, ci = np.ascontiguousarray(lp["rp"], np.uint64), np.ascontiguousarray(lp["ci"], np.uint64)
    val, c, b = (np.ascontiguousarray(lp[k], np.float64) for k in ("val", "c", "b"))
    obj, iters, kern = C.c_double(), C.c_int64(), C.c_uint64()
    P = lambda a, t: a.ctypes.data_as(C.POINTER(t))  # noqa: E731
    st = f(C.c_int64(lp["m"]), C.c_int64(lp["n"]), P(rp, C.c_uint64), P(ci, C.c_uint64), P(val, C.c_double),
           P(c, C.c_double), P(b, C.c_double), C.byref(obj), C.byref(iters), C.byref(kern))
    g = GOLD[name]
    assert st == int(g[0])
    assert abs(obj.value - g[1]) <= 1e-8 * (1.0 + abs(g[1]))
    assert kern.value > 0  # the reference IPM's M x products ran on the GPU
