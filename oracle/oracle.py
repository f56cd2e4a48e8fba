"""ctypes loaders for the two CPU checkers -- TEST INFRASTRUCTURE ONLY.

  * port():  libhn_oracle.so, the C restatement in hn_oracle.c
  * ref():   _ref/libhnref.so, the reference's own LP stack compiled from its
             sources by the Makefile here (None when it was not built)

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module; the product never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_LIB = os.path.join(HERE, "libhn_oracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libhnref.so")

_i64 = C.c_int64
_i64p = C.POINTER(C.c_int64)
_u64p = C.POINTER(C.c_uint64)
_f64p = C.POINTER(C.c_double)
_i32p = C.POINTER(C.c_int32)
_u8p = C.POINTER(C.c_uint8)
_vp = C.c_void_p

_port = None
_ref = None


def build(ref_dir: str | None = None) -> None:
    """make the port (always) and, given the reference's source root (or the
    REF environment variable), the reference build."""
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)
    ref_dir = ref_dir or os.environ.get("REF")
    if ref_dir and os.path.isdir(os.path.join(ref_dir, "core")):
        subprocess.run(["make", "-s", "-j8", "-C", HERE, "ref", f"REF={ref_dir}"], check=True)


def _p(a, ct):
    return a.ctypes.data_as(C.POINTER(ct))


def port():
    global _port
    if _port is None:
        if not os.path.exists(PORT_LIB):
            build()
        lib = C.CDLL(PORT_LIB)
        sig = {
            "hno_csr_multiply": (None, [_i64, _i64p, _i64p, _f64p, _f64p, _f64p]),
            "hno_csr_tmultiply": (None, [_i64, _i64, _i64p, _i64p, _f64p, _f64p, _f64p]),
            "hno_matvec_t": (None, [_i64, _i64, _i64p, _i64p, _f64p, _f64p, _f64p]),
            "hno_csr_transposed": (_i64, [_i64, _i64, _i64p, _i64p, _f64p, _i64p, _i64p, _f64p]),
            "hno_spmm": (None, [_i64, _i64p, _i64p, _f64p, _f64p, _i64, _f64p]),
            "hno_dot": (C.c_double, [_i64, _f64p, _f64p]),
            "hno_axpy": (None, [_i64, C.c_double, _f64p, _f64p]),
            "hno_norm_inf": (C.c_double, [_i64, _f64p]),
            "hno_nrm2": (C.c_double, [_i64, _f64p]),
            "hno_max_step": (C.c_double, [_i64, _f64p, _f64p]),
            "hno_normal_equations_triplets": (_i64, [_i64, _i64, _i64p, _i64p, _f64p]),
            "hno_normal_equations": (_i64, [_i64, _i64, _i64p, _i64p, _f64p, _f64p, C.c_double, _i64p,
                                            _i64p, _f64p, _f64p]),
            "hno_ada_pattern": (_i64, [_i64, _i64, _i64p, _i64p, _i64p, _i32p]),
            "hno_normal_rows": (_i64, [_i64, _i64, _i64p, _i64p, _f64p, _f64p, C.c_double, _i64, _i64p, _i64p,
                                       _i64p, _f64p, _f64p, _f64p]),
            "hno_merge_tiles": (None, [_i64, _i64, _i32p, _i64, _i64, _i32p, _i32p]),
            "hno_price_reduced_costs": (None, [_i64, _i64, _i64p, _i64p, _f64p, _f64p, _f64p, _f64p]),
            "hno_price_devex_update": (None, [_i64, _i64, _i64p, _i64p, _f64p, _f64p, _i32p, _f64p, _f64p]),
            "hno_price_ranked": (_i64, [_i64, _f64p, _f64p, _i32p, _u8p, C.c_int, C.c_int, C.c_double, _i64,
                                        _i64p]),
            "hno_price_bland": (_i64, [_i64, _f64p, _i32p, _u8p, C.c_int, C.c_int, C.c_double]),
            "hno_extract_column": (None, [_i64, _i64p, _i64p, _f64p, _i64, _f64p]),
        }
        for name, (res, args) in sig.items():
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args
        _port = lib
    return _port


def ref():
    """The compiled reference, or None when oracle/_ref was not built."""
    global _ref
    if _ref is None:
        if not os.path.exists(REF_LIB):
            return None
        lib = C.CDLL(REF_LIB)
        sig = {
            "hnref_backend_spmv": (C.c_int, [_i64, _i64, _u64p, _u64p, _f64p, _f64p, _f64p]),
            "hnref_backend_spmm": (C.c_int, [_i64, _i64, _u64p, _u64p, _f64p, _f64p, _i64, _f64p]),
            "hnref_backend_dot": (C.c_double, [_i64, _f64p, _f64p]),
            "hnref_backend_axpy": (None, [_i64, C.c_double, _f64p, _f64p]),
            "hnref_backend_norm_inf": (C.c_double, [_i64, _f64p]),
            "hnref_multiply": (C.c_int, [_i64, _i64, _u64p, _u64p, _f64p, _f64p, _f64p]),
            "hnref_tmultiply": (C.c_int, [_i64, _i64, _u64p, _u64p, _f64p, _f64p, _f64p]),
            "hnref_transposed": (_i64, [_i64, _i64, _u64p, _u64p, _f64p, _u64p, _u64p, _f64p]),
            "hnref_from_triplets": (_i64, [_i64, _i64, _i64, _u64p, _u64p, _f64p, _u64p, _u64p, _f64p]),
            "hnref_mps_parse": (_vp, [C.c_char_p, _i64, C.c_int]),
            "hnref_mps_shape": (C.c_int, [_vp, _i64p, _i64p, _i64p, _i32p, _i32p, _i64p]),
            "hnref_mps_arrays": (C.c_int, [_vp, _u64p, _u64p, _f64p, _f64p, _f64p, _i32p, _f64p, _f64p, _f64p,
                                           _f64p, _i32p]),
            "hnref_mps_name": (C.c_char_p, [_vp, C.c_int, _i64]),
            "hnref_mps_free": (None, [_vp]),
            "hnref_mps_parse_ms": (C.c_double, [C.c_char_p, _i64]),
            "hnref_lp_parse": (_vp, [C.c_char_p, _i64]),
            "hnref_parse_errors": (_i64, [_vp]),
            "hnref_cholesky_solve": (C.c_int, [_i64, _u64p, _u64p, _f64p, _f64p]),
            "hnref_cholesky_stats": (C.c_int, [_i64, _u64p, _u64p, _f64p, _i64p, _f64p, _f64p, _f64p]),
            "hnref_crossover_polish": (C.c_int, [_i64, _i64, _u64p, _u64p, _f64p, _f64p, _f64p, _i32p, _f64p,
                                                 _f64p, C.c_int, C.c_int, _i32p, _f64p, _i64p]),
            "hnref_ipm_solve": (C.c_int, [_i64, _i64, _u64p, _u64p, _f64p, _f64p, _f64p, _i32p, _f64p,
                                          _f64p, C.c_int, C.c_int, C.c_int, _f64p, _i64p, _f64p, _f64p]),
            "hnref_bench_spmv_pair": (C.c_double, [_i64, _i64, _u64p, _u64p, _f64p, _f64p, _f64p, C.c_int,
                                                   C.c_int]),
            "hnref_normal_equations": (_i64, [_i64, _i64, _u64p, _u64p, _f64p, _f64p, C.c_double, _i64, _u64p,
                                              _u64p, _f64p]),
            "hnref_matvec_t": (None, [_i64, _i64, _u64p, _u64p, _f64p, _f64p, _f64p]),
            "hnref_max_step": (C.c_double, [_i64, _f64p, _f64p]),
            "hnref_step_sample": (C.c_double, [_i64, _i64, _u64p, _u64p, _f64p, _f64p, _f64p, _f64p, _i64,
                                               C.c_int, C.c_int, _i64p, _i64p]),
            "hnref_price_reduced_costs": (None, [_i64, _i64, _u64p, _u64p, _f64p, _f64p, _f64p, _f64p]),
            "hnref_price_devex_update": (None, [_i64, _i64, _u64p, _u64p, _f64p, _f64p, _i32p, _f64p]),
            "hnref_price_ranked": (_i64, [_i64, _f64p, _f64p, _i32p, _u8p, C.c_int, C.c_int, _i64, _i64p]),
            "hnref_price_select": (_i64, [_i64, _f64p, _f64p, _i32p, _u8p, C.c_int, C.c_int, C.c_int]),
            "hnref_price_edge_weight": (C.c_double, [_i64, _i64, _u64p, _u64p, _f64p, _i64]),
        }
        for name, (res, args) in sig.items():
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args
        _ref = lib
    return _ref


# ---------------------------------------------------------------- port wrappers
def i64(a):
    return np.ascontiguousarray(a, dtype=np.int64)


def f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def multiply(rp, ci, val, x):
    rp, ci, val, x = i64(rp), i64(ci), f64(val), f64(x)
    y = np.empty(rp.shape[0] - 1)
    port().hno_csr_multiply(rp.shape[0] - 1, _p(rp, C.c_int64), _p(ci, C.c_int64), _p(val, C.c_double),
                            _p(x, C.c_double), _p(y, C.c_double))
    return y


def tmultiply(rp, ci, val, x, n):
    rp, ci, val, x = i64(rp), i64(ci), f64(val), f64(x)
    y = np.empty(n)
    port().hno_csr_tmultiply(rp.shape[0] - 1, n, _p(rp, C.c_int64), _p(ci, C.c_int64), _p(val, C.c_double),
                             _p(x, C.c_double), _p(y, C.c_double))
    return y


def matvec_t(rp, ci, val, x, n):
    rp, ci, val, x = i64(rp), i64(ci), f64(val), f64(x)
    y = np.empty(n)
    port().hno_matvec_t(rp.shape[0] - 1, n, _p(rp, C.c_int64), _p(ci, C.c_int64), _p(val, C.c_double),
                        _p(x, C.c_double), _p(y, C.c_double))
    return y


def transposed(rp, ci, val, n):
    rp, ci, val = i64(rp), i64(ci), f64(val)
    nnz = int(rp[-1])
    rpT = np.empty(n + 1, dtype=np.int64)
    ciT = np.empty(max(nnz, 1), dtype=np.int64)
    valT = np.empty(max(nnz, 1))
    w = port().hno_csr_transposed(rp.shape[0] - 1, n, _p(rp, C.c_int64), _p(ci, C.c_int64),
                                  _p(val, C.c_double), _p(rpT, C.c_int64), _p(ciT, C.c_int64),
                                  _p(valT, C.c_double))
    return rpT, ciT[:w], valT[:w]


def spmm(rp, ci, val, B, k):
    rp, ci, val, B = i64(rp), i64(ci), f64(val), f64(B)
    m = rp.shape[0] - 1
    Cm = np.empty(m * k)
    port().hno_spmm(m, _p(rp, C.c_int64), _p(ci, C.c_int64), _p(val, C.c_double), _p(B, C.c_double), k,
                    _p(Cm, C.c_double))
    return Cm


def dot(a, b):
    a, b = f64(a), f64(b)
    return port().hno_dot(a.shape[0], _p(a, C.c_double), _p(b, C.c_double))


def norm_inf(v):
    v = f64(v)
    return port().hno_norm_inf(v.shape[0], _p(v, C.c_double))


def nrm2(v):
    v = f64(v)
    return port().hno_nrm2(v.shape[0], _p(v, C.c_double))


def axpy(alpha, x, y):
    x, y = f64(x), f64(y).copy()
    port().hno_axpy(x.shape[0], alpha, _p(x, C.c_double), _p(y, C.c_double))
    return y


def max_step(v, d):
    v, d = f64(v), f64(d)
    return port().hno_max_step(v.shape[0], _p(v, C.c_double), _p(d, C.c_double))


def normal_equations(rp, ci, val, D, reg, n):
    rp, ci, val, D = i64(rp), i64(ci), f64(val), f64(D)
    m = rp.shape[0] - 1
    nt = port().hno_normal_equations_triplets(m, n, _p(rp, C.c_int64), _p(ci, C.c_int64), _p(D, C.c_double))
    rpN = np.empty(m + 1, dtype=np.int64)
    ciN = np.empty(max(nt, 1), dtype=np.int64)
    valN = np.empty(max(nt, 1))
    dyn = C.c_double()
    w = port().hno_normal_equations(m, n, _p(rp, C.c_int64), _p(ci, C.c_int64), _p(val, C.c_double),
                                    _p(D, C.c_double), reg, _p(rpN, C.c_int64), _p(ciN, C.c_int64),
                                    _p(valN, C.c_double), C.byref(dyn))
    return rpN, ciN[:w], valN[:w], dyn.value


def normal_rows(rp, ci, val, D, reg, n, rows):
    """Rows `rows` of build_normal_equations' N: (rpS, ciS, valS, absS, dyn)
    with rpS the offsets of the selected rows (hno_normal_rows)."""
    rp, ci, val, D, rows = i64(rp), i64(ci), f64(val), f64(D), i64(rows)
    m = rp.shape[0] - 1
    rpS = np.empty(rows.shape[0] + 1, dtype=np.int64)
    args = (m, n, _p(rp, C.c_int64), _p(ci, C.c_int64), _p(val, C.c_double), _p(D, C.c_double), reg,
            rows.shape[0], _p(rows, C.c_int64), _p(rpS, C.c_int64))
    total = port().hno_normal_rows(*args, None, None, None, None)
    ciS = np.empty(max(total, 1), dtype=np.int64)
    valS = np.empty(max(total, 1))
    absS = np.empty(max(total, 1))
    dyn = C.c_double()
    port().hno_normal_rows(*args, _p(ciS, C.c_int64), _p(valS, C.c_double), _p(absS, C.c_double), C.byref(dyn))
    return rpS, ciS[:total], valS[:total], absS[:total], dyn.value


def ada_pattern(rp, ci, n):
    rp, ci = i64(rp), i64(ci)
    m = rp.shape[0] - 1
    rpN = np.empty(m + 1, dtype=np.int64)
    total = port().hno_ada_pattern(m, n, _p(rp, C.c_int64), _p(ci, C.c_int64), _p(rpN, C.c_int64), None)
    ciN = np.empty(max(total, 1), dtype=np.int32)
    port().hno_ada_pattern(m, n, _p(rp, C.c_int64), _p(ci, C.c_int64), _p(rpN, C.c_int64), _p(ciN, C.c_int32))
    return rpN, ciN[:total]


def merge_tiles(rp32, nnz, items, ntiles):
    rp32 = np.ascontiguousarray(rp32, dtype=np.int32)
    row = np.empty(ntiles + 1, dtype=np.int32)
    nz = np.empty(ntiles + 1, dtype=np.int32)
    port().hno_merge_tiles(rp32.shape[0] - 1, nnz, _p(rp32, C.c_int32), items, ntiles, _p(row, C.c_int32),
                           _p(nz, C.c_int32))
    return row, nz


# ---------------------------------------------------------------- reference wrappers
def u64(a):
    return np.ascontiguousarray(a, dtype=np.uint64)


def ref_multiply(rp, ci, val, x):
    rp, ci, val, x = u64(rp), u64(ci), f64(val), f64(x)
    y = np.empty(rp.shape[0] - 1)
    ref().hnref_multiply(rp.shape[0] - 1, x.shape[0], _p(rp, C.c_uint64), _p(ci, C.c_uint64),
                         _p(val, C.c_double), _p(x, C.c_double), _p(y, C.c_double))
    return y


def ref_backend_spmv(rp, ci, val, x):
    rp, ci, val, x = u64(rp), u64(ci), f64(val), f64(x)
    y = np.empty(rp.shape[0] - 1)
    ref().hnref_backend_spmv(rp.shape[0] - 1, x.shape[0], _p(rp, C.c_uint64), _p(ci, C.c_uint64),
                             _p(val, C.c_double), _p(x, C.c_double), _p(y, C.c_double))
    return y


def ref_tmultiply(rp, ci, val, x, n):
    rp, ci, val, x = u64(rp), u64(ci), f64(val), f64(x)
    y = np.empty(n)
    ref().hnref_tmultiply(rp.shape[0] - 1, n, _p(rp, C.c_uint64), _p(ci, C.c_uint64), _p(val, C.c_double),
                          _p(x, C.c_double), _p(y, C.c_double))
    return y


def ref_transposed(rp, ci, val, n):
    rp, ci, val = u64(rp), u64(ci), f64(val)
    nnz = int(rp[-1])
    rpT = np.empty(n + 1, dtype=np.uint64)
    ciT = np.empty(max(nnz, 1), dtype=np.uint64)
    valT = np.empty(max(nnz, 1))
    w = ref().hnref_transposed(rp.shape[0] - 1, n, _p(rp, C.c_uint64), _p(ci, C.c_uint64), _p(val, C.c_double),
                               _p(rpT, C.c_uint64), _p(ciT, C.c_uint64), _p(valT, C.c_double))
    return rpT, ciT[:w], valT[:w]


def ref_from_triplets(rows, cols, ti, tj, tv):
    ti, tj, tv = u64(ti), u64(tj), f64(tv)
    rp = np.empty(rows + 1, dtype=np.uint64)
    ci = np.empty(max(ti.shape[0], 1), dtype=np.uint64)
    val = np.empty(max(ti.shape[0], 1))
    w = ref().hnref_from_triplets(rows, cols, ti.shape[0], _p(ti, C.c_uint64), _p(tj, C.c_uint64),
                                  _p(tv, C.c_double), _p(rp, C.c_uint64), _p(ci, C.c_uint64), _p(val, C.c_double))
    return rp, ci[:w], val[:w]


def from_triplets_port(rows: int, cols: int, ti, tj, tv):
    """Restatement of SparseMatrix::from_triplets (sparse_matrix.cpp:8-53) and
    sum_duplicates (:230-262): entries ordered by (row, column) -- equal keys
    in input order (the reference's std::sort leaves their order
    unspecified) -- each run of equal keys summed left to right from its
    first value, exact-zero sums dropped. Returns (rp, ci, val)."""
    ti = np.asarray(ti, dtype=np.int64)
    tj = np.asarray(tj, dtype=np.int64)
    tv = np.asarray(tv, dtype=np.float64)
    order = np.lexsort((tj, ti))  # stable: primary row, secondary column
    rp = np.zeros(rows + 1, dtype=np.uint64)
    ci, val = [], []
    k = 0
    while k < order.shape[0]:
        p = order[k]
        s = tv[p]
        q = k + 1
        while q < order.shape[0] and ti[order[q]] == ti[p] and tj[order[q]] == tj[p]:
            s = s + tv[order[q]]
            q += 1
        if s != 0.0:
            ci.append(tj[p])
            val.append(s)
            rp[ti[p] + 1] += 1
        k = q
    rp = np.cumsum(rp).astype(np.uint64)
    return rp, np.array(ci, dtype=np.uint64), np.array(val, dtype=np.float64)


def ref_mps(text: bytes, fmt: int = -1, lp_format: bool = False) -> dict:
    """model::MPSParser::parse_string on `text` (fmt -1: the parser's own
    layout detection, 0 free, 1 fixed), or model::LPParser::parse_string when
    lp_format: the parsed problem's arrays, the constraint matrix as the
    reference's CSR, the row/column names and the error count."""
    h = ref().hnref_lp_parse(text, len(text)) if lp_format else ref().hnref_mps_parse(text, len(text), fmt)
    try:
        m, n, nnz, mx, ok, nw = (C.c_int64(), C.c_int64(), C.c_int64(), C.c_int32(), C.c_int32(), C.c_int64())
        ref().hnref_mps_shape(h, C.byref(m), C.byref(n), C.byref(nnz), C.byref(mx), C.byref(ok), C.byref(nw))
        m, n, nnz = m.value, n.value, nnz.value
        out = {"m": m, "n": n, "maximize": mx.value, "success": ok.value, "warnings": nw.value,
               "rp": np.zeros(m + 1, dtype=np.uint64), "ci": np.zeros(max(nnz, 1), dtype=np.uint64),
               "val": np.zeros(max(nnz, 1)), "c": np.zeros(max(n, 1)), "rhs": np.zeros(max(m, 1)),
               "sense": np.zeros(max(m, 1), dtype=np.int32), "lb": np.zeros(max(n, 1)), "ub": np.zeros(max(n, 1)),
               "range_lo": np.zeros(max(m, 1)), "range_hi": np.zeros(max(m, 1)),
               "vtype": np.zeros(max(n, 1), dtype=np.int32)}
        ref().hnref_mps_arrays(h, *(_p(out[k], C.c_uint64) for k in ("rp", "ci")), _p(out["val"], C.c_double),
                               _p(out["c"], C.c_double), _p(out["rhs"], C.c_double), _p(out["sense"], C.c_int32),
                               _p(out["lb"], C.c_double), _p(out["ub"], C.c_double),
                               _p(out["range_lo"], C.c_double), _p(out["range_hi"], C.c_double),
                               _p(out["vtype"], C.c_int32))
        for k, size in (("ci", nnz), ("val", nnz), ("c", n), ("lb", n), ("ub", n), ("vtype", n), ("rhs", m),
                        ("sense", m), ("range_lo", m), ("range_hi", m)):
            out[k] = out[k][:size]
        out["errors"] = ref().hnref_parse_errors(h)
        out["name"] = ref().hnref_mps_name(h, -1, 0).decode()
        out["row_names"] = [ref().hnref_mps_name(h, 0, i).decode() for i in range(m)]
        out["col_names"] = [ref().hnref_mps_name(h, 1, j).decode() for j in range(n)]
        return out
    finally:
        ref().hnref_mps_free(h)


def ref_mps_parse_ms(text: bytes) -> float:
    return ref().hnref_mps_parse_ms(text, len(text))


def ref_backend_spmm(rp, ci, val, B, k, n):
    rp, ci, val, B = u64(rp), u64(ci), f64(val), f64(B)
    m = rp.shape[0] - 1
    Cm = np.empty(m * k)
    ref().hnref_backend_spmm(m, n, _p(rp, C.c_uint64), _p(ci, C.c_uint64), _p(val, C.c_double),
                             _p(B, C.c_double), k, _p(Cm, C.c_double))
    return Cm


def ref_ipm_solve(lp: dict, sense=None, lb=None, ub=None, maximize=False, max_iter=0, crossover=False):
    """InteriorPointSolver::solve on the LP (rows EQ and x >= 0 by default)."""
    m, n = lp["m"], lp["n"]
    rp, ci, val = u64(lp["rp"]), u64(lp["ci"]), f64(lp["val"])
    c, b = f64(lp["c"]), f64(lp["b"])
    sense = np.ascontiguousarray(np.full(m, 2) if sense is None else sense, dtype=np.int32)
    lb = f64(np.zeros(n) if lb is None else lb)
    ub = f64(np.full(n, np.inf) if ub is None else ub)
    obj, iters, tms = C.c_double(), C.c_int64(), C.c_double()
    x = np.zeros(n)
    st = ref().hnref_ipm_solve(m, n, _p(rp, C.c_uint64), _p(ci, C.c_uint64), _p(val, C.c_double),
                               _p(c, C.c_double), _p(b, C.c_double), _p(sense, C.c_int32), _p(lb, C.c_double),
                               _p(ub, C.c_double), int(maximize), int(max_iter), int(crossover), C.byref(obj),
                               C.byref(iters), C.byref(tms), _p(x, C.c_double))
    return {"status": st, "objective": obj.value, "iterations": iters.value, "time_ms": tms.value, "x": x}


def ref_cholesky_stats(rp, ci, val, b=None) -> dict:
    """SparseCholesky analyze + factorize (+ solve of b): nnz(L), singular,
    phase times, solution."""
    rp, ci, val = u64(rp), u64(ci), f64(val)
    m = rp.shape[0] - 1
    x = None if b is None else f64(np.array(b, dtype=np.float64, copy=True))
    nnz, ta, tf = C.c_int64(), C.c_double(), C.c_double()
    sing = ref().hnref_cholesky_stats(m, _p(rp, C.c_uint64), _p(ci, C.c_uint64), _p(val, C.c_double), C.byref(nnz),
                                      C.byref(ta), C.byref(tf), None if x is None else _p(x, C.c_double))
    return {"nnz_L": nnz.value, "singular": bool(sing), "analyze_ms": ta.value, "factor_ms": tf.value, "x": x}


def ref_crossover_polish(lp: dict, var_status, barrier_status: int, sense=None, lb=None, ub=None,
                         maximize=False) -> dict:
    """The reference's crossover polish (interior_point.cpp:792-876) from the
    caller's warm basis `var_status` and barrier verdict."""
    m, n = lp["m"], lp["n"]
    rp, ci, val = u64(lp["rp"]), u64(lp["ci"]), f64(lp["val"])
    c, b = f64(lp["c"]), f64(lp["b"])
    sense = np.ascontiguousarray(np.full(m, 2) if sense is None else sense, dtype=np.int32)
    lb = f64(np.zeros(n) if lb is None else lb)
    ub = f64(np.full(n, np.inf) if ub is None else ub)
    vs = np.ascontiguousarray(var_status, dtype=np.int32)
    obj, iters = C.c_double(), C.c_int64()
    st = ref().hnref_crossover_polish(m, n, _p(rp, C.c_uint64), _p(ci, C.c_uint64), _p(val, C.c_double),
                                      _p(c, C.c_double), _p(b, C.c_double), _p(sense, C.c_int32),
                                      _p(lb, C.c_double), _p(ub, C.c_double), int(maximize), int(barrier_status),
                                      _p(vs, C.c_int32), C.byref(obj), C.byref(iters))
    return {"status": st, "objective": obj.value, "iterations": iters.value}


def ref_normal_equations(rp, ci, val, D, reg, n):
    """build_normal_equations itself (interior_point.cpp:144-200)."""
    rp, ci, val, D = u64(rp), u64(ci), f64(val), f64(D)
    m = rp.shape[0] - 1
    rpN = np.empty(m + 1, dtype=np.uint64)
    nnz = ref().hnref_normal_equations(m, n, _p(rp, C.c_uint64), _p(ci, C.c_uint64), _p(val, C.c_double),
                                       _p(D, C.c_double), reg, 0, _p(rpN, C.c_uint64), None, None)
    ciN = np.empty(max(nnz, 1), dtype=np.uint64)
    vN = np.empty(max(nnz, 1))
    ref().hnref_normal_equations(m, n, _p(rp, C.c_uint64), _p(ci, C.c_uint64), _p(val, C.c_double),
                                 _p(D, C.c_double), reg, nnz, _p(rpN, C.c_uint64), _p(ciN, C.c_uint64),
                                 _p(vN, C.c_double))
    return rpN, ciN[:nnz], vN[:nnz]


def ref_matvec_t(rp, ci, val, x, n):
    rp, ci, val, x = u64(rp), u64(ci), f64(val), f64(x)
    y = np.empty(n)
    ref().hnref_matvec_t(rp.shape[0] - 1, n, _p(rp, C.c_uint64), _p(ci, C.c_uint64), _p(val, C.c_double),
                         _p(x, C.c_double), _p(y, C.c_double))
    return y


def ref_max_step(v, d):
    v, d = f64(v), f64(d)
    return ref().hnref_max_step(v.shape[0], _p(v, C.c_double), _p(d, C.c_double))


def ref_step_sample(lp, x, lam, D, ncols_sample, threads, reps):
    """Reference CPU pass (spmv, matvec_t, build_normal_equations on column
    slices) on `threads` host threads; returns (seconds, triplets, nnz(N))."""
    rp, ci, val = u64(lp["rp"]), u64(lp["ci"]), f64(lp["val"])
    x, lam, D = f64(x), f64(lam), f64(D)
    trip, nnzn = C.c_int64(), C.c_int64()
    secs = ref().hnref_step_sample(lp["m"], lp["n"], _p(rp, C.c_uint64), _p(ci, C.c_uint64), _p(val, C.c_double),
                                   _p(x, C.c_double), _p(lam, C.c_double), _p(D, C.c_double), int(ncols_sample),
                                   int(threads), int(reps), C.byref(trip), C.byref(nnzn))
    return secs, trip.value, nnzn.value


# ---- revised-simplex pricing (core/lp/simplex.cpp) ----
def price_reduced_costs(m, n, rp, ci, val, y, cost):
    rp, ci = i64(rp), i64(ci)
    rc = np.empty(n)
    port().hno_price_reduced_costs(m, n, _p(rp, C.c_int64), _p(ci, C.c_int64), _p(f64(val), C.c_double),
                                   _p(f64(y), C.c_double), _p(f64(cost), C.c_double), _p(rc, C.c_double))
    return rc


def price_devex_update(m, n, rp, ci, val, u, nonbasis, weights):
    """Returns (new weights, alpha = A^T u)."""
    rp, ci = i64(rp), i64(ci)
    w = np.array(weights, dtype=np.float64)
    alpha = np.empty(n)
    nb = np.ascontiguousarray(nonbasis, dtype=np.int32)
    port().hno_price_devex_update(m, n, _p(rp, C.c_int64), _p(ci, C.c_int64), _p(f64(val), C.c_double),
                                  _p(f64(u), C.c_double), _p(nb, C.c_int32), _p(w, C.c_double),
                                  _p(alpha, C.c_double))
    return w, alpha


def price_ranked(rc, w, nonbasis, artificial, phase1=False, maximize=False, tol=1e-9, cap=None):
    n = len(rc)
    cap = n if cap is None else cap
    out = np.empty(max(cap, 1), dtype=np.int64)
    nb = np.ascontiguousarray(nonbasis, dtype=np.int32)
    art = np.ascontiguousarray(artificial, dtype=np.uint8)
    cnt = port().hno_price_ranked(n, _p(f64(rc), C.c_double), _p(f64(w), C.c_double), _p(nb, C.c_int32),
                                  _p(art, C.c_uint8), int(phase1), int(maximize), tol, cap,
                                  _p(out, C.c_int64))
    return cnt, out[:cap]


def price_bland(rc, nonbasis, artificial, phase1=False, maximize=False, tol=1e-9):
    nb = np.ascontiguousarray(nonbasis, dtype=np.int32)
    art = np.ascontiguousarray(artificial, dtype=np.uint8)
    return port().hno_price_bland(len(rc), _p(f64(rc), C.c_double), _p(nb, C.c_int32), _p(art, C.c_uint8),
                                  int(phase1), int(maximize), tol)


def extract_column(m, rp, ci, val, j):
    rp, ci = i64(rp), i64(ci)
    col = np.empty(m)
    port().hno_extract_column(m, _p(rp, C.c_int64), _p(ci, C.c_int64), _p(f64(val), C.c_double), j,
                              _p(col, C.c_double))
    return col


def ref_price_reduced_costs(m, n, rp, ci, val, y, cost):
    rc = np.empty(n)
    ref().hnref_price_reduced_costs(m, n, _p(u64(rp), C.c_uint64), _p(u64(ci), C.c_uint64),
                                    _p(f64(val), C.c_double), _p(f64(y), C.c_double), _p(f64(cost), C.c_double),
                                    _p(rc, C.c_double))
    return rc


def ref_price_devex_update(m, n, rp, ci, val, u, nonbasis, weights):
    w = np.array(weights, dtype=np.float64)
    nb = np.ascontiguousarray(nonbasis, dtype=np.int32)
    ref().hnref_price_devex_update(m, n, _p(u64(rp), C.c_uint64), _p(u64(ci), C.c_uint64),
                                   _p(f64(val), C.c_double), _p(f64(u), C.c_double), _p(nb, C.c_int32),
                                   _p(w, C.c_double))
    return w


def ref_price_ranked(rc, w, nonbasis, artificial, phase1=False, maximize=False, cap=None):
    n = len(rc)
    cap = n if cap is None else cap
    out = np.empty(max(cap, 1), dtype=np.int64)
    nb = np.ascontiguousarray(nonbasis, dtype=np.int32)
    art = np.ascontiguousarray(artificial, dtype=np.uint8)
    cnt = ref().hnref_price_ranked(n, _p(f64(rc), C.c_double), _p(f64(w), C.c_double), _p(nb, C.c_int32),
                                   _p(art, C.c_uint8), int(phase1), int(maximize), cap, _p(out, C.c_int64))
    return cnt, out[: min(cap, cnt)]


def ref_price_select(rc, w, nonbasis, artificial, phase1=False, maximize=False, rule=1):
    nb = np.ascontiguousarray(nonbasis, dtype=np.int32)
    art = np.ascontiguousarray(artificial, dtype=np.uint8)
    return ref().hnref_price_select(len(rc), _p(f64(rc), C.c_double), _p(f64(w), C.c_double), _p(nb, C.c_int32),
                                    _p(art, C.c_uint8), int(phase1), int(maximize), rule)


def ref_price_edge_weight(m, n, rp, ci, val, var):
    return ref().hnref_price_edge_weight(m, n, _p(u64(rp), C.c_uint64), _p(u64(ci), C.c_uint64),
                                         _p(f64(val), C.c_double), var)
