"""ctypes binding of libhn_sm100.so (include/hn_sm100.h) for Python callers.

The binding is thin: every call goes straight to the C ABI, device buffers
are passed as raw pointers (e.g. torch.Tensor.data_ptr()), host arrays as
numpy arrays. A missing or unloadable library raises -- there is no CPU
fallback anywhere on this path.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libhn_sm100.so")
HOST_LIB_PATH = os.path.join(HERE, "libhn_host.so")

HN_OK = 0
HN_ERR_INVALID_ARG = 1
HN_ERR_CUDA = 2
HN_ERR_OUT_OF_MEMORY = 3
HN_ERR_NOT_INITIALIZED = 4
HN_ERR_UNSUPPORTED = 5
HN_ERR_NUMERICAL = 6
HN_ERR_INJECTED = 7
HN_CSR_NO_AUTOTUNE = 2
SPMV_MERGE, SPMV_BINNED = 0, 1
HN_CSR_NO_TRANSPOSE = 1

_i64, _u64p, _f64p, _vp, _i32p = C.c_int64, C.POINTER(C.c_uint64), C.POINTER(C.c_double), C.c_void_p, C.POINTER(C.c_int32)
_i64p = C.POINTER(C.c_int64)


class HnError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"[{status}] {msg}")
        self.status = status


class DeviceInfo(C.Structure):
    _fields_ = [("name", C.c_char * 256), ("device", C.c_int), ("sm_count", C.c_int),
                ("cc_major", C.c_int), ("cc_minor", C.c_int), ("total_mem", C.c_size_t),
                ("free_mem", C.c_size_t)]


# name -> argtypes (restype is int status unless listed in _RESTYPE)
SIGNATURES = {
    "hn_init": [C.c_int],
    "hn_shutdown": [],
    "hn_last_error": [],
    "hn_device_info": [C.POINTER(DeviceInfo)],
    "hn_stats": [C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)],
    "hn_reset_stats": [],
    "hn_fault_inject": [_i64, C.c_int],
    "hn_malloc": [C.POINTER(C.c_void_p), C.c_size_t],
    "hn_free": [_vp],
    "hn_memcpy_h2d": [_vp, _vp, C.c_size_t, _vp],
    "hn_memcpy_d2h": [_vp, _vp, C.c_size_t, _vp],
    "hn_memcpy_d2d": [_vp, _vp, C.c_size_t, _vp],
    "hn_memset": [_vp, C.c_int, C.c_size_t, _vp],
    "hn_stream_sync": [_vp],
    "hn_csr_create": [_i64, _i64, _u64p, _u64p, _f64p, C.c_uint, C.POINTER(_vp)],
    "hn_csr_set_values": [_vp, _f64p],
    "hn_csr_destroy": [_vp],
    "hn_csr_shape": [_vp, _i64p, _i64p, _i64p, _i64p],
    "hn_csr_export": [_vp, C.c_int, _u64p, _u64p, _f64p],
    "hn_csr_create_coo": [_i64, _i64, _i64, _i64p, _i64p, _f64p, C.c_uint, C.POINTER(_vp)],
    "hn_csr_tiles": [_vp, C.c_int, _i64p, _i64p],
    "hn_csr_export_tiles": [_vp, C.c_int, _i32p, _i32p],
    "hn_spmv": [_vp, C.c_int, C.c_double, _vp, C.c_double, _vp, _vp],
    "hn_spmv_host": [_vp, C.c_int, _f64p, _f64p],
    "hn_spmm": [_vp, C.c_int, _vp, _i64, _vp, _vp],
    "hn_spmm_host": [_vp, C.c_int, _f64p, _i64, _f64p],
    "hn_dot": [_i64, _vp, _vp, _vp, _vp],
    "hn_axpy": [_i64, C.c_double, _vp, _vp, _vp],
    "hn_nrm_inf": [_i64, _vp, _vp, _vp],
    "hn_nrm2": [_i64, _vp, _vp, _vp],
    "hn_ada_symbolic": [_vp, C.POINTER(_vp)],
    "hn_ada_symbolic_ex": [_vp, C.c_uint, C.POINTER(_vp)],
    "hn_pattern_mode": [_vp, C.POINTER(C.c_int), _i64p],
    "hn_pattern_info": [_vp, _i64p, _i64p],
    "hn_pattern_export": [_vp, _u64p, _u64p],
    "hn_pattern_device": [_vp, C.POINTER(_vp), C.POINTER(_vp), C.POINTER(_vp)],
    "hn_ada_numeric": [_vp, _vp, C.c_double, _vp, _vp, _vp],
    "hn_pattern_destroy": [_vp],
    "hn_ipm_residuals": [_vp] + [_vp] * 11 + [_vp],
    "hn_ipm_rhs": [_vp, _vp, _vp, _vp, _vp, _vp],
    "hn_ipm_direction": [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp],
    "hn_ipm_step_lengths": [_i64, _i64, _vp, _vp, _vp, _vp, _vp, _vp, _vp],
    "hn_ipm_corrector": [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp],
    "hn_ipm_update": [_i64, _i64, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp],
    "hn_max_step": [_i64, _vp, _vp, _vp, _vp],
    "hn_ipm_kkt": [_i64, _i64] + [_vp] * 8 + [C.c_double, _vp, _vp],
    "hn_spmv_noalloc": [_i64, _i64, _i64, _vp, _vp, _vp, _vp, _vp, _vp],
    "hn_csr_spmv_kind": [_vp, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)],
    "hn_spmv_residual": [_vp, C.c_int, _vp, _vp, _vp, _vp],
    "hn_csr_set_spmv_kind": [_vp, C.c_int, C.c_int, C.c_int],
    "hn_price_reduced_costs": [_vp, _vp, _vp, _vp, _vp],
    "hn_price_devex_update": [_vp, _vp, _vp, _vp, _vp, _vp],
    "hn_price_select": [_i64, _vp, _vp, _vp, _vp, C.c_int, C.c_int, C.c_double, C.c_int, _i64, _vp, _vp],
    "hn_price_columns": [_vp, _i64, _vp, _vp, _vp],
    "hn_gnn_spmm": [_vp, C.c_int, _vp, _vp, C.c_int, _vp],
    "hn_gnn_cast_weights": [C.c_int, _vp, _vp, _vp, _vp],
    "hn_gnn_linear": [_i64, C.c_int, C.c_int, _vp, _vp, _vp, C.c_int, _vp, C.c_int, _vp, _vp],
    "hn_gnn_linear_umma": [_i64, C.c_int, C.c_int, _vp, _vp, _vp, _vp, C.c_int, _vp, _vp],
    "hn_gnn_check": [_vp],
    "hn_gnn_set_wait_limit": [C.c_uint32],
    "hn_gnn_linear_bwd": [_i64, C.c_int, C.c_int, _vp, _vp, _vp, _vp, _vp, C.c_int, _vp, _vp, _vp, _vp, _vp, _i64,
                          _vp],
    "hn_gnn_split_grad": [_i64, _vp, _vp, _vp, _vp],
    "hn_gnn_head_grad": [_i64, _vp, _vp, C.c_int, C.c_float, _vp, _vp, _i64, _vp],
    "hn_gnn_adam": [_i64, _vp, _vp, _vp, _vp, C.c_float, C.c_float, C.c_float, C.c_float, _i64, _vp],
    "hn_batch_create": [_i64, _i64p, _i64p, _vp, C.POINTER(_vp)],
    "hn_batch_destroy": [_vp],
    "hn_batch_residuals": [_vp, _vp] + [_vp] * 13 + [C.c_int, C.c_double, C.c_double, _vp],
    "hn_batch_factor": [_vp, _vp, C.c_double, C.c_double, _vp, _vp, _vp],
    "hn_batch_solve": [_vp, _vp, _vp, _vp, _vp, _vp],
    "hn_batch_steps": [_vp] + [_vp] * 7 + [_vp],
    "hn_batch_corrector": [_vp, _vp] + [_vp] * 9 + [_vp],
    "hn_batch_update": [_vp] + [_vp] * 9 + [C.c_int, _vp],
    "hn_batch_set_kkt": [_vp, _vp, _vp, _vp, C.c_double, C.c_int],
    "hn_batch_kkt": [_vp, _f64p, _i32p],
    "hn_batch_finish": [_vp, _vp, _vp, _vp, _vp, _vp, _vp],
}
_RESTYPE = {"hn_last_error": C.c_char_p}

_lib = None


def load(path: str = LIB_PATH) -> C.CDLL:
    """Load the library once and declare every exported signature."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} is missing: build it with build.py (no CPU fallback exists)")
    lib = C.CDLL(path)
    for name, args in SIGNATURES.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = _RESTYPE.get(name, C.c_int)
    _lib = lib
    return lib


def check(status: int) -> None:
    if status != HN_OK:
        raise HnError(status, load().hn_last_error().decode(errors="replace"))


def _p(a: np.ndarray, ct):
    return a.ctypes.data_as(C.POINTER(ct))


def u64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.uint64)


def _as_u64(a: np.ndarray) -> np.ndarray:
    """Index array as uint64: int64 input is reinterpreted in place when
    non-negative, anything else converted."""
    a = np.ascontiguousarray(a)
    if a.dtype == np.int64 and (a.size == 0 or a.min() >= 0):
        return a.view(np.uint64)
    return np.ascontiguousarray(a, dtype=np.uint64)


def f64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


def init(device: int = 0) -> None:
    check(load().hn_init(device))


def device_info() -> DeviceInfo:
    d = DeviceInfo()
    check(load().hn_device_info(C.byref(d)))
    return d


def stats() -> tuple[int, int]:
    a, b = C.c_uint64(), C.c_uint64()
    check(load().hn_stats(C.byref(a), C.byref(b)))
    return a.value, b.value


def reset_stats() -> None:
    check(load().hn_reset_stats())


def fault_inject(after_calls: int, status: int) -> None:
    check(load().hn_fault_inject(after_calls, status))


def _ptr(t) -> int | None:
    """Device pointer of a torch tensor / int / None."""
    if t is None:
        return None
    if isinstance(t, int):
        return t
    return t.data_ptr()


class Csr:
    """Device-resident CSR matrix handle (hn_csr)."""

    def __init__(self, m: int, n: int, rp, ci, val, transpose: bool = True, autotune: bool = True):
        self.m, self.n = int(m), int(n)
        self._rp, self._ci, self._val = u64(rp), u64(ci), f64(val)
        h = C.c_void_p()
        flags = (0 if transpose else HN_CSR_NO_TRANSPOSE) | (0 if autotune else HN_CSR_NO_AUTOTUNE)
        check(load().hn_csr_create(self.m, self.n, _p(self._rp, C.c_uint64), _p(self._ci, C.c_uint64),
                                   _p(self._val, C.c_double), flags, C.byref(h)))
        self.h = h
        m_, n_, nnz, nnzt = C.c_int64(), C.c_int64(), C.c_int64(), C.c_int64()
        check(load().hn_csr_shape(h, C.byref(m_), C.byref(n_), C.byref(nnz), C.byref(nnzt)))
        self.nnz, self.nnz_t = nnz.value, nnzt.value

    @classmethod
    def from_coo(cls, m: int, n: int, rows, cols, vals, transpose: bool = True, autotune: bool = True) -> "Csr":
        """A from triplets in any order (duplicates summed in input order,
        exact-zero sums dropped), sorted into CSR on the device
        (hn_csr_create_coo)."""
        self = cls.__new__(cls)
        self.m, self.n = int(m), int(n)
        r, c, v = (np.ascontiguousarray(rows, dtype=np.int64), np.ascontiguousarray(cols, dtype=np.int64),
                   f64(vals))
        h = C.c_void_p()
        flags = (0 if transpose else HN_CSR_NO_TRANSPOSE) | (0 if autotune else HN_CSR_NO_AUTOTUNE)
        check(load().hn_csr_create_coo(self.m, self.n, r.shape[0], _p(r, C.c_int64), _p(c, C.c_int64),
                                       _p(v, C.c_double), flags, C.byref(h)))
        self.h = h
        m_, n_, nnz, nnzt = C.c_int64(), C.c_int64(), C.c_int64(), C.c_int64()
        check(load().hn_csr_shape(h, C.byref(m_), C.byref(n_), C.byref(nnz), C.byref(nnzt)))
        self.nnz, self.nnz_t = nnz.value, nnzt.value
        self._rp = self._ci = self._val = None
        return self

    def spmv_kind(self, trans: int = 0):
        """(kind, t): 0 merge path, 1 binned vector kernel with t nonzeros per lane."""
        k, t = C.c_int(), C.c_int()
        check(load().hn_csr_spmv_kind(self.h, trans, C.byref(k), C.byref(t)))
        return k.value, t.value

    def set_spmv_kind(self, kind: int, t: int = 8, trans: int = 0) -> None:
        check(load().hn_csr_set_spmv_kind(self.h, trans, kind, t))

    def set_values(self, val) -> None:
        self._val = f64(val)
        check(load().hn_csr_set_values(self.h, _p(self._val, C.c_double)))
        m_, n_, nnz, nnzt = C.c_int64(), C.c_int64(), C.c_int64(), C.c_int64()
        check(load().hn_csr_shape(self.h, C.byref(m_), C.byref(n_), C.byref(nnz), C.byref(nnzt)))
        self.nnz_t = nnzt.value

    def close(self) -> None:
        if self.h:
            check(load().hn_csr_destroy(self.h))
            self.h = None

    def __del__(self):
        try:
            if getattr(self, "h", None) and _lib is not None:
                _lib.hn_csr_destroy(self.h)
                self.h = None
        except Exception:
            pass

    def spmv(self, x, y, trans: int = 0, alpha: float = 1.0, beta: float = 0.0, stream=None) -> None:
        check(load().hn_spmv(self.h, trans, alpha, _ptr(x), beta, _ptr(y), _ptr(stream)))

    def residual(self, x, b, y, trans: int = 0, stream=None) -> None:
        """y = op(A) x - b."""
        check(load().hn_spmv_residual(self.h, trans, _ptr(x), _ptr(b), _ptr(y), _ptr(stream)))

    def spmv_host(self, x, trans: int = 0) -> np.ndarray:
        x = f64(x)
        y = np.empty(self.n if trans else self.m, dtype=np.float64)
        check(load().hn_spmv_host(self.h, trans, _p(x, C.c_double), _p(y, C.c_double)))
        return y

    def spmm(self, B, k: int, Cout, trans: int = 0, stream=None) -> None:
        check(load().hn_spmm(self.h, trans, _ptr(B), k, _ptr(Cout), _ptr(stream)))

    def spmm_host(self, B, k: int, trans: int = 0) -> np.ndarray:
        B = f64(B)
        rows = self.n if trans else self.m
        Cout = np.empty(rows * k, dtype=np.float64)
        check(load().hn_spmm_host(self.h, trans, _p(B, C.c_double), k, _p(Cout, C.c_double)))
        return Cout

    def export(self, trans: int = 0):
        rows = self.n if trans else self.m
        nnz = self.nnz_t if trans else self.nnz
        rp = np.empty(rows + 1, dtype=np.uint64)
        ci = np.empty(max(nnz, 1), dtype=np.uint64)
        val = np.empty(max(nnz, 1), dtype=np.float64)
        check(load().hn_csr_export(self.h, trans, _p(rp, C.c_uint64), _p(ci, C.c_uint64),
                                   _p(val, C.c_double)))
        return rp, ci[:nnz], val[:nnz]

    def tiles(self, trans: int = 0):
        nt, items = C.c_int64(), C.c_int64()
        check(load().hn_csr_tiles(self.h, trans, C.byref(nt), C.byref(items)))
        row = np.empty(nt.value + 1, dtype=np.int32)
        nz = np.empty(nt.value + 1, dtype=np.int32)
        check(load().hn_csr_export_tiles(self.h, trans, _p(row, C.c_int32), _p(nz, C.c_int32)))
        return items.value, row, nz


class Pattern:
    """Fixed pattern of A diag(d) A^T + reg I (hn_pattern)."""

    # numeric layouts (hn_ada_symbolic_ex flags; hn_pattern_mode numbers)
    GATHER, ROW, RELATIVE = 0, 1, 2

    def __init__(self, A: Csr, compact: bool = False, layout: int | None = None):
        """layout: None = the library's choice, or GATHER / RELATIVE / ROW
        (ROW is also what compact=True asks for)."""
        flags = 1 if compact else 0
        if layout is not None:
            flags = {self.GATHER: 2, self.ROW: 1, self.RELATIVE: 4}[layout]
        h = C.c_void_p()
        check(load().hn_ada_symbolic_ex(A.h, flags, C.byref(h)))
        self.h = h
        self.A = A
        m, nnz = C.c_int64(), C.c_int64()
        check(load().hn_pattern_info(h, C.byref(m), C.byref(nnz)))
        self.m, self.nnz = m.value, nnz.value

    def mode(self):
        """(layout: GATHER / ROW / RELATIVE, longest row of N)."""
        rm, mr = C.c_int(), C.c_int64()
        check(load().hn_pattern_mode(self.h, C.byref(rm), C.byref(mr)))
        return rm.value, mr.value

    def export(self):
        rp = np.empty(self.m + 1, dtype=np.uint64)
        ci = np.empty(max(self.nnz, 1), dtype=np.uint64)
        check(load().hn_pattern_export(self.h, _p(rp, C.c_uint64), _p(ci, C.c_uint64)))
        return rp, ci[: self.nnz]

    def device_arrays(self):
        rp, ci, dp = C.c_void_p(), C.c_void_p(), C.c_void_p()
        check(load().hn_pattern_device(self.h, C.byref(rp), C.byref(ci), C.byref(dp)))
        return rp.value, ci.value, dp.value

    def numeric(self, d, reg: float, nval, dyn=None, stream=None) -> None:
        check(load().hn_ada_numeric(self.h, _ptr(d), reg, _ptr(nval), _ptr(dyn), _ptr(stream)))

    def close(self) -> None:
        if self.h:
            check(load().hn_pattern_destroy(self.h))
            self.h = None

    def __del__(self):
        try:
            if getattr(self, "h", None) and _lib is not None:
                _lib.hn_pattern_destroy(self.h)
                self.h = None
        except Exception:
            pass


def dot(n, a, b, out, stream=None) -> None:
    check(load().hn_dot(n, _ptr(a), _ptr(b), _ptr(out), _ptr(stream)))


def axpy(n, alpha, x, y, stream=None) -> None:
    check(load().hn_axpy(n, alpha, _ptr(x), _ptr(y), _ptr(stream)))


def nrm_inf(n, v, out, stream=None) -> None:
    check(load().hn_nrm_inf(n, _ptr(v), _ptr(out), _ptr(stream)))


def nrm2(n, v, out, stream=None) -> None:
    check(load().hn_nrm2(n, _ptr(v), _ptr(out), _ptr(stream)))


# ---- revised-simplex pricing (device vectors are torch CUDA tensors) ----
PRICE_BLAND, PRICE_RANKED = 0, 1


def price_reduced_costs(A: Csr, y, cost, rc, stream=None) -> None:
    """rc = cost - A^T y (SimplexSolver::compute_reduced_costs)."""
    check(load().hn_price_reduced_costs(A.h, _ptr(y), _ptr(cost), _ptr(rc), _ptr(stream)))


def price_devex_update(A: Csr, u, nonbasis, weights, alpha, stream=None) -> None:
    """Devex weights from the BTRAN row u (SimplexSolver::update_devex_weights)."""
    check(load().hn_price_devex_update(A.h, _ptr(u), _ptr(nonbasis), _ptr(weights), _ptr(alpha), _ptr(stream)))


def price_select(n, rc, weights, nonbasis, artificial, out, phase1=False, maximize=False, tol=1e-9,
                 rule=PRICE_RANKED, k=1, stream=None) -> None:
    """Entering-column choice into out (device int64, k+1): count, then indices."""
    check(load().hn_price_select(n, _ptr(rc), _ptr(weights), _ptr(nonbasis), _ptr(artificial), int(phase1),
                                 int(maximize), tol, rule, k, _ptr(out), _ptr(stream)))


def price_columns(A: Csr, cols, out, stream=None) -> None:
    """Dense columns of A (m x k, column-major) for the given device int64 indices."""
    check(load().hn_price_columns(A.h, int(cols.numel()), _ptr(cols), _ptr(out), _ptr(stream)))


def exported_symbols() -> list[str]:
    return list(SIGNATURES)


# ---------------------------------------------------------------- host layer (libhn_host.so)
INTERRUPT_CB = C.CFUNCTYPE(C.c_int, C.c_void_p)


class IpmOptions(C.Structure):
    _fields_ = [("max_iterations", C.c_int), ("time_limit_seconds", C.c_double), ("convergence_tol", C.c_double),
                ("complementarity_tol", C.c_double), ("regularization", C.c_double), ("device", C.c_int),
                ("verbose", C.c_int), ("interrupt_cb", INTERRUPT_CB), ("interrupt_user", C.c_void_p),
                ("initial_x", _f64p), ("initial_y", _f64p), ("initial_s", _f64p), ("warm_start_floor", C.c_double),
                ("factorization", C.c_int), ("kkt_tol", C.c_double), ("kkt_extra_iterations", C.c_int)]


class IpmResult(C.Structure):
    _fields_ = [("status", C.c_int), ("iterations", C.c_int64), ("objective", C.c_double),
                ("solve_time_ms", C.c_double), ("device_ms", C.c_double), ("factor_ms", C.c_double),
                ("solve_ms", C.c_double), ("nnz_normal", C.c_int64), ("warm_start_used", C.c_int),
                ("kkt_default", C.c_double), ("kkt_warm", C.c_double), ("kkt", C.c_double),
                ("kkt_primal", C.c_double), ("kkt_dual", C.c_double), ("kkt_gap", C.c_double),
                ("reference_iterations", C.c_int64)]


class SparseLdltStats(C.Structure):
    _fields_ = [("nnz_L", C.c_int64), ("supernodes", C.c_int64), ("singular", C.c_int), ("analyze_ms", C.c_double),
                ("factor_ms", C.c_double)]


HOST_SIGNATURES = {
    "hn_ipm_default_options": (None, [C.POINTER(IpmOptions)]),
    "hn_lp_solve": (C.c_int, [_i64, _i64, _u64p, _u64p, _f64p, _f64p, _f64p, C.POINTER(C.c_int), _f64p, _f64p,
                              C.c_int, C.c_double, C.POINTER(IpmOptions), C.POINTER(IpmResult), _f64p,
                              _f64p, _f64p]),
    "hn_host_last_error": (C.c_char_p, []),
    "hn_lp_solve_batch": (C.c_int, [_i64, _i64p, _i64p, _i64p, _u64p, _u64p, _f64p, _f64p, _f64p,
                                    C.POINTER(C.c_int), _f64p, _f64p, C.POINTER(C.c_int), _f64p,
                                    C.POINTER(IpmOptions), C.POINTER(C.c_int), _f64p, _i64p, _f64p, _vp,
                                    C.POINTER(C.c_int), _f64p, _f64p, _f64p, _i64p]),
    "hn_mps_read_file": (C.c_int, [C.c_char_p, C.c_int, C.POINTER(_vp)]),
    "hn_mps_read_string": (C.c_int, [C.c_char_p, _i64, C.c_int, C.POINTER(_vp)]),
    "hn_lp_read_file": (C.c_int, [C.c_char_p, C.POINTER(_vp)]),
    "hn_lp_read_string": (C.c_int, [C.c_char_p, _i64, C.POINTER(_vp)]),
    "hn_mps_shape": (C.c_int, [_vp, _i64p, _i64p, _i64p, C.POINTER(C.c_int)]),
    "hn_mps_arrays": (C.c_int, [_vp, _i64p, _i64p, _f64p, _f64p, _f64p, _i32p, _f64p, _f64p, _f64p, _f64p, _i32p]),
    "hn_mps_counts": (C.c_int, [_vp, _i64p, _i64p, _i64p]),
    "hn_mps_warning": (C.c_char_p, [_vp, _i64]),
    "hn_mps_name": (C.c_char_p, [_vp, C.c_int, _i64]),
    "hn_mps_free": (C.c_int, [_vp]),
    "hn_crossover_basis": (C.c_int, [_i64, _f64p, _f64p, _f64p, C.POINTER(C.c_int)]),
    "hn_amd_order": (C.c_int, [_i64, _u64p, _u64p, _i64p]),
    "hn_sparse_ldlt_solve": (C.c_int, [_i64, _u64p, _u64p, _f64p, C.c_double, _i64, _f64p,
                                       C.POINTER(SparseLdltStats)]),
    "hn_be_create": (C.c_int, [C.c_int, C.POINTER(_vp)]),
    "hn_be_destroy": (C.c_int, [_vp]),
    "hn_be_spmv": (C.c_int, [_vp, _i64, _i64, _u64p, _u64p, _f64p, _i64, _f64p, _f64p]),
    "hn_be_spmv_t": (C.c_int, [_vp, _i64, _i64, _i64, _u64p, _u64p, _f64p, _f64p, _f64p]),
    "hn_be_spmm": (C.c_int, [_vp, _i64, _i64, _u64p, _u64p, _f64p, _i64, _f64p, _i64, _f64p]),
    "hn_be_dot": (C.c_int, [_vp, _i64, _f64p, _f64p, _f64p]),
    "hn_be_axpy": (C.c_int, [_vp, _i64, C.c_double, _f64p, _f64p]),
    "hn_be_norm_inf": (C.c_int, [_vp, _i64, _f64p, _f64p]),
    "hn_be_kernel_executions": (C.c_int, [_vp, C.POINTER(C.c_uint64)]),
}
_host = None

STATUS = ["UNKNOWN", "OPTIMAL", "INFEASIBLE", "UNBOUNDED", "SUBOPTIMAL", "TIME_LIMIT", "ITER_LIMIT",
          "NUMERICAL_ERROR", "INTERRUPTED"]


def host() -> C.CDLL:
    global _host
    if _host is not None:
        return _host
    load()
    if not os.path.exists(HOST_LIB_PATH):
        raise FileNotFoundError(f"{HOST_LIB_PATH} is missing: build it with build.py")
    lib = C.CDLL(HOST_LIB_PATH)
    for name, (res, args) in HOST_SIGNATURES.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _host = lib
    return lib


def host_check(status: int) -> None:
    if status != HN_OK:
        raise HnError(status, host().hn_host_last_error().decode(errors="replace"))


def _warm_arrays(opt, x0, y0, s0):
    keep = []
    for name, a in (("initial_x", x0), ("initial_y", y0), ("initial_s", s0)):
        if a is not None:
            a = f64(a)
            keep.append(a)
            setattr(opt, name, _p(a, C.c_double))
    return keep


def mps_read(text: bytes | str | None = None, path: str | None = None, fmt: int = -1) -> dict:
    """The MPS reader (hn_mps_*, host): rows, columns, objective sense and the
    constraint coefficients as triplets in file order. fmt -1 detects the
    layout as the reference's MPSParser does, 0 free, 1 fixed."""
    h = C.c_void_p()
    if path is not None:
        host_check(host().hn_mps_read_file(os.fsencode(path), fmt, C.byref(h)))
    else:
        data = text.encode() if isinstance(text, str) else bytes(text)
        host_check(host().hn_mps_read_string(data, len(data), fmt, C.byref(h)))
    return _read_result(h)


def lp_read(text: bytes | str | None = None, path: str | None = None) -> dict:
    """The LP-format reader (hn_lp_read_*, host), same result layout as
    mps_read. Text the reference's LPParser would reject raises HnError."""
    h = C.c_void_p()
    if path is not None:
        host_check(host().hn_lp_read_file(os.fsencode(path), C.byref(h)))
    else:
        data = text.encode() if isinstance(text, str) else bytes(text)
        host_check(host().hn_lp_read_string(data, len(data), C.byref(h)))
    return _read_result(h)


def _read_result(h) -> dict:
    try:
        m, n, nt, mx = C.c_int64(), C.c_int64(), C.c_int64(), C.c_int()
        host_check(host().hn_mps_shape(h, C.byref(m), C.byref(n), C.byref(nt), C.byref(mx)))
        m, n, nt = m.value, n.value, nt.value
        o = {"m": m, "n": n, "maximize": mx.value,
             "trow": np.zeros(max(nt, 1), dtype=np.int64), "tcol": np.zeros(max(nt, 1), dtype=np.int64),
             "tval": np.zeros(max(nt, 1)), "c": np.zeros(max(n, 1)), "rhs": np.zeros(max(m, 1)),
             "sense": np.zeros(max(m, 1), dtype=np.int32), "lb": np.zeros(max(n, 1)), "ub": np.zeros(max(n, 1)),
             "range_lo": np.zeros(max(m, 1)), "range_hi": np.zeros(max(m, 1)),
             "vtype": np.zeros(max(n, 1), dtype=np.int32)}
        host_check(host().hn_mps_arrays(h, _p(o["trow"], C.c_int64), _p(o["tcol"], C.c_int64),
                                        _p(o["tval"], C.c_double), _p(o["c"], C.c_double),
                                        _p(o["rhs"], C.c_double), _p(o["sense"], C.c_int32),
                                        _p(o["lb"], C.c_double), _p(o["ub"], C.c_double),
                                        _p(o["range_lo"], C.c_double), _p(o["range_hi"], C.c_double),
                                        _p(o["vtype"], C.c_int32)))
        for k, size in (("trow", nt), ("tcol", nt), ("tval", nt), ("c", n), ("lb", n), ("ub", n), ("vtype", n),
                        ("rhs", m), ("sense", m), ("range_lo", m), ("range_hi", m)):
            o[k] = o[k][:size]
        nw, nsos, nq = C.c_int64(), C.c_int64(), C.c_int64()
        host_check(host().hn_mps_counts(h, C.byref(nw), C.byref(nsos), C.byref(nq)))
        o["warnings"] = [host().hn_mps_warning(h, i).decode() for i in range(nw.value)]
        o["sos_records"], o["quadratic_records"] = nsos.value, nq.value
        o["name"] = host().hn_mps_name(h, -1, 0).decode()
        o["row_names"] = [host().hn_mps_name(h, 0, i).decode() for i in range(m)]
        o["col_names"] = [host().hn_mps_name(h, 1, j).decode() for j in range(n)]
        return o
    finally:
        host().hn_mps_free(h)


def read_mps(path: str | None = None, text: bytes | str | None = None, fmt: int = -1) -> dict:
    """An MPS file as the LP dict lp_solve / lp_solve_batch take: the reader's
    triplets go to the device (hn_csr_create_coo) and come back as the CSR the
    reference's from_triplets builds; rhs -> b, sense, bounds, maximize."""
    return _lp_dict(mps_read(text=text, path=path, fmt=fmt))


def read_lp(path: str | None = None, text: bytes | str | None = None) -> dict:
    """An LP-format file as the LP dict lp_solve / lp_solve_batch take (device
    CSR as in read_mps)."""
    return _lp_dict(lp_read(text=text, path=path))


def _lp_dict(r: dict) -> dict:
    A = Csr.from_coo(r["m"], r["n"], r["trow"], r["tcol"], r["tval"], transpose=False, autotune=False)
    try:
        rp, ci, val = A.export()
    finally:
        A.close()
    return {"m": r["m"], "n": r["n"], "rp": rp, "ci": ci, "val": val, "b": r["rhs"], "c": r["c"],
            "sense": r["sense"], "lb": r["lb"], "ub": r["ub"], "maximize": bool(r["maximize"]),
            "vtype": r["vtype"], "range_lo": r["range_lo"], "range_hi": r["range_hi"], "name": r["name"]}


def amd_order(rp, ci) -> np.ndarray:
    """Approximate-minimum-degree ordering of a symmetric pattern (both
    triangles): perm[new] = old (hn_amd_order)."""
    rp, ci = u64(rp), u64(ci)
    m = rp.shape[0] - 1
    perm = np.zeros(m, dtype=np.int64)
    host_check(host().hn_amd_order(m, _p(rp, C.c_uint64), _p(ci, C.c_uint64), _p(perm, C.c_int64)))
    return perm


def sparse_ldlt_solve(rp, ci, val, B, singular_tol: float = 1e-12):
    """Solve N X = B with the host sparse LDL^T (hn_sparse_ldlt_solve); N in
    CSR with both triangles, B of shape (m,) or (nrhs, m). Returns (X, stats)."""
    rp, ci, val = u64(rp), u64(ci), f64(val)
    m = rp.shape[0] - 1
    X = np.array(B, dtype=np.float64, order="C", copy=True)
    nrhs = 1 if X.ndim == 1 else X.shape[0]
    st = SparseLdltStats()
    host_check(host().hn_sparse_ldlt_solve(m, _p(rp, C.c_uint64), _p(ci, C.c_uint64), _p(val, C.c_double),
                                           float(singular_tol), nrhs, _p(X, C.c_double), C.byref(st)))
    return X, {"nnz_L": st.nnz_L, "supernodes": st.supernodes, "singular": bool(st.singular),
               "analyze_ms": st.analyze_ms, "factor_ms": st.factor_ms}


def crossover_basis(x, lb, ub) -> np.ndarray:
    """The warm basis the reference's crossover gives its simplex polisher
    (hn_crossover_basis): -1 at lower bound, +1 at upper bound, 0 basic."""
    x, lb, ub = f64(x), f64(lb), f64(ub)
    out = np.zeros(x.shape[0], dtype=np.int32)
    host_check(host().hn_crossover_basis(x.shape[0], _p(x, C.c_double), _p(lb, C.c_double), _p(ub, C.c_double),
                                         out.ctypes.data_as(C.POINTER(C.c_int))))
    return out


def lp_solve(lp: dict, sense=None, lb=None, ub=None, maximize=False, obj_offset=0.0, max_iter=100,
             time_limit=0.0, device=0, interrupt=None, verbose=False, x0=None, y0=None, s0=None, warm_floor=None,
             factorization=0, kkt_tol=1e-8, kkt_extra=10):
    """GPU IPM on an LP given as CSR (rows EQ and x >= 0 unless told otherwise);
    x0/y0/s0: optional warm start in the original space. kkt_tol / kkt_extra:
    tightening past the reference's stop (kkt_tol <= 0: the reference's rule
    alone); the result's `kkt` is the relative KKT residual on the unscaled LP."""
    m, n = int(lp["m"]), int(lp["n"])
    rp, ci, val = u64(lp["rp"]), u64(lp["ci"]), f64(lp["val"])
    c, b = f64(lp["c"]), f64(lp["b"])
    sense = np.ascontiguousarray(np.full(m, 2) if sense is None else sense, dtype=np.int32)
    lb = f64(np.zeros(n) if lb is None else lb)
    ub = f64(np.full(n, np.inf) if ub is None else ub)
    opt = IpmOptions()
    host().hn_ipm_default_options(C.byref(opt))
    opt.max_iterations = max_iter
    opt.time_limit_seconds = time_limit
    opt.device = device
    opt.verbose = int(verbose)
    cb = INTERRUPT_CB(lambda _u: int(bool(interrupt()))) if interrupt is not None else INTERRUPT_CB()
    opt.interrupt_cb = cb
    # the C API reads n (x, s) and m (y) entries: a point of another size is
    # not a warm start for this LP and is not passed at all
    if any(a is not None and np.asarray(a).shape != (k,) for a, k in ((x0, n), (y0, m), (s0, n))):
        x0 = y0 = s0 = None
    keep = _warm_arrays(opt, x0, y0, s0)  # noqa: F841 (alive through the call)
    if warm_floor is not None:
        opt.warm_start_floor = warm_floor
    opt.factorization = int(factorization)  # 0 auto, 1 dense, 2 sparse (host normal-matrix factorisation)
    opt.kkt_tol = float(kkt_tol)
    opt.kkt_extra_iterations = int(kkt_extra)
    res = IpmResult()
    x = np.zeros(n)
    y = np.full(m, np.nan)
    s = np.full(n, np.nan)
    host_check(host().hn_lp_solve(m, n, _p(rp, C.c_uint64), _p(ci, C.c_uint64), _p(val, C.c_double),
                                  _p(c, C.c_double), _p(b, C.c_double), sense.ctypes.data_as(C.POINTER(C.c_int)),
                                  _p(lb, C.c_double), _p(ub, C.c_double), int(maximize), float(obj_offset),
                                  C.byref(opt), C.byref(res), _p(x, C.c_double), _p(y, C.c_double),
                                  _p(s, C.c_double)))
    err = host().hn_host_last_error().decode(errors="replace")
    return {"status": res.status, "status_name": STATUS[res.status], "objective": res.objective,
            "iterations": res.iterations, "time_ms": res.solve_time_ms, "device_ms": res.device_ms,
            "factor_ms": res.factor_ms, "solve_ms": res.solve_ms, "nnz_normal": res.nnz_normal, "x": x,
            "y": y, "s": s, "warm_start_used": bool(res.warm_start_used), "kkt_default": res.kkt_default,
            "kkt_warm": res.kkt_warm, "kkt": res.kkt, "kkt_parts": (res.kkt_primal, res.kkt_dual, res.kkt_gap),
            "reference_iterations": res.reference_iterations, "error": err}


class BatchStats(C.Structure):
    _fields_ = [("rows", C.c_int64), ("cols", C.c_int64), ("nnz", C.c_int64), ("nnz_normal", C.c_int64),
                ("iterations", C.c_int64), ("total_ms", C.c_double), ("factor_ms", C.c_double),
                ("solve_ms", C.c_double), ("forms_ms", C.c_double), ("setup_ms", C.c_double)]


def lp_solve_batch(lps: list, max_iter=100, device=0, senses=None, lbs=None, ubs=None, x0s=None, y0s=None,
                   s0s=None, warm_floor=None, kkt_tol=1e-8, kkt_extra=10):
    """Batched GPU IPM over a list of LP dicts (rows EQ, x >= 0 unless given);
    x0s/y0s/s0s: optional per-instance warm starts (lists of arrays);
    kkt_tol / kkt_extra as in lp_solve (per instance). The result's `kkt` is
    K x 4: relative KKT residual, primal, dual and gap parts."""
    K = len(lps)
    row_off = np.zeros(K + 1, np.int64)
    col_off = np.zeros(K + 1, np.int64)
    nnz_off = np.zeros(K + 1, np.int64)
    for i, lp in enumerate(lps):
        row_off[i + 1] = row_off[i] + lp["m"]
        col_off[i + 1] = col_off[i] + lp["n"]
        nnz_off[i + 1] = nnz_off[i] + len(lp["ci"])
    # one concatenation, then the non-negative int64 indices reinterpreted
    # as uint64 (a per-instance conversion costs ten times as much)
    rp = _as_u64(np.concatenate([np.asarray(lp["rp"]) for lp in lps]))
    ci = _as_u64(np.concatenate([np.asarray(lp["ci"]) for lp in lps]))
    val = f64(np.concatenate([lp["val"] for lp in lps]))
    c = f64(np.concatenate([lp["c"] for lp in lps]))
    b = f64(np.concatenate([lp["b"] for lp in lps]))
    sense = np.ascontiguousarray(np.concatenate(senses) if senses else np.full(row_off[-1], 2), dtype=np.int32)
    lb = f64(np.concatenate(lbs) if lbs else np.zeros(col_off[-1]))
    ub = f64(np.concatenate(ubs) if ubs else np.full(col_off[-1], np.inf))
    maxi = np.zeros(K, np.int32)
    off = np.zeros(K)
    opt = IpmOptions()
    host().hn_ipm_default_options(C.byref(opt))
    opt.max_iterations = max_iter
    opt.device = device
    opt.kkt_tol = float(kkt_tol)
    opt.kkt_extra_iterations = int(kkt_extra)
    for arrs, key in ((x0s, "n"), (y0s, "m"), (s0s, "n")):
        if arrs is not None and (len(arrs) != K or any(np.asarray(a).shape != (int(lp[key]),)
                                                       for a, lp in zip(arrs, lps))):
            raise ValueError(f"warm-start arrays must have one entry per instance of length {key}")
    keep = _warm_arrays(opt, None if x0s is None else np.concatenate(x0s),  # noqa: F841
                        None if y0s is None else np.concatenate(y0s), None if s0s is None else np.concatenate(s0s))
    if warm_floor is not None:
        opt.warm_start_floor = warm_floor
    warm_used = np.zeros(K, np.int32)
    status = np.zeros(K, np.int32)
    obj = np.zeros(K)
    iters = np.zeros(K, np.int64)
    x = np.zeros(col_off[-1])
    y = np.full(row_off[-1], np.nan)
    s = np.full(col_off[-1], np.nan)
    st = BatchStats()
    kkt = np.full((K, 4), np.nan)
    ref_it = np.zeros(K, np.int64)
    P = lambda a, t: a.ctypes.data_as(C.POINTER(t))  # noqa: E731
    host_check(host().hn_lp_solve_batch(K, P(row_off, C.c_int64), P(col_off, C.c_int64), P(nnz_off, C.c_int64),
                                        P(rp, C.c_uint64), P(ci, C.c_uint64), P(val, C.c_double), P(c, C.c_double),
                                        P(b, C.c_double), P(sense, C.c_int), P(lb, C.c_double), P(ub, C.c_double),
                                        P(maxi, C.c_int), P(off, C.c_double), C.byref(opt), P(status, C.c_int),
                                        P(obj, C.c_double), P(iters, C.c_int64), P(x, C.c_double),
                                        C.cast(C.pointer(st), C.c_void_p), P(warm_used, C.c_int), P(y, C.c_double),
                                        P(s, C.c_double), P(kkt, C.c_double), P(ref_it, C.c_int64)))
    return {"status": status, "objective": obj, "iterations": iters, "x": x, "y": y, "s": s, "col_off": col_off,
            "row_off": row_off, "kkt": kkt, "reference_iterations": ref_it,
            "warm_used": warm_used.astype(bool),
            "stats": {k: getattr(st, k) for k, _ in BatchStats._fields_}}


class Backend:
    """hn::execution::B200Backend (IComputeBackend) through the host C ABI."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        host_check(host().hn_be_create(device, C.byref(h)))
        self.h = h

    def close(self):
        if self.h:
            host().hn_be_destroy(self.h)
            self.h = None

    def spmv(self, rp, ci, val, x):
        rp, ci, val, x = u64(rp), u64(ci), f64(val), f64(x)
        m = rp.shape[0] - 1
        y = np.empty(m)
        host_check(host().hn_be_spmv(self.h, m, val.shape[0], _p(rp, C.c_uint64), _p(ci, C.c_uint64),
                                     _p(val, C.c_double), x.shape[0], _p(x, C.c_double), _p(y, C.c_double)))
        return y

    def spmv_t(self, rp, ci, val, x, n):
        rp, ci, val, x = u64(rp), u64(ci), f64(val), f64(x)
        m = rp.shape[0] - 1
        y = np.empty(n)
        host_check(host().hn_be_spmv_t(self.h, m, n, val.shape[0], _p(rp, C.c_uint64), _p(ci, C.c_uint64),
                                       _p(val, C.c_double), _p(x, C.c_double), _p(y, C.c_double)))
        return y

    def spmm(self, rp, ci, val, B, k):
        rp, ci, val, B = u64(rp), u64(ci), f64(val), f64(B)
        m = rp.shape[0] - 1
        Cm = np.empty(m * k)
        host_check(host().hn_be_spmm(self.h, m, val.shape[0], _p(rp, C.c_uint64), _p(ci, C.c_uint64),
                                     _p(val, C.c_double), B.shape[0] // max(k, 1), _p(B, C.c_double), k,
                                     _p(Cm, C.c_double)))
        return Cm

    def dot(self, a, b):
        a, b = f64(a), f64(b)
        out = C.c_double()
        host_check(host().hn_be_dot(self.h, min(a.shape[0], b.shape[0]), _p(a, C.c_double), _p(b, C.c_double),
                                    C.byref(out)))
        return out.value

    def axpy(self, alpha, x, y):
        x, y = f64(x), f64(y).copy()
        host_check(host().hn_be_axpy(self.h, min(x.shape[0], y.shape[0]), alpha, _p(x, C.c_double),
                                     _p(y, C.c_double)))
        return y

    def norm_inf(self, v):
        v = f64(v)
        out = C.c_double()
        host_check(host().hn_be_norm_inf(self.h, v.shape[0], _p(v, C.c_double), C.byref(out)))
        return out.value

    def kernel_executions(self):
        out = C.c_uint64()
        host_check(host().hn_be_kernel_executions(self.h, C.byref(out)))
        return out.value
