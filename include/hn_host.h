/* hn_host -- host C++ layer above hn_sm100 (libhn_host.so), as a C ABI.
 *
 *  - hn_lp_solve: the GPU Mehrotra IPM (hn::lp::InteriorPointSolver), a
 *    drop-in for HyperNova's lp::InteriorPointSolver::solve
 *    (core/lp/interior_point.cpp:402-886) with crossover off.
 *  - hn_be_*: hn::execution::B200Backend, the IComputeBackend implementation
 *    (core/execution/gpu_backend.hpp:18-51) over std::vector arguments.
 * Status codes are those of hn_sm100.h; hn_host_last_error() gives the text.
 */
#ifndef HN_HOST_H
#define HN_HOST_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* InteriorPointOptions (core/lp/interior_point.hpp:16-27) */
typedef struct hn_ipm_options {
    int max_iterations;          /* 100 */
    double time_limit_seconds;   /* 0 = none */
    double convergence_tol;      /* 1e-8 */
    double complementarity_tol;  /* 1e-8 */
    double regularization;       /* 1e-8 */
    int device;                  /* 0 */
    int verbose;                 /* 0 */
    /* interrupt_callback: polled once per iteration; nonzero stops the solve
     * with status INTERRUPTED (interior_point.cpp:490-493). May be NULL. */
    int (*interrupt_cb)(void* user);
    void* interrupt_user;
    /* Warm start (no counterpart in the reference, whose IPM always starts
     * from interior_point.cpp:443-453): x (n), y (m), s (n) in the original
     * space of the minimisation form, A^T y + s = c at a dual-feasible point;
     * y or s may be NULL. Mapped to the scaled standard form, shifted to strict
     * interiority (Mehrotra's heuristic) and used only when its relative KKT
     * residual is below the default start's. All NULL = default start. For
     * hn_lp_solve_batch the arrays are packed by the instances' col_off /
     * row_off. */
    const double* initial_x;
    const double* initial_y;
    const double* initial_s;
    /* the warm start's final shift is at least this times the default
     * start's entries (0.01) */
    double warm_start_floor;
    /* hn_lp_solve's normal-matrix factorisation on the host (the reference's
     * SparseCholesky seat): 0 auto = dense LDL^T up to 12,000 rows, sparse
     * LDL^T (AMD + supernodal, hn_sparse_ldlt_solve) above; 1 dense; 2 sparse */
    int factorization;
    /* Tightening past the reference's stop (no reference counterpart): once
     * the reference's absolute tests on the scaled form hold (the status is
     * theirs), keep iterating until the relative KKT residual of the unscaled
     * LP (hn_ipm_kkt in hn_sm100.h) is <= kkt_tol or kkt_extra_iterations more
     * iterations have run, and return the better of the two iterates.
     * kkt_tol <= 0: the reference's rule alone. Defaults 1e-8, 10. */
    double kkt_tol;
    int kkt_extra_iterations;
} hn_ipm_options;

/* InteriorPointResult (core/lp/interior_point.hpp:29-38) plus phase times;
 * status uses model::ProblemStatus numbering (core/model/problem.hpp:35-45). */
typedef struct hn_ipm_result {
    int status;
    int64_t iterations;
    double objective;
    double solve_time_ms;
    double device_ms;
    double factor_ms;
    double solve_ms;
    int64_t nnz_normal;
    int warm_start_used;  /* 1 when the warm start was taken */
    double kkt_default;   /* relative KKT residual of the default start */
    double kkt_warm;      /* ... of the shifted warm start (0 if none) */
    /* relative KKT residual of the returned iterate on the unscaled LP: the
     * max of its primal, dual and duality-gap parts (hn_ipm_kkt) */
    double kkt, kkt_primal, kkt_dual, kkt_gap;
    /* iteration at which the reference's stopping rule first held (-1: never) */
    int64_t reference_iterations;
} hn_ipm_result;

void hn_ipm_default_options(hn_ipm_options* opt);
/* min/max c^T x + obj_offset s.t. row i of A (sense 0 LE, 1 GE, 2 EQ) vs b_i,
 * lb <= x <= ub; A as CSR in the reference layout. x_out (n) may be NULL.
 * y_out (m) and s_out (n), may be NULL: the barrier's dual estimate in the
 * original space of the minimisation form (A^T y + s = c) -- an extension;
 * the reference's barrier returns no duals without crossover. */
int hn_lp_solve(int64_t m, int64_t n, const uint64_t* row_ptr, const uint64_t* col_idx, const double* val,
                const double* c, const double* b, const int* sense, const double* lb, const double* ub,
                int maximize, double obj_offset, const hn_ipm_options* opt, hn_ipm_result* res, double* x_out,
                double* y_out, double* s_out);
const char* hn_host_last_error(void);

/* K LPs solved in lockstep by the batched GPU IPM (hn::lp::BatchInteriorPointSolver).
 * Instance i: rows row_off[i]..row_off[i+1] of b/sense, columns
 * col_off[i]..col_off[i+1] of c/lb/ub/x_out, nonzeros nnz_off[i]..nnz_off[i+1]
 * of col_idx/val (column indices local to the instance), and row pointer
 * entries row_off[i]+i .. row_off[i+1]+i+1 of row_ptr (local, starting at 0).
 * Per-instance outputs: status (model::ProblemStatus), objective, iterations;
 * optional (NULL = not wanted): x_out / s_out packed by col_off, y_out by
 * row_off, warm_used (K), kkt_out (K x 4: relative KKT residual, primal, dual,
 * gap parts as hn_ipm_result's) and reference_iterations (K). */
typedef struct hn_batch_stats {
    int64_t rows, cols, nnz, nnz_normal;
    int64_t iterations;
    double total_ms, factor_ms, solve_ms;
    double forms_ms;  /* host: standard forms and start points of every instance */
    double setup_ms;  /* device matrix, A^T, A D A^T pattern and batch tables */
} hn_batch_stats;
int hn_lp_solve_batch(int64_t K, const int64_t* row_off, const int64_t* col_off, const int64_t* nnz_off,
                      const uint64_t* row_ptr, const uint64_t* col_idx, const double* val, const double* c,
                      const double* b, const int* sense, const double* lb, const double* ub, const int* maximize,
                      const double* obj_offset, const hn_ipm_options* opt, int* status, double* objective,
                      int64_t* iterations, double* x_out, hn_batch_stats* stats, int* warm_used, double* y_out,
                      double* s_out, double* kkt_out, int64_t* reference_iterations);

/* ---- MPS reader (MPSParser, core/model/mps_parser.hpp:18-78) ----
 * Reads MPS text with the reference's results: free/fixed layout (format -1
 * detects it as mps_parser.cpp:124-158 does, 0 free, 1 fixed), sections NAME,
 * OBJSENSE, ROWS, COLUMNS (integer MARKER blocks), RHS (with its fixed-layout
 * retry), RANGES, BOUNDS; SOS / QUADOBJ / QCMATRIX records are read past and
 * counted. Rows and columns are looked up by hash (first occurrence of a
 * name wins, as in the reference's linear searches). The constraint
 * coefficients come out as triplets in file order; hn_csr_create_coo makes
 * the device CSR the reference's from_triplets would make. */
typedef struct hn_mps hn_mps; /* a problem read from MPS or LP text */
int hn_mps_read_file(const char* path, int format, hn_mps** out);
int hn_mps_read_string(const char* text, int64_t len, int format, hn_mps** out);
/* ---- LP-format reader (LPParser, core/model/lp_parser.hpp:17-64) ----
 * CPLEX-style LP text with the reference's results: MIN/MAX objective
 * (bracketed quadratic groups read past; their variables still created in
 * the reference's order), SUBJECT TO constraints over one or more lines
 * (<=, >=, =), BOUNDS in its five whole-line forms, GENERAL(S), BINARY,
 * SOS and QUADRATIC sections, END. Where the reference would report errors
 * (and no problem) the call fails with HN_ERR_INVALID_ARG and the first
 * error's text. The result is read with the hn_mps_* accessors below. */
int hn_lp_read_file(const char* path, hn_mps** out);
int hn_lp_read_string(const char* text, int64_t len, hn_mps** out);
/* m rows (constraints), n columns, triplet count, objective sense (1 = MAX) */
int hn_mps_shape(const hn_mps* h, int64_t* m, int64_t* n, int64_t* ntriplets, int* maximize);
/* Copies out (each may be NULL): triplets (ntriplets), c / lb / ub / vtype
 * (n; vtype in model::VarType numbering), rhs / sense (0 LE, 1 GE, 2 EQ) /
 * range_lo / range_hi (m). */
int hn_mps_arrays(const hn_mps* h, int64_t* trow, int64_t* tcol, double* tval, double* c, double* rhs,
                  int32_t* sense, double* lb, double* ub, double* range_lo, double* range_hi, int32_t* vtype);
int hn_mps_counts(const hn_mps* h, int64_t* warnings, int64_t* sos_records, int64_t* quadratic_records);
const char* hn_mps_warning(const hn_mps* h, int64_t i);
/* what -1: problem name; 0: row i's name; 1: column i's name (NULL if none) */
const char* hn_mps_name(const hn_mps* h, int what, int64_t i);
int hn_mps_free(hn_mps* h);

/* ---- sparse LDL^T (the SparseCholesky interface, core/numerical/factorization.hpp:162-208) ----
 * Approximate minimum degree ordering, supernodes, multifrontal numerics
 * with the reference's pivot clamp (d <= singular_tol -> singular_tol,
 * factorization.cpp:1310-1313). The matrix is given in CSR with both
 * triangles (the IPM's normal-matrix layout). hn_amd_order returns the
 * ordering alone (perm[new] = old); hn_sparse_ldlt_solve analyses,
 * factorises and solves nrhs right-hand sides in place (x: nrhs x m). */
typedef struct hn_sparse_ldlt_stats {
    int64_t nnz_L;       /* strictly lower entries of L */
    int64_t supernodes;
    int singular;        /* a pivot was clamped */
    double analyze_ms, factor_ms;
} hn_sparse_ldlt_stats;
int hn_amd_order(int64_t m, const uint64_t* rp, const uint64_t* ci, int64_t* perm);
int hn_sparse_ldlt_solve(int64_t m, const uint64_t* rp, const uint64_t* ci, const double* val, double singular_tol,
                         int64_t nrhs, double* x, hn_sparse_ldlt_stats* stats);

/* ---- crossover seam (InteriorPointSolver::solve, interior_point.cpp:792-876) ----
 * The warm basis the reference's crossover hands SimplexSolver::
 * solve_with_basis (simplex.hpp:64), computed from a barrier endpoint x
 * (e.g. hn_lp_solve's x_out) and the variable bounds: var_status[j] = -1 at
 * lower bound, +1 at upper bound, 0 basic candidate, by the reference's rule
 * (tolerance 1e-6 (1 + max(|lb|, |ub|)), lower tested first). The simplex
 * polish itself stays the caller's (host) code. */
int hn_crossover_basis(int64_t n, const double* x, const double* lb, const double* ub, int* var_status);

/* B200Backend through C: the matrix arrives as the reference's three vectors
 * each call; the backend keeps it resident between calls. */
typedef struct hn_backend hn_backend;
int hn_be_create(int device, hn_backend** out);
int hn_be_destroy(hn_backend* be);
int hn_be_spmv(hn_backend* be, int64_t m, int64_t nnz, const uint64_t* rp, const uint64_t* ci, const double* val,
               int64_t nx, const double* x, double* y);
int hn_be_spmv_t(hn_backend* be, int64_t m, int64_t n, int64_t nnz, const uint64_t* rp, const uint64_t* ci,
                 const double* val, const double* x, double* y);
int hn_be_spmm(hn_backend* be, int64_t m, int64_t nnz, const uint64_t* rp, const uint64_t* ci, const double* val,
               int64_t nb, const double* B, int64_t k, double* C);
int hn_be_dot(hn_backend* be, int64_t n, const double* a, const double* b, double* out);
int hn_be_axpy(hn_backend* be, int64_t n, double alpha, const double* x, double* y);
int hn_be_norm_inf(hn_backend* be, int64_t n, const double* v, double* out);
int hn_be_kernel_executions(hn_backend* be, uint64_t* out);

#ifdef __cplusplus
}
#endif
#endif
