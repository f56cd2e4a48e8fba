/* hn_sm100 -- B200 (sm_100a) FP64 sparse linear algebra for the HyperNova LP
 * solvers, exported as a plain C ABI.
 *
 * This library replaces the GPU half of HyperNova's compute backend: the
 * dlopen'ed CUDA driver loader (core/execution/cuda_driver.cpp:24-56,112-147),
 * the embedded sm_50 PTX kernels (core/execution/cuda_kernels_ptx.cpp:21-378)
 * and the device work of CudaDriverBackend (core/execution/gpu_backend.cpp:141-617),
 * and moves on to the device the host loops of the IPM hot path
 * (core/lp/interior_point.cpp:52-69,134-200,507-696).
 *
 * Conventions
 *  - Every entry point returns an int status (HN_OK == 0). On failure the
 *    thread-local message from hn_last_error() says why. No C++ exception
 *    crosses this boundary. There is no CPU fallback: a call that cannot run
 *    on the GPU fails.
 *  - Matrix arguments are CSR arrays in the reference's layout: row_ptr and
 *    col_idx as 64-bit unsigned (std::size_t), values as double.
 *    Device storage is int32 indices; nnz, m and n must each be < 2^31.
 *  - Pointers named *_dev are device pointers; *_host are host pointers.
 *    `stream` is a cudaStream_t passed as void* (NULL = legacy default stream).
 *  - Products and reductions on one handle must not overlap on the GPU
 *    (each handle owns its merge-path carry buffers); reductions issued on
 *    one stream are serialised by that stream's workspace.
 *  - Reductions (dot, norms, maxima) are deterministic: the same inputs on the
 *    same device give the same bits on every run.
 */
#ifndef HN_SM100_H
#define HN_SM100_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---- */
#define HN_OK 0
#define HN_ERR_INVALID_ARG 1
#define HN_ERR_CUDA 2
#define HN_ERR_OUT_OF_MEMORY 3
#define HN_ERR_NOT_INITIALIZED 4
#define HN_ERR_UNSUPPORTED 5
#define HN_ERR_NUMERICAL 6
#define HN_ERR_INJECTED 7

/* ---- hn_csr_create flags ---- */
#define HN_CSR_NO_TRANSPOSE 1u /* do not build the device A^T */
#define HN_CSR_NO_AUTOTUNE 2u  /* keep the merge-path SpMV without timing the alternatives */

typedef struct hn_csr hn_csr;         /* device-resident CSR matrix (+ its A^T) */
typedef struct hn_pattern hn_pattern; /* fixed pattern of A diag(d) A^T + reg I */

typedef struct hn_device_info_t {
    char name[256];
    int device;
    int sm_count;
    int cc_major;
    int cc_minor;
    size_t total_mem;
    size_t free_mem;
} hn_device_info_t;

/* ---- lifecycle ----
 * hn_init replaces CudaDriverBackend::initialize (gpu_backend.cpp:159-192) and
 * DriverApi::load/init_context (cuda_driver.cpp:112-147,204-236): binds the
 * calling thread to `device` (primary context). Fails with
 * HN_ERR_UNSUPPORTED unless the device is compute capability 10.0. */
int hn_init(int device);
/* Releases per-stream workspaces. Handles must be destroyed first.
 * (CudaDriverBackend::finalize, gpu_backend.cpp:194-198) */
int hn_shutdown(void);
/* Thread-local text of the last failure (CudaDriverBackend::last_error_). */
const char* hn_last_error(void);
/* Device name and memory (CudaDriverBackend::name/device_memory/free_memory,
 * gpu_backend.cpp:150-153,249-259). */
int hn_device_info(hn_device_info_t* out);
/* Kernel launch counter (IComputeBackend::gpu_kernel_executions,
 * gpu_backend.hpp:47-50). */
int hn_stats(uint64_t* kernel_launches, uint64_t* api_calls);
int hn_reset_stats(void);
/* Host-side fault injection for failure tests: after `after_calls` further
 * API calls, the next call returns `status` without touching the GPU.
 * after_calls < 0 disarms. No reference counterpart (the reference has no
 * fault injection); it lets tests reach every error path without a GPU fault. */
int hn_fault_inject(int64_t after_calls, int status);

/* ---- device memory for callers without a CUDA runtime ----
 * (DriverApi::allocate/free/copy_h2d/copy_d2h/memset_d8, cuda_driver.hpp:44-93) */
int hn_malloc(void** ptr_dev, size_t bytes);
int hn_free(void* ptr_dev);
int hn_memcpy_h2d(void* dst_dev, const void* src_host, size_t bytes, void* stream);
int hn_memcpy_d2h(void* dst_host, const void* src_dev, size_t bytes, void* stream);
int hn_memcpy_d2d(void* dst_dev, const void* src_dev, size_t bytes, void* stream);
int hn_memset(void* ptr_dev, int byte, size_t bytes, void* stream);
int hn_stream_sync(void* stream);

/* ---- CSR matrices ----
 * Uploads A (host arrays, reference layout) once and builds on the device:
 * int32 indices, the merge-path tile table (row binning) and, unless
 * HN_CSR_NO_TRANSPOSE, A^T as its own CSR. A^T equals the reference's
 * SparseMatrix::transposed() bit for bit (sparse_matrix.cpp:84-96): entries
 * ordered by (column,row), equal keys summed in input order, exact zero sums
 * dropped. Replaces CudaDriverBackend::upload_matrix/resident_matrix
 * (gpu_backend.cpp:289-306,360-393) with an explicit handle. */
int hn_csr_create(int64_t m, int64_t n, const uint64_t* row_ptr_host,
                  const uint64_t* col_idx_host, const double* val_host, unsigned flags,
                  hn_csr** out);
/* A from `count` triplets (host arrays; rows in [0, m), cols in [0, n), any
 * order, duplicates allowed), built on the device with the semantics of
 * SparseMatrix::from_triplets (sparse_matrix.cpp:8-53, sum_duplicates
 * :230-262): entries ordered by (row, column), equal (row, column) entries
 * summed in input order, exact-zero sums dropped -- the matrix MPSParser
 * assembles from its coefficient list (mps_parser.cpp:106-111). Two stable
 * radix passes on the device, then the same set-up as hn_csr_create. */
int hn_csr_create_coo(int64_t m, int64_t n, int64_t count, const int64_t* rows_host, const int64_t* cols_host,
                      const double* val_host, unsigned flags, hn_csr** out);
/* New values for the same pattern (host array, nnz entries); A^T follows. */
int hn_csr_set_values(hn_csr* A, const double* val_host);
int hn_csr_destroy(hn_csr* A);
int hn_csr_shape(const hn_csr* A, int64_t* m, int64_t* n, int64_t* nnz, int64_t* nnz_t);
/* Host copy of A (trans=0) or A^T (trans=1) in the reference layout.
 * rp: rows+1 entries; ci/val: nnz entries. */
int hn_csr_export(const hn_csr* A, int trans, uint64_t* rp_host, uint64_t* ci_host,
                  double* val_host);
/* Merge-path tile table (row binning) of A or A^T: ntiles+1 coordinates. */
/* SpMV path of a direction (trans 0: A, 1: A^T). HN_SPMV_MERGE: merge-path
 * tiles (the default, any row-length distribution). HN_SPMV_BINNED: rows
 * grouped by length, a group of 2^k lanes per row sized for about t nonzeros
 * per lane. hn_csr_create times both (t = 4, 8, 16) on matrices with >= 2^20
 * nonzeros per direction and keeps the binned kernel when it is >= 5 % faster
 * (unless HN_CSR_NO_AUTOTUNE). Both sum each row in a fixed order; they
 * differ from each other by rounding only. This is the reference's row binning
 * (one kernel per matrix chosen by mean row length, gpu_backend.cpp:413-415)
 * made per matrix and measured. */
#define HN_SPMV_MERGE 0
#define HN_SPMV_BINNED 1
int hn_csr_spmv_kind(const hn_csr* A, int trans, int* kind, int* t);
int hn_csr_set_spmv_kind(hn_csr* A, int trans, int kind, int t);
int hn_csr_tiles(const hn_csr* A, int trans, int64_t* ntiles, int64_t* items_per_tile);
int hn_csr_export_tiles(const hn_csr* A, int trans, int32_t* tile_row_host,
                        int32_t* tile_nz_host);

/* ---- products ----
 * y = alpha*op(A)*x + beta*y, op(A) = A (trans=0) or A^T (trans=1).
 * beta == 0 never reads y. Replaces IComputeBackend::spmv
 * (gpu_backend.hpp:30-34; CudaDriverBackend::launch_spmv gpu_backend.cpp:395-443)
 * and, for trans=1, SparseMatrix::transpose_multiply / the IPM's matvec_t
 * (sparse_matrix.cpp:161-184, interior_point.cpp:61-69). */
int hn_spmv(const hn_csr* A, int trans, double alpha, const double* x_dev, double beta,
            double* y_dev, void* stream);
/* y = op(A) x - b in one pass (the IPM's primal residual rp = M x - b,
 * interior_point.cpp:512); y may not alias b. */
int hn_spmv_residual(const hn_csr* A, int trans, const double* x_dev, const double* b_dev, double* y_dev,
                     void* stream);
/* Same product with host vectors, synchronous: copies x in and y out through
 * pinned staging (IComputeBackend::spmv's calling convention). */
int hn_spmv_host(const hn_csr* A, int trans, const double* x_host, double* y_host);
/* C = op(A) * B with B row-major (cols(op A) x k) and C (rows(op A) x k)
 * overwritten (IComputeBackend::spmm, gpu_backend.hpp:36-41, gpu_backend.cpp:445-487). */
int hn_spmm(const hn_csr* A, int trans, const double* B_dev, int64_t k, double* C_dev,
            void* stream);
int hn_spmm_host(const hn_csr* A, int trans, const double* B_host, int64_t k, double* C_host);

/* ---- BLAS-1 on device vectors; scalar results go to a device double ----
 * (IComputeBackend::dot/axpy/norm_inf, gpu_backend.hpp:43-45; the reference's
 * CUDA path ran these on the host, gpu_backend.cpp:236-248) */
int hn_dot(int64_t n, const double* a_dev, const double* b_dev, double* result_dev,
           void* stream);
int hn_axpy(int64_t n, double alpha, const double* x_dev, double* y_dev, void* stream);
/* max |v_i|, NaN entries ignored (std::max semantics of the reference). */
int hn_nrm_inf(int64_t n, const double* v_dev, double* result_dev, void* stream);
int hn_nrm2(int64_t n, const double* v_dev, double* result_dev, void* stream);

/* ---- normal equations N = A diag(d) A^T + dyn_reg I ----
 * (build_normal_equations, interior_point.cpp:144-200)
 * Symbolic: the pattern of A A^T plus the full diagonal, both triangles,
 * columns sorted (the pattern the reference builds when every d_j > 0).
 * Needs the handle's A^T. Each row of N may reach at most 400,000 columns
 * (the span from its smallest to its largest k; block-diagonal batches are
 * limited by their largest block only), and nnz(N) < 2^31. */
int hn_ada_symbolic(const hn_csr* A, hn_pattern** out);
/* The numeric phase has three layouts with bit-identical results.
 *  - Gather mode keeps an 8-byte source pair (A^T entry, A entry) per slot
 *    of N; one thread per slot, in slot order. The default unless the
 *    relative map is.
 *  - Relative map, used when the offsets fit 32 bits (longest row of A x
 *    longest row of A^T < 2^31) and every row of A has <= 256 entries, and
 *    either HN_ADA_RELATIVE asks for it or the rows of N average >= 2,048
 *    slots (without HN_ADA_COMPACT): 4 bytes per slot, the single term's
 *    entry within its row of A and within its row of A^T (or the slot's
 *    index among its row's multi-term slots); one warp per row of N, longest
 *    rows first, the row's A entries staged in shared memory. Half the map
 *    memory, 5 % faster than gather mode on the 200k x 500k LP.
 *    HN_ADA_GATHER8 asks for gather mode.
 *  - Row mode, asked for with HN_ADA_COMPACT and used when every row of N has
 *    <= 65,534 slots and every row of A <= 256 entries, keeps a 2-byte slot
 *    offset per term and assembles each row of N in shared-memory windows. */
#define HN_ADA_COMPACT 1u
#define HN_ADA_GATHER8 2u
#define HN_ADA_RELATIVE 4u
int hn_ada_symbolic_ex(const hn_csr* A, unsigned flags, hn_pattern** out);
/* row_mode: 0 gather mode, 1 row mode, 2 relative map; max_row: longest row of N. */
int hn_pattern_mode(const hn_pattern* P, int* row_mode, int64_t* max_row);
int hn_pattern_info(const hn_pattern* P, int64_t* m, int64_t* nnz);
/* Host copy of the pattern: rp m+1, ci nnz (reference layout). */
int hn_pattern_export(const hn_pattern* P, uint64_t* rp_host, uint64_t* ci_host);
/* Device arrays of the pattern: rp (int64, m+1), ci (int32, nnz), diag_pos
 * (int64, m: position of (i,i) in ci). */
int hn_pattern_device(const hn_pattern* P, const int64_t** rp_dev, const int32_t** ci_dev,
                      const int64_t** diag_pos_dev);
/* Numeric: nval_dev[p] for every pattern position; columns with d_j <= 0 add
 * nothing (their entries stay explicit zeros); each term is
 * (a_ij * a_kj) * d_j, summed per entry in column order; the diagonal then
 * gains dyn_reg = max(reg, 1e-12 * max_i sum_j a_ij^2 d_j). dyn_reg_dev
 * (device double, may be NULL) receives dyn_reg. */
int hn_ada_numeric(const hn_pattern* P, const double* d_dev, double reg, double* nval_dev,
                   double* dyn_reg_dev, void* stream);
int hn_pattern_destroy(hn_pattern* P);

/* ---- Mehrotra predictor-corrector iteration kernels ----
 * (InteriorPointSolver::solve's loop, core/lp/interior_point.cpp:507-708)
 * Device scalar block: double scal[HN_IPM_NSCAL]; the FLAGS slot holds uint64
 * bits (1: a direction or dlam entry is not finite, :617-627 / :676-686;
 * 2: the updated x or z has a negative or non-finite entry, :698-708). */
#define HN_IPM_NRP 0   /* ||M x - b||_inf */
#define HN_IPM_NRD 1   /* ||M^T lam + z - c||_inf */
#define HN_IPM_MU 2    /* x^T z / n */
#define HN_IPM_AP 3    /* primal step length */
#define HN_IPM_AD 4    /* dual step length */
#define HN_IPM_MUAFF 5 /* affine complementarity */
#define HN_IPM_SIGMA 6 /* centring parameter */
#define HN_IPM_FLAGS 7
#define HN_IPM_NSCAL 8

/* mx = M x; rp = mx - b; rd = M^T lam + z - c; then mu, ||rp||_inf,
 * ||rd||_inf into scal, D = x / z clamped to (0, 1e10] and Drd = D rd
 * (:507-539, :584). All vectors device, n = cols, m = rows. FLAGS bits are
 * sticky: the caller clears the slot before a solve. */
int hn_ipm_residuals(const hn_csr* M, const double* x_dev, const double* lam_dev, const double* z_dev,
                     const double* b_dev, const double* c_dev, double* mx_dev, double* rp_dev,
                     double* rd_dev, double* D_dev, double* Drd_dev, double* scal_dev, void* stream);
/* rhs = -rp - M Drd + mx (normal-equation right-hand side, :585-600). */
int hn_ipm_rhs(const hn_csr* M, const double* Drd_dev, const double* rp_dev, const double* mx_dev,
               double* rhs_dev, void* stream);
/* t = M^T dlam; dx = D (t + rd) - x (+ corr if non-null); dz = -(t + rd)
 * (:607-615 predictor, :666-673 corrector). */
int hn_ipm_direction(const hn_csr* M, const double* dlam_dev, const double* D_dev, const double* rd_dev,
                     const double* x_dev, const double* corr_dev, double* dx_dev, double* dz_dev,
                     void* stream);
/* scal[AP] = max_step(x, dx), scal[AD] = max_step(z, dz) (:134-142) and the
 * non-finite guard over dx, dz (n) and dlam (m) into FLAGS bit 1. */
int hn_ipm_step_lengths(int64_t n, int64_t m, const double* x_dev, const double* dx_dev,
                        const double* z_dev, const double* dz_dev, const double* dlam_dev,
                        double* scal_dev, void* stream);
/* mu_aff and sigma from the current steps (:632-643), zs = (sigma mu - dx dz)
 * * (1/z) (:645-651) and rhs = rhs_pred - M zs (:652-659). */
int hn_ipm_corrector(const hn_csr* M, const double* x_dev, const double* dx_dev, const double* z_dev,
                     const double* dz_dev, const double* rhs_pred_dev, double* zs_dev, double* rhs_dev,
                     double* scal_dev, void* stream);
/* x += ap dx; z += ad dz; lam += ad dlam; guard into FLAGS bit 2 (:690-708). */
int hn_ipm_update(int64_t n, int64_t m, double* x_dev, const double* dx_dev, double* z_dev,
                  const double* dz_dev, double* lam_dev, const double* dlam_dev, double* scal_dev,
                  void* stream);
/* Relative KKT residual of an iterate on the LP with the standard form's row
 * and column scaling undone. No reference counterpart: the reference stops on
 * absolute tests of the scaled form (interior_point.cpp:525-530) and never
 * measures this; it is the accuracy measure of the solves/s metric.
 *   P = max_i |rp_i| ru_i / (1 + max_i |b_i| ru_i)
 *   D = max_j |rd_j| cu_j / (1 + max_j |c_j| cu_j)
 *   G = |c^T x - b^T lam| / (1 + |c^T x + offset|)
 * kkt_dev[0..3] = max(P, D, G), P, D, G (a non-finite residual entry makes
 * its part infinite). rp = M x - b, rd = M^T lam + z - c as hn_ipm_residuals
 * leaves them for the same (x, lam, z); ru_i = 1 / |scale of row i|, cu_j =
 * 1 / (scale of column j), offset = the objective's constant. For an LP given
 * as min c^T x, A x = b, x >= 0 this is max(||Ax-b||/(1+||b||),
 * ||A^T y + s - c||/(1+||c||), |c^T x - b^T y|/(1+|c^T x|)) (inf-norms) of the
 * original LP at x, y = row-scaled lam, s = column-unscaled z. */
int hn_ipm_kkt(int64_t n, int64_t m, const double* x_dev, const double* lam_dev, const double* b_dev,
               const double* c_dev, const double* rp_dev, const double* rd_dev, const double* ru_dev,
               const double* cu_dev, double offset, double* kkt_dev, void* stream);
/* *result_dev = min(1, 0.99 * min_{d_i<0} -v_i/d_i) (max_step, :134-142). */
int hn_max_step(int64_t n, const double* v_dev, const double* d_dev, double* result_dev, void* stream);

/* ---- batched Mehrotra IPM (many LPs advanced in lockstep) ----
 * The instances are packed as one block-diagonal matrix: instance i owns rows
 * row_off[i]..row_off[i+1] and columns col_off[i]..col_off[i+1] of M (an
 * hn_csr with A^T) and the matching block of P = hn_ada_symbolic(M). The
 * SpMV-based kernels above (hn_ipm_rhs, hn_ipm_direction) run unchanged on
 * the packed vectors; these entry points add what is per instance. `scal`
 * is double[K * HN_IPM_NSCAL] (one scalar block per instance), `status`
 * int32[K] (0 = iterating, else a model::ProblemStatus value: 1 converged,
 * 7 numerical error) and `iters` int32[K]; a non-zero status masks the
 * instance out of the factorisation, solves and update. No reference
 * counterpart exists (the reference solves one LP at a time,
 * interior_point.cpp:402-886); each step restates the lines cited in the
 * single-LP kernels. The normal equations are factorised on the GPU (dense
 * blocked LDL^T per instance, pivot clamp of factorization.cpp:1299-1305). */
typedef struct hn_batch hn_batch;
int hn_batch_create(int64_t K, const int64_t* row_off_host, const int64_t* col_off_host, const hn_pattern* P,
                    hn_batch** out);
int hn_batch_destroy(hn_batch* B);
/* rp = M x - b, rd = M^T lam + z - c, per-instance mu / norms, D, Drd; an
 * iterating instance that meets the tolerances becomes status 1 with
 * iters = iter (:507-539). */
int hn_batch_residuals(hn_batch* B, const hn_csr* M, const double* x_dev, const double* lam_dev,
                       const double* z_dev, const double* b_dev, const double* c_dev, double* mx_dev, double* rp_dev,
                       double* rd_dev, double* D_dev, double* Drd_dev, double* scal_dev, int32_t* status_dev,
                       int32_t* iters_dev, int iter, double tol, double ctol, void* stream);
/* Relative KKT residual per instance and tightening past the reference's
 * stop (no reference counterpart). With ru_dev / cu_dev (per packed row /
 * column, as hn_ipm_kkt) and offset_dev (K) set, every hn_batch_residuals
 * call measures each instance's residual as hn_ipm_kkt does. With
 * kkt_tol > 0, an instance that meets the reference's rule has that iterate
 * saved and keeps iterating until its residual is <= kkt_tol or
 * extra_iterations more iterations have run; hn_batch_finish then puts the
 * saved iterate back where the later one is worse or failed. kkt_tol <= 0:
 * the reference's rule alone (the residual is still measured when ru_dev is
 * given). The arrays are caller-owned and must stay valid while the batch
 * iterates. Resets the per-instance records. */
int hn_batch_set_kkt(hn_batch* B, const double* ru_dev, const double* cu_dev, const double* offset_dev,
                     double kkt_tol, int extra_iterations);
/* kkt_host: K x 4 (as hn_ipm_kkt's kkt_dev) at the last hn_batch_residuals
 * call, or after hn_batch_finish the residual of the returned iterate;
 * ref_iter_host: K, the iteration at which the reference's rule first held
 * (-1: never). Either may be NULL. Synchronises the device. */
int hn_batch_kkt(const hn_batch* B, double* kkt_host, int32_t* ref_iter_host);
/* Call after the last hn_batch_residuals: every instance that met the
 * reference's rule becomes status 1; where it then failed (status 7), or its
 * residual is larger than when the rule first held, it gets that iterate back
 * (x, z, lam), iters = that iteration and that residual. */
int hn_batch_finish(hn_batch* B, double* x_dev, double* z_dev, double* lam_dev, int32_t* status_dev,
                    int32_t* iters_dev, void* stream);
/* N = A D A^T + dyn_reg_i I per instance (:144-200), then the dense LDL^T of
 * every iterating instance. nval_dev: nnz(P) doubles. */
int hn_batch_factor(hn_batch* B, const double* D_dev, double reg, double singular_tol, double* nval_dev,
                    const int32_t* status_dev, void* stream);
/* x = N^-1 rhs per iterating instance, with iterative refinement against N
 * (refinement.cpp:7-37: <= 5 sweeps, 1e-10 relative). */
int hn_batch_solve(hn_batch* B, const double* nval_dev, const double* rhs_dev, double* x_dev,
                   const int32_t* status_dev, void* stream);
/* per-instance step lengths (:134-142) and non-finite guard (:617-627). */
int hn_batch_steps(hn_batch* B, const double* x_dev, const double* dx_dev, const double* z_dev,
                   const double* dz_dev, const double* dlam_dev, double* scal_dev, int32_t* status_dev, void* stream);
/* per-instance mu_aff, sigma, zs, then rhs = rhs_pred - M zs (:632-659). */
int hn_batch_corrector(hn_batch* B, const hn_csr* M, const double* x_dev, const double* dx_dev, const double* z_dev,
                       const double* dz_dev, const double* rhs_pred_dev, double* zs_dev, double* rhs_dev,
                       double* scal_dev, const int32_t* status_dev, void* stream);
/* x += ap dx, z += ad dz, lam += ad dlam for iterating instances; iters = iter+1,
 * or status 7 on a negative / non-finite iterate (:690-708). */
int hn_batch_update(hn_batch* B, double* x_dev, const double* dx_dev, double* z_dev, const double* dz_dev,
                    double* lam_dev, const double* dlam_dev, const double* scal_dev, int32_t* status_dev,
                    int32_t* iters_dev, int iter, void* stream);

/* ---- revised-simplex pricing (core/lp/simplex.cpp) ----
 * The per-iteration O(nnz + n) pricing work of SimplexSolver over the
 * matrix's device A^T; FTRAN/BTRAN (the basis factorisation) stay on the host.
 * All vectors are device pointers of the matrix's sizes. */

/* rc = cost - A^T y, bit-identical to compute_reduced_costs
 * (simplex.cpp:1225-1233) through SparseMatrix::transpose_multiply. */
int hn_price_reduced_costs(const hn_csr* A, const double* y_dev, const double* cost_dev, double* rc_dev,
                           void* stream);
/* Devex reference-framework update of update_devex_weights
 * (simplex.cpp:1235-1271): alpha = A^T u (u = e_leaving^T B^-1 from the
 * host's BTRAN, written to alpha_dev, n doubles), s = max |alpha_j| over
 * nonbasic j (nonbasis_dev[j] >= 0), and, when s != 0, for nonbasic j
 * w_j = max(w_j, (alpha_j / s)^2). */
int hn_price_devex_update(const hn_csr* A, const double* u_dev, const int32_t* nonbasis_dev, double* weights_dev,
                          double* alpha_dev, void* stream);

#define HN_PRICE_BLAND 0  /* first improving column (bland_rule, simplex.cpp:1328-1338) */
#define HN_PRICE_RANKED 1 /* |rc|/sqrt(w) descending, index ascending (ranked_candidates, :1283-1308) */
#define HN_PRICE_MAX_K 64
/* Entering-column choice of select_entering_variable (simplex.cpp:1321-1361).
 * Column j is improving when nonbasis[j] >= 0, it is not artificial
 * (artificial_dev[j] == 0, or phase1 != 0, or artificial_dev NULL) and
 * rc' < -optimality_tol with rc' = maximize ? -rc_j : rc_j. Writes to out_dev
 * (device, k + 1 int64): out[0] = number of improving columns; for
 * HN_PRICE_BLAND out[1] = the lowest improving index or -1; for
 * HN_PRICE_RANKED (1 <= k <= HN_PRICE_MAX_K) out[1..k] = the first k of
 * ranked_candidates' order (score |rc'|/sqrt(w_j), w_j replaced by 1 when not
 * finite and positive, weights_dev NULL meaning all 1; ties by lower index),
 * -1 past the end. Reduced costs must not be NaN (the reference's ordering
 * is undefined there). */
int hn_price_select(int64_t n, const double* rc_dev, const double* weights_dev, const int32_t* nonbasis_dev,
                    const uint8_t* artificial_dev, int phase1, int maximize, double optimality_tol, int rule,
                    int64_t k, int64_t* out_dev, void* stream);
/* Dense columns cols[r] of A into out (device, m x k column-major), the
 * vectors extract_column (simplex.cpp:25-35) builds for the ratio test and
 * exact steepest-edge weights. Indices outside [0, n) leave their column zero
 * and make the call fail with HN_ERR_INVALID_ARG (the call synchronises the
 * stream to report it). */
int hn_price_columns(const hn_csr* A, int64_t k, const int64_t* cols_dev, double* out_dev, void* stream);

/* ---- GNN warm start (no counterpart in the reference) ----
 * Kernels of a bipartite variable-constraint network with hidden width 64
 * whose prediction warm-starts the IPM. Activations are FP32 row-major
 * (rows x 64); GEMM operands are rounded to BF16 (round to nearest even) and
 * multiplied on the tensor cores with FP32 accumulation. Weights: FP32
 * masters W (K x 64 row-major); hn_gnn_cast_weights makes the BF16 copies
 * Wt (64 x K) used by hn_gnn_linear and Wb (K x 64) used by the backward. */
/* out (rows x 64) = A H (trans 0; H n x 64) or A^T H (trans 1; H m x 64);
 * A's values rounded to FP32; out += when accumulate != 0. */
int hn_gnn_spmm(const hn_csr* A, int trans, const float* H_dev, float* out_dev, int accumulate, void* stream);
int hn_gnn_cast_weights(int K, const float* W_dev, void* Wt_bf16_dev, void* Wb_bf16_dev, void* stream);
/* Y (M x N) = act([X1 | X2] W + bias); K1, K2 multiples of 16, K1 + K2 <= 128
 * (<= 64 when N = 128); N = 64 or 128; relu != 0 applies max(., 0); X2 and
 * bias may be NULL (K2 = 0 / no bias). */
int hn_gnn_linear(int64_t M, int K1, int K2, const float* X1_dev, const float* X2_dev, const void* Wt_bf16_dev,
                  int N, const float* bias_dev, int relu, float* Y_dev, void* stream);
/* hn_gnn_linear with N = 64 on the 5th-generation tensor cores: tcgen05.mma
 * (kind::f16, BF16 operands from shared memory, FP32 accumulator in tensor
 * memory); a persistent CTA per SM streams 128-row tiles of X in by bulk
 * copy. X1, X2, Y and Wt must be 16-byte aligned. Same operand rounding as
 * hn_gnn_linear; results differ from it only by accumulation order. A wait
 * that times out leaves Y undefined and sets the stream's flag, which
 * hn_gnn_check reports (HN_ERR_CUDA) and clears; hn_gnn_check synchronises
 * the stream. */
int hn_gnn_linear_umma(int64_t M, int K1, int K2, const float* X1_dev, const float* X2_dev, const void* Wt_bf16_dev,
                       const float* bias_dev, int relu, float* Y_dev, void* stream);
int hn_gnn_check(void* stream);
/* Test hook of the bounded waits above (no reference counterpart): the
 * pipeline waits of the tcgen05 kernels (the layer and both GEMMs of its
 * backward: bulk copies in, MMA done) give up after
 * `polls` non-blocking mbarrier polls instead of 2^24 blocking ones (0
 * restores the default). A call with a small limit gives up while its own
 * copies are in flight; the CTA then
 * records the timeout, settles those copies and its MMA with the full bound,
 * frees TMEM and returns, and hn_gnn_check reports the error. Process-wide;
 * for tests only. */
int hn_gnn_set_wait_limit(uint32_t polls);
/* Backward of hn_gnn_linear with N = 64: G = dY * relu'(Y); dX (M x K, may be
 * NULL; K = 64 or 128) = G W^T; dW (K x 64) = [X1 | X2]^T G; db (64) = sum of
 * G's rows. dX and dW run on the tcgen05 tensor cores (BF16 operands, FP32
 * accumulation in tensor memory; dW as one partial per persistent CTA,
 * summed in a fixed order). scratch: >= min(ceil(M / 64), SM count) *
 * (64 K + 64) floats. X1, X2, G, dX, Wb and scratch 16-byte aligned.
 * Deterministic on a given GPU. A timed-out wait sets the flag that
 * hn_gnn_check reports. */
int hn_gnn_linear_bwd(int64_t M, int K1, int K2, const float* X1_dev, const float* X2_dev, const void* Wb_bf16_dev,
                      const float* Y_dev, const float* dY_dev, int relu, float* G_dev, float* dX_dev, float* dW_dev,
                      float* db_dev, float* scratch_dev, int64_t scratch_floats, void* stream);
/* dH (M x 64) += dX[:, :64]; dAgg (M x 64) = dX[:, 64:] (dX M x 128). */
int hn_gnn_split_grad(int64_t M, const float* dX_dev, float* dH_dev, float* dAgg_dev, void* stream);
/* dO (M x 64) = scale * 2 (O - T) in the first nt columns (T: M x 2), 0 in the
 * others; loss_part (nparts floats): per-block sums of the squared errors. */
int hn_gnn_head_grad(int64_t M, const float* O_dev, const float* T_dev, int nt, float scale, float* dO_dev,
                     float* loss_part_dev, int64_t nparts, void* stream);
/* Adam (bias-corrected, step >= 1) on FP32 weights. */
int hn_gnn_adam(int64_t len, float* w_dev, const float* g_dev, float* m1_dev, float* m2_dev, float lr, float beta1,
                float beta2, float eps, int64_t step, void* stream);

/* ---- SpMV for callers that cannot allocate device memory ----
 * No counterpart in the reference. y = A x with A given as device CSR arrays
 * (int32 row_ptr m+1, int32 col_idx and double values nnz, row_ptr[m] == nnz,
 * column indices < n -- not checked on the device). It allocates nothing:
 * the merge-path tile table and carries live in one fixed 2 MB __device__
 * array, which bounds m + nnz to 117,440,512 (larger sizes fail with
 * HN_ERR_INVALID_ARG). It is for callers whose device memory belongs to
 * another allocator or that must not call cudaMalloc inside a solve loop.
 * The first call on a device looks up the array's address
 * (cudaGetSymbolAddress); make that first call before any stream capture.
 * All calls share the array: calls that overlap on the GPU race. */
int hn_spmv_noalloc(int64_t m, int64_t n, int64_t nnz, const int32_t* row_ptr_dev, const int32_t* col_idx_dev,
                    const double* val_dev, const double* x_dev, double* y_dev, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* HN_SM100_H */
