/* CPU restatement of the HyperNova sparse hot path (TEST INFRASTRUCTURE ONLY).
 *
 * This is the oracle the tests, smoke() and bench.py's CPU leg check the
 * sm_100a library against. It is never linked into or called by the product.
 * Each function names the reference file:line whose algorithm it restates;
 * it is pinned against the reference itself (oracle/_ref/libhnref.so, built
 * from the reference's own sources) and against committed golden fixtures.
 *
 * Index arrays are int64 (the reference's std::size_t) unless stated.
 */
#ifndef HN_ORACLE_H
#define HN_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* y = A x, left-to-right per row from 0.0 (sparse_matrix.cpp:136-159). */
void hno_csr_multiply(int64_t m, const int64_t* rp, const int64_t* ci, const double* val,
                      const double* x, double* y);
/* y = A^T x by row scatter, skipping x_i == 0 (sparse_matrix.cpp:161-184). */
void hno_csr_tmultiply(int64_t m, int64_t n, const int64_t* rp, const int64_t* ci,
                       const double* val, const double* x, double* y);
/* y = A^T x by row scatter without the zero skip (interior_point.cpp:61-69). */
void hno_matvec_t(int64_t m, int64_t n, const int64_t* rp, const int64_t* ci,
                  const double* val, const double* x, double* y);
/* A^T as CSR: entries ordered by (col,row) keeping input order among equal
 * keys, duplicates summed in that order, exact zero sums dropped
 * (sparse_matrix.cpp:84-96 via to_triplets, from_triplets :8-53 and
 * sum_duplicates :230-262). Returns nnz(A^T). rpT: n+1, ciT/valT: nnz(A). */
int64_t hno_csr_transposed(int64_t m, int64_t n, const int64_t* rp, const int64_t* ci,
                           const double* val, int64_t* rpT, int64_t* ciT, double* valT);
/* C = A B, B row-major n x k, C m x k overwritten (gpu_backend.cpp:104-121). */
void hno_spmm(int64_t m, const int64_t* rp, const int64_t* ci, const double* val,
              const double* B, int64_t k, double* C);
/* CPUBackend dot / axpy / norm_inf (gpu_backend.cpp:123-132); nrm2 is the
 * Euclidean norm accumulated left to right. */
double hno_dot(int64_t n, const double* a, const double* b);
void hno_axpy(int64_t n, double alpha, const double* x, double* y);
double hno_norm_inf(int64_t n, const double* v);
double hno_nrm2(int64_t n, const double* v);
/* alpha = min(1, 0.99 * min_{d_i<0} -v_i/d_i) (interior_point.cpp:134-142). */
double hno_max_step(int64_t n, const double* v, const double* d);

/* Number of triplets build_normal_equations emits for this D
 * (sum over columns with D_j > 0 of count_j^2, plus m diagonal terms). */
int64_t hno_normal_equations_triplets(int64_t m, int64_t n, const int64_t* rp,
                                      const int64_t* ci, const double* D);
/* N = M diag(D) M^T + dyn_reg I as CSR (interior_point.cpp:144-200): column
 * lists by counting sort, triplets emitted column by column, diagonal sums in
 * emission order give max_diag, dyn_reg = max(reg, 1e-12 * max_diag), then
 * from_triplets semantics (sort by (row,col) keeping emission order among
 * equal keys, sum, drop exact zeros). rpN: m+1; ciN/valN: room for the
 * triplet count. Returns nnz(N); *dyn_reg_out receives dyn_reg. */
int64_t hno_normal_equations(int64_t m, int64_t n, const int64_t* rp, const int64_t* ci,
                             const double* val, const double* D, double reg, int64_t* rpN,
                             int64_t* ciN, double* valN, double* dyn_reg_out);
/* selected rows of the same N, with |term| sums (see hn_oracle.c) */
int64_t hno_normal_rows(int64_t m, int64_t n, const int64_t* rp, const int64_t* ci, const double* val,
                        const double* D, double reg, int64_t nsel, const int64_t* rows, int64_t* rpS,
                        int64_t* ciS, double* valS, double* absS, double* dyn_out);

/* Structural pattern of M M^T plus the full diagonal, rows sorted, no values
 * (the pattern build_normal_equations produces when every D_j > 0 and no sum
 * cancels to exactly zero). Returns nnz; pass ciN == NULL to count only. */
int64_t hno_ada_pattern(int64_t m, int64_t n, const int64_t* rp, const int64_t* ci,
                        int64_t* rpN, int32_t* ciN);

/* Merge-path partition of the (m row ends + nnz nonzeros) list into tiles of
 * `items` entries: for tile t (0..ntiles), the coordinate (row, nz) where
 * diagonal t*items crosses the path; diagonal clamped to m+nnz. This is the
 * library's row binning (int32 row pointer, see csrc); no reference
 * counterpart exists (the reference picks one kernel for the whole matrix from
 * the mean row length, gpu_backend.cpp:413-415). */
void hno_merge_tiles(int64_t m, int64_t nnz, const int32_t* rp, int64_t items, int64_t ntiles,
                     int32_t* tile_row, int32_t* tile_nz);

/* ---- revised-simplex pricing (core/lp/simplex.cpp) ---- */
/* rc = cost - A^T y, A^T y by transpose_multiply's scatter
 * (compute_reduced_costs, simplex.cpp:1225-1233). */
void hno_price_reduced_costs(int64_t m, int64_t n, const int64_t* rp, const int64_t* ci, const double* val,
                             const double* y, const double* cost, double* rc);
/* update_devex_weights (simplex.cpp:1235-1271) with the BTRAN row u given;
 * alpha (n) receives A^T u. */
void hno_price_devex_update(int64_t m, int64_t n, const int64_t* rp, const int64_t* ci, const double* val,
                            const double* u, const int32_t* nonbasis, double* weights, double* alpha);
/* ranked_candidates (simplex.cpp:1283-1308): writes the first `cap` indices
 * of the ranking into out, returns the number of candidates. */
int64_t hno_price_ranked(int64_t n, const double* rc, const double* w, const int32_t* nonbasis,
                         const uint8_t* artificial, int phase1, int maximize, double tol, int64_t cap,
                         int64_t* out);
/* The Bland branch of select_entering_variable (simplex.cpp:1328-1338). */
int64_t hno_price_bland(int64_t n, const double* rc, const int32_t* nonbasis, const uint8_t* artificial,
                        int phase1, int maximize, double tol);
/* extract_column (simplex.cpp:25-35): col (m) = column j of A, the first
 * entry with that column in each row. */
void hno_extract_column(int64_t m, const int64_t* rp, const int64_t* ci, const double* val, int64_t j,
                        double* col);

#ifdef __cplusplus
}
#endif
#endif
