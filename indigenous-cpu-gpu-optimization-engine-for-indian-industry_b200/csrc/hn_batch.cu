// Batched Mehrotra IPM: many LPs of uneven sizes advanced in lockstep.
//
// The instances are packed as one block-diagonal CSR M = diag(M_1 .. M_K)
// (rows row_off[i]..row_off[i+1], columns col_off[i]..col_off[i+1]), so the
// merge-path SpMVs with their IPM epilogues, the device A^T and the A D A^T
// assembly run on the whole batch in single launches (the assembly's
// per-row windows keep its bitmaps to one block). What differs per instance
// lives here:
//   - reductions per instance (one CTA each): mu, ||rp||_inf, ||rd||_inf, step
//     lengths, mu_aff, sigma -- the scalars of interior_point.cpp:517-530,
//     :629-643, :683-684 -- in a K x HN_IPM_NSCAL block, plus a per-instance
//     status word (0 = iterating) that masks converged or failed instances out
//     of the factorisation, the solves and the update;
//   - dyn_reg = max(reg, 1e-12 * max diag) per instance (:188-196);
//   - the normal-equation factorisation: each instance's N block is scattered
//     into a dense lower triangle and factorised by a blocked LDL^T on the GPU
//     with the reference's pivot clamp (factorization.cpp:1299-1305), level-
//     synchronously in 64-column blocks: per block one launch factorises every
//     instance's diagonal block, one spreads all instances' panel rows and one
//     all instances' trailing tiles over the GPU. This is a deliberate
//     deviation from keeping factorisations on the host: thousands of
//     factorisations per iteration do not fit in host time;
//   - the two triangular solves, level-synchronous in the same blocks, and
//     iterative refinement (refinement.cpp:7-37: up to 5 sweeps, stop at
//     1e-10 relative) per instance, with N x as one SpMV over the packed N.
#include <algorithm>
#include <cmath>
#include <numeric>
#include <vector>

#include "hn_spmv.cuh"

struct hn_batch {
    int64_t K = 0, m = 0, n = 0;
    const hn_pattern* P = nullptr;
    int64_t* row_off = nullptr;  // K+1
    int64_t* col_off = nullptr;  // K+1
    int32_t* row_inst = nullptr; // m
    int64_t* dn_off = nullptr;   // K+1, offsets of the dense blocks
    int32_t* order = nullptr;    // instances by decreasing size
    double* dense = nullptr;     // sum m_i^2
    double* dD = nullptr;        // LDL^T pivots, m
    int32_t* refine = nullptr;   // per-instance refinement flag (1 = keep sweeping)
    int32_t* nref = nullptr;     // number of instances still refining
    // N as an SpMV operand (int32 row pointer copy + merge-path tables)
    int32_t* nrp = nullptr;
    int64_t ntiles = 0;
    int32_t *tile_row = nullptr, *tile_nz = nullptr, *carry_row = nullptr, *head_row = nullptr;
    double *carry_val = nullptr, *head_val = nullptr;
    double* r = nullptr;         // refinement residual, m
    double* ax = nullptr;        // N x, m
    // level schedule of the blocked factorisation: at block step s the
    // instances order[0 .. cnt[s]) still have a block; step_pairs (offset
    // pair_off[s]) holds, per such instance, the cumulative count of trailing
    // 32x32 tile pairs, so one launch spreads every instance's tiles over the GPU
    int64_t nsteps = 0;
    std::vector<int32_t> step_cnt;       // host, nsteps
    std::vector<int64_t> step_pairs_h;   // host, total pairs per step
    std::vector<int64_t> pair_off_h;     // host, nsteps+1 offsets into step_pairs
    int64_t* step_pairs = nullptr;       // device, cumulative pairs per (step, instance)
    // panel rows below each instance's diagonal block, in chunks of kT rows
    std::vector<int64_t> step_chunks_h;  // host, total chunks per step
    std::vector<int64_t> chunk_off_h;    // host, nsteps+1 offsets into step_chunks
    int64_t* step_chunks = nullptr;      // device, cumulative chunks per (step, instance)
    double* solve_part = nullptr;        // backward-solve partial dot products, 64 per chunk
    // relative KKT residual per instance and the tightening past the
    // reference's stop (hn_batch_set_kkt): ru / cu / offset are caller-owned
    // unscale factors (null = not measured); kkt and kkt_ref hold K x 4
    // (residual, primal, dual, gap) at the last residual call and at the
    // iteration the reference's rule first held (ref_iter, -1 = not yet);
    // xb / zb / lb keep the iterate of that iteration
    const double *ru = nullptr, *cu = nullptr, *offset = nullptr;
    double kkt_tol = 0.0;
    int kkt_extra = 0;
    double *kkt = nullptr, *kkt_ref = nullptr;
    int32_t* ref_iter = nullptr;
    double *xb = nullptr, *zb = nullptr, *lb = nullptr;
};

namespace hn {
namespace {

constexpr int kT = 256;
constexpr int S_NRP = HN_IPM_NRP, S_NRD = HN_IPM_NRD, S_MU = HN_IPM_MU, S_AP = HN_IPM_AP, S_AD = HN_IPM_AD,
              S_MUAFF = HN_IPM_MUAFF, S_SIGMA = HN_IPM_SIGMA;
constexpr int ST_RUN = 0, ST_OPTIMAL = 1, ST_NUMERICAL = 7;

// Row stride of an instance's dense block: m rounded up to even, so every row
// starts on a 16-byte boundary (16-byte asynchronous copies of the panels).
__host__ __device__ __forceinline__ int dense_ld(int m) { return (m + 1) & ~1; }

__device__ __forceinline__ bool fin(double v) { return isfinite(v); }

// ---- per-instance reductions ----
// What the residual pass needs for the relative KKT residual and the
// tightening: see hn_batch_set_kkt.
struct KktArgs {
    const double *lam, *b, *c, *ru, *cu, *offset;
    double *kkt, *kkt_ref, *xb, *zb, *lb;
    int32_t* ref_iter;
    double tol;
    int extra;
};

__device__ __forceinline__ double fin_or_inf(double t) { return t <= 1.7976931348623157e308 ? t : INFINITY; }

__global__ void __launch_bounds__(kT) batch_prep_kernel(const int64_t* __restrict__ row_off,
                                                        const int64_t* __restrict__ col_off,
                                                        const double* __restrict__ x, const double* __restrict__ z,
                                                        const double* __restrict__ rd, const double* __restrict__ rp,
                                                        double* __restrict__ D, double* __restrict__ Drd,
                                                        double* __restrict__ scal, int32_t* __restrict__ status,
                                                        int32_t* __restrict__ iters, int iter, double tol,
                                                        double ctol, KktArgs k) {
    __shared__ double sh[32];
    __shared__ int s_save;
    const int64_t i = blockIdx.x;
    const int64_t c0 = col_off[i], c1 = col_off[i + 1], r0 = row_off[i], r1 = row_off[i + 1];
    const bool measure = k.ru != nullptr;
    double smu = 0.0, mrd = 0.0, mrp = 0.0, du = 0.0, cn = 0.0, cx = 0.0, pr = 0.0, bn = 0.0, by = 0.0;
    for (int64_t j = c0 + threadIdx.x; j < c1; j += kT) {
        const double xj = x[j], zj = z[j], r = rd[j];
        smu += xj * zj;
        mrd = fmax(mrd, fabs(r));
        double d = xj / zj;
        if (!(d >= 0.0) || !fin(d) || d > 1e10) d = 1e10;  // interior_point.cpp:532-539
        D[j] = d;
        Drd[j] = d * r;
        if (measure) {
            const double u = k.cu[j], cj = k.c[j];
            du = fmax(du, fin_or_inf(fabs(r) * u));
            cn = fmax(cn, fabs(cj) * u);
            cx += cj * xj;
        }
    }
    for (int64_t q = r0 + threadIdx.x; q < r1; q += kT) {
        const double r = rp[q];
        mrp = fmax(mrp, fabs(r));
        if (measure) {
            const double u = k.ru[q], bq = k.b[q];
            pr = fmax(pr, fin_or_inf(fabs(r) * u));
            bn = fmax(bn, fabs(bq) * u);
            by += bq * k.lam[q];
        }
    }
    smu = block_sum<kT>(smu, sh);
    mrd = block_max<kT>(mrd, sh);
    mrp = block_max<kT>(mrp, sh);
    if (measure) {
        du = block_max<kT>(du, sh);
        cn = block_max<kT>(cn, sh);
        cx = block_sum<kT>(cx, sh);
        pr = block_max<kT>(pr, sh);
        bn = block_max<kT>(bn, sh);
        by = block_sum<kT>(by, sh);
    }
    if (threadIdx.x == 0) {
        const double mu = smu / static_cast<double>(c1 - c0);
        double* s = scal + i * HN_IPM_NSCAL;
        s[S_MU] = mu;
        s[S_NRD] = mrd;
        s[S_NRP] = mrp;
        double kk = 0.0;
        if (measure) {
            const double P = pr / (1.0 + bn), Dl = du / (1.0 + cn),
                         Gp = fabs(cx - by) / (1.0 + fabs(cx + k.offset[i]));
            kk = (P != P || Dl != Dl || Gp != Gp) ? nan("") : fmax(P, fmax(Dl, Gp));
            double* o = k.kkt + 4 * i;
            o[0] = kk;
            o[1] = P;
            o[2] = Dl;
            o[3] = Gp;
        }
        int save = 0;
        if (status[i] == ST_RUN) {
            int r = k.ref_iter[i];
            if (r < 0 && mrp < tol && mrd < tol && mu < ctol) {  // the reference's rule, :525-530
                r = iter;
                k.ref_iter[i] = iter;
                save = measure && k.tol > 0.0;
                if (measure)
                    for (int q = 0; q < 4; ++q) k.kkt_ref[4 * i + q] = k.kkt[4 * i + q];
            }
            // stop at the reference's rule, or past it once the KKT residual
            // is within tolerance or the extra iterations are spent
            if (r >= 0 && (!(measure && k.tol > 0.0) || kk <= k.tol || iter - r >= k.extra)) {
                status[i] = ST_OPTIMAL;
                iters[i] = iter;
            }
        }
        s_save = save;
    }
    __syncthreads();
    if (s_save) {  // keep the iterate the reference would return
        for (int64_t j = c0 + threadIdx.x; j < c1; j += kT) {
            k.xb[j] = x[j];
            k.zb[j] = z[j];
        }
        for (int64_t q = r0 + threadIdx.x; q < r1; q += kT) k.lb[q] = k.lam[q];
    }
}

// After the last residual pass: an instance that met the reference's rule
// and then failed (status 7), was still iterating, or ended with a larger
// KKT residual than at that point gets the saved iterate back.
__global__ void __launch_bounds__(kT) batch_finish_kernel(const int64_t* __restrict__ row_off,
                                                          const int64_t* __restrict__ col_off, double* __restrict__ x,
                                                          double* __restrict__ z, double* __restrict__ lam,
                                                          int32_t* __restrict__ status, int32_t* __restrict__ iters,
                                                          KktArgs k) {
    __shared__ int s_restore;
    const int64_t i = blockIdx.x;
    const int r = k.ref_iter[i];
    if (r < 0) return;
    if (threadIdx.x == 0) {
        const double now = k.kkt[4 * i], then = k.kkt_ref[4 * i];
        const int st = status[i];
        const bool worse = !(now <= then);  // NaN now counts as worse
        s_restore = (st == ST_NUMERICAL || worse) ? 1 : 0;
        status[i] = ST_OPTIMAL;
        if (s_restore) {
            iters[i] = r;
            for (int q = 0; q < 4; ++q) k.kkt[4 * i + q] = k.kkt_ref[4 * i + q];
        }
    }
    __syncthreads();
    if (!s_restore) return;
    const int64_t c0 = col_off[i], c1 = col_off[i + 1], r0 = row_off[i], r1 = row_off[i + 1];
    for (int64_t j = c0 + threadIdx.x; j < c1; j += kT) {
        x[j] = k.xb[j];
        z[j] = k.zb[j];
    }
    for (int64_t q = r0 + threadIdx.x; q < r1; q += kT) lam[q] = k.lb[q];
}

__global__ void __launch_bounds__(kT) batch_steps_kernel(const int64_t* __restrict__ row_off,
                                                         const int64_t* __restrict__ col_off,
                                                         const double* __restrict__ x, const double* __restrict__ dx,
                                                         const double* __restrict__ z, const double* __restrict__ dz,
                                                         const double* __restrict__ dlam, double* __restrict__ scal,
                                                         int32_t* __restrict__ status) {
    __shared__ double sh[32];
    __shared__ int s_bad;
    const int64_t i = blockIdx.x;
    if (status[i] != ST_RUN) return;
    if (threadIdx.x == 0) s_bad = 0;
    __syncthreads();
    const int64_t c0 = col_off[i], c1 = col_off[i + 1], r0 = row_off[i], r1 = row_off[i + 1];
    double ap = 1.0, ad = 1.0;
    bool bad = false;
    for (int64_t j = c0 + threadIdx.x; j < c1; j += kT) {
        const double a = dx[j], b = dz[j];
        if (a < 0.0) ap = fmin(ap, -x[j] / a);
        if (b < 0.0) ad = fmin(ad, -z[j] / b);
        bad |= !fin(a) || !fin(b);
    }
    for (int64_t k = r0 + threadIdx.x; k < r1; k += kT) bad |= !fin(dlam[k]);
    if (bad) s_bad = 1;
    ap = block_min<kT>(ap, sh);
    ad = block_min<kT>(ad, sh);
    if (threadIdx.x == 0) {
        double* s = scal + i * HN_IPM_NSCAL;
        const double sp = 0.99 * ap, sq = 0.99 * ad;  // max_step, :134-142
        s[S_AP] = sp < 1.0 ? sp : 1.0;
        s[S_AD] = sq < 1.0 ? sq : 1.0;
        if (s_bad) status[i] = ST_NUMERICAL;  // :617-627, :676-686
    }
}

// mu_aff, sigma and zs = (sigma mu - dx dz) (1/z) of one instance per CTA.
__global__ void __launch_bounds__(kT) batch_corr_kernel(const int64_t* __restrict__ col_off,
                                                        const double* __restrict__ x, const double* __restrict__ dx,
                                                        const double* __restrict__ z, const double* __restrict__ dz,
                                                        double* __restrict__ scal, const int32_t* __restrict__ status,
                                                        double* __restrict__ zs) {
    __shared__ double sh[32];
    __shared__ double s_sm;
    const int64_t i = blockIdx.x;
    const int64_t c0 = col_off[i], c1 = col_off[i + 1];
    double* s = scal + i * HN_IPM_NSCAL;
    if (status[i] != ST_RUN) {
        for (int64_t j = c0 + threadIdx.x; j < c1; j += kT) zs[j] = 0.0;
        return;
    }
    const double ap = s[S_AP], ad = s[S_AD];
    double acc = 0.0;
    for (int64_t j = c0 + threadIdx.x; j < c1; j += kT) acc += (x[j] + ap * dx[j]) * (z[j] + ad * dz[j]);
    acc = block_sum<kT>(acc, sh);
    if (threadIdx.x == 0) {
        const double mu_aff = acc / static_cast<double>(c1 - c0);  // :632-636
        const double mu = s[S_MU];
        double sigma;
        if (!fin(mu_aff) || mu_aff < 0.0 || !(mu > 0.0)) {
            sigma = 0.5;
        } else {
            const double r = pow(mu_aff / fmax(mu, 1e-300), 3.0);
            sigma = r < 0.1 ? 0.1 : (r > 0.9 ? 0.9 : r);  // :638-643
        }
        s[S_MUAFF] = mu_aff;
        s[S_SIGMA] = sigma;
        s_sm = sigma * mu;
    }
    __syncthreads();
    const double sm = s_sm;
    for (int64_t j = c0 + threadIdx.x; j < c1; j += kT) {
        const double zinv = 1.0 / z[j];
        zs[j] = (sm - dx[j] * dz[j]) * zinv;  // :645-651
    }
}

__global__ void __launch_bounds__(kT) batch_update_kernel(const int64_t* __restrict__ row_off,
                                                          const int64_t* __restrict__ col_off, double* __restrict__ x,
                                                          const double* __restrict__ dx, double* __restrict__ z,
                                                          const double* __restrict__ dz, double* __restrict__ lam,
                                                          const double* __restrict__ dlam,
                                                          const double* __restrict__ scal,
                                                          int32_t* __restrict__ status, int32_t* __restrict__ iters,
                                                          int iter) {
    __shared__ int s_bad;
    const int64_t i = blockIdx.x;
    if (status[i] != ST_RUN) return;
    if (threadIdx.x == 0) s_bad = 0;
    __syncthreads();
    const int64_t c0 = col_off[i], c1 = col_off[i + 1], r0 = row_off[i], r1 = row_off[i + 1];
    const double ap = scal[i * HN_IPM_NSCAL + S_AP], ad = scal[i * HN_IPM_NSCAL + S_AD];
    bool bad = false;
    for (int64_t j = c0 + threadIdx.x; j < c1; j += kT) {
        const double xn = x[j] + ap * dx[j];
        const double zn = z[j] + ad * dz[j];
        x[j] = xn;
        z[j] = zn;
        bad |= xn < 0.0 || zn < 0.0 || !fin(xn) || !fin(zn);  // :698-708
    }
    for (int64_t k = r0 + threadIdx.x; k < r1; k += kT) lam[k] += ad * dlam[k];
    if (bad) s_bad = 1;
    __syncthreads();
    if (threadIdx.x == 0) {
        if (s_bad)
            status[i] = ST_NUMERICAL;
        else
            iters[i] = iter + 1;
    }
}

// ---- normal equations per instance ----
__global__ void __launch_bounds__(kT) batch_reg_kernel(const int64_t* __restrict__ row_off,
                                                       const int64_t* __restrict__ diag_pos, double reg,
                                                       const int32_t* __restrict__ status, double* __restrict__ nval) {
    __shared__ double sh[32];
    __shared__ double s_dyn;
    const int64_t i = blockIdx.x;
    if (status[i] != ST_RUN) return;
    const int64_t r0 = row_off[i], r1 = row_off[i + 1];
    double md = 0.0;
    for (int64_t r = r0 + threadIdx.x; r < r1; r += kT) md = fmax(md, nval[diag_pos[r]]);  // NaN ignored
    md = block_max<kT>(md, sh);
    if (threadIdx.x == 0) {
        const double dyn = 1e-12 * md;
        s_dyn = (reg < dyn) ? dyn : reg;  // std::max(regularization, 1e-12 * max_diag)
    }
    __syncthreads();
    const double dyn = s_dyn;
    for (int64_t r = r0 + threadIdx.x; r < r1; r += kT) nval[diag_pos[r]] += dyn;
}

// One warp per packed row: zero the dense lower row, then scatter N's entries.
__global__ void batch_dense_kernel(int64_t m, const int64_t* __restrict__ row_off, const int32_t* __restrict__ row_inst,
                                   const int64_t* __restrict__ dn_off, const int32_t* __restrict__ status,
                                   const int64_t* __restrict__ rpN, const int32_t* __restrict__ ciN,
                                   const double* __restrict__ nval, double* __restrict__ dense) {
    const int64_t r = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (r >= m) return;
    const int inst = row_inst[r];
    if (status[inst] != ST_RUN) return;
    const int64_t b0 = row_off[inst], mi = row_off[inst + 1] - b0, lr = r - b0;
    double* row = dense + dn_off[inst] + lr * dense_ld(static_cast<int>(mi));
    for (int64_t c = lane; c <= lr; c += 32) row[c] = 0.0;
    __syncwarp();
    for (int64_t p = rpN[r] + lane; p < rpN[r + 1]; p += 32) {
        const int64_t c = (int64_t)ciN[p] - b0;
        if (c >= 0 && c <= lr) row[c] = nval[p];
    }
}

// Blocked right-looking LDL^T, level-synchronous over the batch, in blocks of
// kFb columns: block step s runs two launches for every instance that still
// has a block s --
//   batch_ldlt_diag_kernel: one CTA per instance factorises the kFb x kFb
//     diagonal block (pivot clamp of factorization.cpp:1299-1305);
//   batch_ldlt_panel_kernel: every instance's panel below its diagonal block,
//     in chunks of kT rows spread over the GPU, one row per thread;
//   batch_ldlt_update_kernel: all instances' trailing kFb x kFb tiles
//     A_rc -= sum_q (L_rq D_q) L_cq, spread over every CTA of the GPU, on the
//     FP64 tensor cores (mma.sync m8n8k4, FP64 in and out).
constexpr int kFb = 64;

// D(8x8) += A(8x4) B(4x8) in FP64 on the tensor cores. Fragments: lane l
// holds A[l/4][l%4], B[l%4][l/4] and D[l/4][2(l%4)], D[l/4][2(l%4)+1].
__device__ __forceinline__ void dmma_m8n8k4(double* d, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(d[0]), "+d"(d[1])
                 : "d"(a), "d"(b));
}
constexpr int kFbP = kFb + 1;  // padded smem row (conflict-free column walks)
constexpr size_t kPanelSmem = sizeof(double) * (2 * kFb * kFbP + 2 * kFb);

__global__ void __launch_bounds__(kT) batch_ldlt_diag_kernel(int s, const int64_t* __restrict__ row_off,
                                                             const int64_t* __restrict__ dn_off,
                                                             const int32_t* __restrict__ order,
                                                             const int32_t* __restrict__ status,
                                                             double* __restrict__ dense, double* __restrict__ dD,
                                                             double tol) {
    extern __shared__ double smem[];
    double(*sA)[kFbP] = reinterpret_cast<double(*)[kFbP]>(smem);
    double(*sL)[kFbP] = reinterpret_cast<double(*)[kFbP]>(smem + kFb * kFbP);
    double* sD = smem + 2 * kFb * kFbP;
    double* sLc = sD + kFb;  // column j of L during pivot j
    const int tid = threadIdx.x;
    const int inst = order[blockIdx.x];
    if (status[inst] != ST_RUN) return;
    const int64_t r0 = row_off[inst];
    const int m = static_cast<int>(row_off[inst + 1] - r0);
    const int ld = dense_ld(m);
    const int k0 = s * kFb;
    if (k0 >= m) return;
    const int nb = min(kFb, m - k0);
    double* A = dense + dn_off[inst];
    for (int idx = tid; idx < kFb * kFb; idx += kT) {
        const int r = idx / kFb, c = idx % kFb;
        sA[r][c] = (r < nb && c <= r) ? A[(int64_t)(k0 + r) * ld + k0 + c] : 0.0;
    }
    __syncthreads();
    // pivot j: every thread forms the clamped pivot itself; column j of L,
    // l = A_.,j / d, is divided out once (to sLc and sL; column j of sA stays
    // unscaled); then warp w takes rows rr = j + 1 + w, j + 9 + w, ..., lanes
    // the columns j < cc <= rr, and each element takes A_rr,cc -= (l_rr d) l_cc:
    // the sequence and roundings of the column-by-column elimination
    const int lane = tid & 31, warp = tid >> 5;
    for (int j = 0; j < nb; ++j) {
        double d = sA[j][j];
        if (d <= tol) d = tol;  // SparseCholesky pivot clamp
        if (tid == 0) sD[j] = d;
        for (int cc = j + 1 + tid; cc < nb; cc += kT) {
            const double l = sA[cc][j] / d;
            sLc[cc] = l;
            sL[cc][j] = l;
        }
        __syncthreads();
        for (int rr = j + 1 + warp; rr < nb; rr += kT / 32) {
            const double wr = sLc[rr] * d;
            for (int cc = j + 1 + lane; cc <= rr; cc += 32) sA[rr][cc] -= wr * sLc[cc];
        }
        __syncthreads();
    }
    for (int idx = tid; idx < nb * nb; idx += kT) {
        const int r = idx / nb, c = idx % nb;
        if (c < r) A[(int64_t)(k0 + r) * ld + k0 + c] = sL[r][c];
    }
    if (tid < nb) dD[r0 + k0 + tid] = sD[tid];
}

// L[r, k0:k1] = A[r, k0:k1] (L_blk D)^-T for the kT rows of chunk `local`
// of one instance's panel (the instance: first b with chunks[b] > chunk).
__global__ void __launch_bounds__(kT) batch_ldlt_panel_kernel(int s, int cnt, const int64_t* __restrict__ chunks,
                                                              const int64_t* __restrict__ row_off,
                                                              const int64_t* __restrict__ dn_off,
                                                              const int32_t* __restrict__ order,
                                                              const int32_t* __restrict__ status,
                                                              double* __restrict__ dense,
                                                              const double* __restrict__ dD) {
    __shared__ double sL[kFb][kFbP];
    __shared__ double sD[kFb];
    const int tid = threadIdx.x;
    const int64_t chunk = blockIdx.x;
    int lo = 0, hi = cnt - 1;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (chunks[mid] <= chunk)
            lo = mid + 1;
        else
            hi = mid;
    }
    const int inst = order[lo];
    if (status[inst] != ST_RUN) return;
    const int64_t local = chunk - (lo > 0 ? chunks[lo - 1] : 0);
    const int64_t r0 = row_off[inst];
    const int m = static_cast<int>(row_off[inst + 1] - r0);
    const int ld = dense_ld(m);
    const int k0 = s * kFb;
    const int nb = min(kFb, m - k0), k1 = k0 + nb;
    double* A = dense + dn_off[inst];
    for (int idx = tid; idx < kFb * kFb; idx += kT) {
        const int r = idx / kFb, c = idx % kFb;
        sL[r][c] = (r < nb && c < r) ? A[(int64_t)(k0 + r) * ld + k0 + c] : 0.0;
    }
    if (tid < kFb) sD[tid] = tid < nb ? dD[r0 + k0 + tid] : 1.0;
    __syncthreads();
    const int r = k1 + static_cast<int>(local) * kT + tid;
    if (r >= m) return;
    // lv[c] holds A[r, k0 + c] until column c is final; then L[r, c] goes to
    // memory and lv[c] keeps L[r, c] D_c, the factor every later column
    // multiplies (the same single rounding as computing it there each time)
    double lv[kFb];
    double* Ar = A + (int64_t)r * ld + k0;
#pragma unroll
    for (int c = 0; c < kFb; ++c) lv[c] = (c < nb) ? Ar[c] : 0.0;
#pragma unroll
    for (int c = 0; c < kFb; ++c) {
        if (c < nb) {
            double v = lv[c];
#pragma unroll
            for (int q = 0; q < c; ++q) v -= lv[q] * sL[c][q];
            const double l = v / sD[c];
            Ar[c] = l;
            lv[c] = l * sD[c];
        }
    }
}

// Trailing update of one 64 x 64 tile pair per CTA iteration. Both 64-column
// panel slices arrive by 16-byte asynchronous copies (rows start on 16-byte
// boundaries: even row stride), in two commit groups of 32 columns, so the
// second half is in flight while the first is multiplied; the output tile
// arrives the same way (a third group) and is read back from shared memory in
// the epilogue. D is applied at the
// fragment load: a = L[r, k] D_k rounds once, as a staged product would, and
// every output fragment takes the same DMMA sequence (k ascending in steps of
// 4), so the result does not depend on the staging.
constexpr int kUpdP = kFb + 4;  // smem row stride: a half-warp's fragment loads hit 16 distinct bank pairs
constexpr size_t kUpdSmem = sizeof(double) * (3 * kFb * kUpdP + kFb);

__device__ __forceinline__ void cp_async16(void* dst, const void* src, bool valid) {
    const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(src), "r"(valid ? 16 : 0)
                 : "memory");
}

struct UpdPair {
    int m, ld, rb, cb;
    int64_t r0;
    double* A;
};

// Persistent: each CTA walks pairs blockIdx.x, + grid, ... and overlaps the
// next pair's panel copies with the current pair's epilogue (the panels are
// free once the multiply is done; the output tile's buffer once the epilogue
// has read it).
__global__ void __launch_bounds__(kT, 2) batch_ldlt_update_kernel(int s, int cnt, int64_t npairs,
                                                               const int64_t* __restrict__ pairs,
                                                               const int64_t* __restrict__ row_off,
                                                               const int64_t* __restrict__ dn_off,
                                                               const int32_t* __restrict__ order,
                                                               const int32_t* __restrict__ status,
                                                               double* __restrict__ dense,
                                                               const double* __restrict__ dD) {
    extern __shared__ __align__(16) double upd_smem[];
    double(*sW)[kUpdP] = reinterpret_cast<double(*)[kUpdP]>(upd_smem);                // L[rb + r, k0 + k]
    double(*sL)[kUpdP] = reinterpret_cast<double(*)[kUpdP]>(upd_smem + kFb * kUpdP);  // L[cb + c, k0 + k]
    double(*sC)[kUpdP] = reinterpret_cast<double(*)[kUpdP]>(upd_smem + 2 * kFb * kUpdP);  // A[rb + r, cb + c]
    double* sD = upd_smem + 3 * kFb * kUpdP;
    const int tid = threadIdx.x;
    const int k0 = s * kFb;
    const int k1 = k0 + kFb;  // a trailing part exists only below a full block
    int lo = 0;               // the instance of the previous pair: pairs arrive in increasing order
    int64_t pidx = blockIdx.x;
    // the next pair of a running instance from pidx on (pidx moves past it);
    // the same answer in every thread
    auto next_pair = [&](UpdPair& P) -> bool {
        for (; pidx < npairs; pidx += gridDim.x) {
            // instance of this pair: first b with pairs[b] > pidx (pairs is
            // inclusive), searched from the previous one by doubling steps
            if (pairs[lo] <= pidx) {
                int step = 1, base = lo;
                while (base + step < cnt - 1 && pairs[base + step] <= pidx) {
                    base += step;
                    step <<= 1;
                }
                int a = base + 1, b = min(base + step, cnt - 1);
                while (a < b) {
                    const int mid = (a + b) >> 1;
                    if (pairs[mid] <= pidx)
                        a = mid + 1;
                    else
                        b = mid;
                }
                lo = a;
            }
            const int inst = order[lo];
            if (status[inst] != ST_RUN) continue;
            const int64_t local = pidx - (lo > 0 ? pairs[lo - 1] : 0);
            int ti = static_cast<int>((sqrt(8.0 * (double)local + 1.0) - 1.0) * 0.5);
            while ((int64_t)(ti + 1) * (ti + 2) / 2 <= local) ++ti;
            while ((int64_t)ti * (ti + 1) / 2 > local) --ti;
            const int tj = static_cast<int>(local - (int64_t)ti * (ti + 1) / 2);
            P.r0 = row_off[inst];
            P.m = static_cast<int>(row_off[inst + 1] - P.r0);
            P.ld = dense_ld(P.m);
            P.rb = k1 + ti * kFb;
            P.cb = k1 + tj * kFb;
            P.A = dense + dn_off[inst];
            pidx += gridDim.x;
            return true;
        }
        return false;
    };
    // 2 slices x 64 rows x 16 chunks of 16 bytes per half, one commit group
    // per half; rows past m are zero-filled
    auto issue_panels = [&](const UpdPair& P) {
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            for (int idx = tid; idx < 2 * kFb * 16; idx += kT) {
                const int side = idx >> 10, rr = (idx >> 4) & (kFb - 1), q2 = idx & 15;
                const int row = (side ? P.cb : P.rb) + rr;
                const bool ok = row < P.m;
                const double* src = P.A + (int64_t)(ok ? row : P.rb) * P.ld + k0 + h * 32 + 2 * q2;
                double* dst = (side ? sL[rr] : sW[rr]) + h * 32 + 2 * q2;
                cp_async16(dst, src, ok);
            }
            asm volatile("cp.async.commit_group;\n" ::: "memory");
        }
    };
    // the output tile, one commit group: rows or columns past m are zero-filled
    auto issue_tile = [&](const UpdPair& P) {
        for (int idx = tid; idx < kFb * 32; idx += kT) {
            const int rr = idx >> 5, q2 = idx & 31;
            const int row = P.rb + rr, col = P.cb + 2 * q2;
            const bool ok = row < P.m && col < P.m;
            const double* src = P.A + (ok ? (int64_t)row * P.ld + col : (int64_t)P.rb * P.ld + k0);
            cp_async16(sC[rr] + 2 * q2, src, ok);
        }
        asm volatile("cp.async.commit_group;\n" ::: "memory");
    };
    UpdPair cur;
    if (!next_pair(cur)) return;
    issue_panels(cur);
    issue_tile(cur);
    if (tid < kFb) sD[tid] = dD[cur.r0 + k0 + tid];
    // warp w: rows 16 (w >> 1) .. + 16 (two 8-row tiles), columns
    // 32 (w & 1) .. + 32 (four 8-column tiles) of the 64 x 64 output
    const int lane = tid & 31, warp = tid >> 5;
    const int wr = (warp >> 1) * 16, wc = (warp & 1) * 32;
    const int fr = lane >> 2, fk = lane & 3;
    for (;;) {
        // in flight: this pair's panel halves, then its output tile
        double acc[2][4][2];
#pragma unroll
        for (int i = 0; i < 2; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            if (h == 0)
                asm volatile("cp.async.wait_group 2;\n" ::: "memory");
            else
                asm volatile("cp.async.wait_group 1;\n" ::: "memory");
            __syncthreads();
#pragma unroll
            for (int kq = h * 32; kq < h * 32 + 32; kq += 4) {
                const double dk = sD[kq + fk];
                double a[2], b[4];
#pragma unroll
                for (int i = 0; i < 2; ++i) a[i] = sW[wr + 8 * i + fr][kq + fk] * dk;  // A(8x4)[fr][fk]
#pragma unroll
                for (int j = 0; j < 4; ++j) b[j] = sL[wc + 8 * j + fr][kq + fk];  // B(4x8)[fk][fr]
#pragma unroll
                for (int i = 0; i < 2; ++i)
#pragma unroll
                    for (int j = 0; j < 4; ++j) dmma_m8n8k4(acc[i][j], a[i], b[j]);
            }
        }
        __syncthreads();  // every warp is done with the panels and D
        UpdPair nxt;
        const bool more = next_pair(nxt);
        if (more) {
            issue_panels(nxt);
            if (tid < kFb) sD[tid] = dD[nxt.r0 + k0 + tid];
            asm volatile("cp.async.wait_group 2;\n" ::: "memory");  // this pair's tile; the next panels stay in flight
        } else {
            asm volatile("cp.async.wait_group 0;\n" ::: "memory");
        }
        __syncthreads();  // the output tile is in shared memory
#pragma unroll
        for (int i = 0; i < 2; ++i) {
            const int gr = cur.rb + wr + 8 * i + fr;
            if (gr >= cur.m) continue;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
#pragma unroll
                for (int t = 0; t < 2; ++t) {
                    const int gc = cur.cb + wc + 8 * j + 2 * fk + t;
                    if (gc <= gr)
                        cur.A[(int64_t)gr * cur.ld + gc] = sC[wr + 8 * i + fr][wc + 8 * j + 2 * fk + t] - acc[i][j][t];
                }
            }
        }
        if (!more) break;
        __syncthreads();  // every warp is done reading the output tile
        issue_tile(nxt);
        cur = nxt;
    }
}

// ---- batched triangular solves: N_i x = b in place, N_i = L_i D_i L_i^T ----
// Level-synchronous in the factorisation's 64-row blocks and its schedule
// (instances in decreasing size, panel rows in chunks of kT): per block,
// forward: one launch solves every instance's unit-lower diagonal block,
// one launch subtracts the block's contribution from the rows below (chunks
// spread over the GPU, one warp per row, coalesced loads); then x /= D;
// backward: one launch forms, per chunk, the column-block dot products of
// L^T x over the rows below, one launch sums them in chunk order per
// instance and solves the diagonal block. Every sum has a fixed order.
// An instance takes part when it is iterating and, with a refine mask, still
// refining.
__device__ __forceinline__ bool solving(const int32_t* status, const int32_t* refine, int inst) {
    return status[inst] == ST_RUN && (!refine || refine[inst]);
}

__device__ __forceinline__ int chunk_instance(const int64_t* chunks, int cnt, int64_t chunk) {
    int lo = 0, hi = cnt - 1;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (chunks[mid] <= chunk)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

__global__ void __launch_bounds__(kFb) batch_fwd_diag_kernel(int s, const int64_t* __restrict__ row_off,
                                                            const int64_t* __restrict__ dn_off,
                                                            const int32_t* __restrict__ order,
                                                            const int32_t* __restrict__ status,
                                                            const int32_t* __restrict__ refine,
                                                            const double* __restrict__ dense, double* __restrict__ xv) {
    __shared__ double sL[kFb][kFbP];
    __shared__ double sy[kFb];
    const int inst = order[blockIdx.x];
    if (!solving(status, refine, inst)) return;
    const int64_t r0 = row_off[inst];
    const int m = static_cast<int>(row_off[inst + 1] - r0);
    const int ld = dense_ld(m);
    const int k0 = s * kFb;
    if (k0 >= m) return;
    const int nb = min(kFb, m - k0);
    const double* L = dense + dn_off[inst];
    double* x = xv + r0;
    const int i = threadIdx.x;
    for (int idx = i; idx < kFb * kFb; idx += kFb) {
        const int r = idx / kFb, c = idx % kFb;
        sL[r][c] = (r < nb && c < r) ? L[(int64_t)(k0 + r) * ld + k0 + c] : 0.0;
    }
    sy[i] = i < nb ? x[k0 + i] : 0.0;
    __syncthreads();
    // warp 0 runs the substitution, rows lane and lane + 32, broadcasting
    // each solved entry by a shuffle (no barriers); same operations per
    // entry in the same order as a row-per-thread substitution
    if (i >= 32) return;
    double v0 = sy[i], v1 = sy[i + 32];
    for (int j = 0; j < nb; ++j) {
        const double yj = __shfl_sync(0xffffffffu, j < 32 ? v0 : v1, j & 31);
        if (i > j && i < nb) v0 -= sL[i][j] * yj;
        if (i + 32 > j && i + 32 < nb) v1 -= sL[i + 32][j] * yj;
    }
    if (i < nb) x[k0 + i] = v0;
    if (i + 32 < nb) x[k0 + i + 32] = v1;
}

__global__ void __launch_bounds__(kT) batch_fwd_gemv_kernel(int s, int cnt, const int64_t* __restrict__ chunks,
                                                           const int64_t* __restrict__ row_off,
                                                           const int64_t* __restrict__ dn_off,
                                                           const int32_t* __restrict__ order,
                                                           const int32_t* __restrict__ status,
                                                           const int32_t* __restrict__ refine,
                                                           const double* __restrict__ dense, double* __restrict__ xv) {
    __shared__ double sx[kFb];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int b = chunk_instance(chunks, cnt, blockIdx.x);
    const int inst = order[b];
    if (!solving(status, refine, inst)) return;
    const int64_t local = blockIdx.x - (b > 0 ? chunks[b - 1] : 0);
    const int64_t r0 = row_off[inst];
    const int m = static_cast<int>(row_off[inst + 1] - r0);
    const int ld = dense_ld(m);
    const int k0 = s * kFb;
    const int nb = min(kFb, m - k0), k1 = k0 + nb;
    const double* L = dense + dn_off[inst];
    double* x = xv + r0;
    if (tid < kFb) sx[tid] = tid < nb ? x[k0 + tid] : 0.0;
    __syncthreads();
    const int rb = k1 + static_cast<int>(local) * kT, re = min(m, rb + kT);
    for (int rw = rb + warp * 4; rw < re; rw += (kT / 32) * 4) {
        double p[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int r = rw + u;
            double a = 0.0;
            if (r < re) {
                const double* Lr = L + (int64_t)r * ld + k0;
                const double p0 = lane < nb ? Lr[lane] * sx[lane] : 0.0;
                const double p1 = lane + 32 < nb ? Lr[lane + 32] * sx[lane + 32] : 0.0;
                a = p0 + p1;
            }
            p[u] = a;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) p[u] += __shfl_xor_sync(0xffffffffu, p[u], o);
        }
        if (lane < 4 && rw + lane < re) {
            const double t = lane == 0 ? p[0] : lane == 1 ? p[1] : lane == 2 ? p[2] : p[3];
            x[rw + lane] -= t;
        }
    }
}

__global__ void batch_scale_kernel(int64_t m, const int32_t* __restrict__ row_inst,
                                   const int32_t* __restrict__ status, const int32_t* __restrict__ refine,
                                   const double* __restrict__ dD, double* __restrict__ x) {
    const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= m) return;
    if (solving(status, refine, row_inst[k])) x[k] /= dD[k];
}

// part[chunk][q] = sum over the chunk's rows c (in order, per warp, then the
// warps in order) of L[c][k0 + q] x[c]
__global__ void __launch_bounds__(kT) batch_bwd_gemv_kernel(int s, int cnt, const int64_t* __restrict__ chunks,
                                                           const int64_t* __restrict__ row_off,
                                                           const int64_t* __restrict__ dn_off,
                                                           const int32_t* __restrict__ order,
                                                           const int32_t* __restrict__ status,
                                                           const int32_t* __restrict__ refine,
                                                           const double* __restrict__ dense,
                                                           const double* __restrict__ xv, double* __restrict__ part) {
    __shared__ double sacc[kT / 32][kFb];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int b = chunk_instance(chunks, cnt, blockIdx.x);
    const int inst = order[b];
    if (!solving(status, refine, inst)) return;
    const int64_t local = blockIdx.x - (b > 0 ? chunks[b - 1] : 0);
    const int64_t r0 = row_off[inst];
    const int m = static_cast<int>(row_off[inst + 1] - r0);
    const int ld = dense_ld(m);
    const int k0 = s * kFb;
    const int nb = min(kFb, m - k0), k1 = k0 + nb;
    const double* L = dense + dn_off[inst];
    const double* x = xv + r0;
    const int rb = k1 + static_cast<int>(local) * kT, re = min(m, rb + kT);
    double a0 = 0.0, a1 = 0.0;
    for (int c = rb + warp; c < re; c += kT / 32) {
        const double* Lc = L + (int64_t)c * ld + k0;
        const double xc = x[c];
        if (lane < nb) a0 += Lc[lane] * xc;
        if (lane + 32 < nb) a1 += Lc[lane + 32] * xc;
    }
    sacc[warp][lane] = a0;
    sacc[warp][lane + 32] = a1;
    __syncthreads();
    if (tid < kFb) {
        double t = 0.0;
        for (int w = 0; w < kT / 32; ++w) t += sacc[w][tid];
        part[blockIdx.x * (int64_t)kFb + tid] = t;
    }
}

__global__ void __launch_bounds__(kFb) batch_bwd_diag_kernel(int s, const int64_t* __restrict__ chunks,
                                                            const int64_t* __restrict__ row_off,
                                                            const int64_t* __restrict__ dn_off,
                                                            const int32_t* __restrict__ order,
                                                            const int32_t* __restrict__ status,
                                                            const int32_t* __restrict__ refine,
                                                            const double* __restrict__ dense,
                                                            const double* __restrict__ part,
                                                            double* __restrict__ xv) {
    __shared__ double sL[kFb][kFbP];
    __shared__ double sxj[kFb];
    const int b = blockIdx.x;
    const int inst = order[b];
    if (!solving(status, refine, inst)) return;
    const int64_t r0 = row_off[inst];
    const int m = static_cast<int>(row_off[inst + 1] - r0);
    const int ld = dense_ld(m);
    const int k0 = s * kFb;
    if (k0 >= m) return;
    const int nb = min(kFb, m - k0);
    const double* L = dense + dn_off[inst];
    double* x = xv + r0;
    const int q = threadIdx.x;
    for (int idx = q; idx < kFb * kFb; idx += kFb) {
        const int r = idx / kFb, c = idx % kFb;
        sL[r][c] = (r < nb && c < r) ? L[(int64_t)(k0 + r) * ld + k0 + c] : 0.0;
    }
    const int64_t c0 = b > 0 ? chunks[b - 1] : 0, c1 = chunks[b];
    double t = 0.0;
    if (q < nb)
        for (int64_t ch = c0; ch < c1; ++ch) t += part[ch * kFb + q];
    sxj[q] = q < nb ? x[k0 + q] - t : 0.0;
    __syncthreads();
    // warp 0 runs the back substitution over rows lane and lane + 32 with
    // shuffle broadcasts (no barriers), operations as row-per-thread
    if (q >= 32) return;
    double v0 = sxj[q], v1 = sxj[q + 32];
    for (int j = nb - 1; j >= 0; --j) {
        const double xj = __shfl_sync(0xffffffffu, j < 32 ? v0 : v1, j & 31);
        if (q < j) v0 -= sL[j][q] * xj;
        if (q + 32 < j) v1 -= sL[j][q + 32] * xj;
    }
    if (q < nb) x[k0 + q] = v0;
    if (q + 32 < nb) x[k0 + q + 32] = v1;
}

// Refinement bookkeeping per instance (refinement.cpp:15-30): with r = rhs - N x,
// rel = max|r| / max|rhs|; an instance keeps sweeping while rel > 1e-10 and
// sweeps remain; a sweeping instance's r is then solved and added to x.
__global__ void __launch_bounds__(kT) batch_refine_check_kernel(const int64_t* __restrict__ row_off,
                                                                const int32_t* __restrict__ status,
                                                                const double* __restrict__ rhs,
                                                                const double* __restrict__ ax, double* __restrict__ r,
                                                                int32_t* __restrict__ refine, int32_t* nref) {
    __shared__ double sh[32];
    const int64_t i = blockIdx.x;
    if (status[i] != ST_RUN || !refine[i]) return;
    const int64_t r0 = row_off[i], r1 = row_off[i + 1];
    double nb = 0.0, nr = 0.0;
    for (int64_t k = r0 + threadIdx.x; k < r1; k += kT) {
        const double b = rhs[k], d = b - ax[k];
        nb = fmax(nb, fabs(b));
        nr = fmax(nr, fabs(d));
        r[k] = d;
    }
    nb = block_max<kT>(nb, sh);
    nr = block_max<kT>(nr, sh);
    if (threadIdx.x == 0) {
        const bool go = nb != 0.0 && nb == nb && nr / nb > 1e-10;
        refine[i] = go ? 1 : 0;
        if (go) atomicAdd(nref, 1);
    }
}

__global__ void __launch_bounds__(kT) batch_refine_start_kernel(const int64_t* __restrict__ row_off,
                                                                const int32_t* __restrict__ status,
                                                                const double* __restrict__ rhs,
                                                                int32_t* __restrict__ refine) {
    __shared__ double sh[32];
    const int64_t i = blockIdx.x;
    const int64_t r0 = row_off[i], r1 = row_off[i + 1];
    double nb = 0.0;
    for (int64_t k = r0 + threadIdx.x; k < r1; k += kT) nb = fmax(nb, fabs(rhs[k]));
    nb = block_max<kT>(nb, sh);
    // a zero or NaN right-hand side is not refined (refinement.cpp:17-18); fmax drops NaN,
    // so look for one explicitly
    __shared__ int s_nan;
    if (threadIdx.x == 0) s_nan = 0;
    __syncthreads();
    for (int64_t k = r0 + threadIdx.x; k < r1; k += kT)
        if (rhs[k] != rhs[k]) s_nan = 1;
    __syncthreads();
    if (threadIdx.x == 0) refine[i] = (status[i] == ST_RUN && nb != 0.0 && !s_nan) ? 1 : 0;
}

__global__ void batch_axpy_masked_kernel(int64_t m, const int32_t* __restrict__ row_inst,
                                         const int32_t* __restrict__ status, const int32_t* __restrict__ refine,
                                         const double* __restrict__ r, double* __restrict__ x) {
    const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= m) return;
    const int inst = row_inst[k];
    if (status[inst] == ST_RUN && refine[inst]) x[k] += r[k];
}

__global__ void row_inst_kernel(int64_t K, const int64_t* __restrict__ row_off, int32_t* __restrict__ row_inst) {
    const int64_t i = blockIdx.x;
    for (int64_t r = row_off[i] + threadIdx.x; r < row_off[i + 1]; r += blockDim.x) row_inst[r] = (int32_t)i;
}

__global__ void narrow_rp_kernel(int64_t n, const int64_t* __restrict__ in, int32_t* __restrict__ out) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) out[i] = static_cast<int32_t>(in[i]);
}

void free_batch(hn_batch* B) {
    if (!B) return;
    for (void* p : {(void*)B->row_off, (void*)B->col_off, (void*)B->row_inst, (void*)B->dn_off, (void*)B->order,
                    (void*)B->dense, (void*)B->dD, (void*)B->refine, (void*)B->nref, (void*)B->nrp,
                    (void*)B->tile_row, (void*)B->tile_nz, (void*)B->carry_row, (void*)B->head_row,
                    (void*)B->carry_val, (void*)B->head_val, (void*)B->r, (void*)B->ax, (void*)B->step_pairs, (void*)B->step_chunks,
                    (void*)B->solve_part, (void*)B->kkt, (void*)B->kkt_ref, (void*)B->ref_iter, (void*)B->xb,
                    (void*)B->zb, (void*)B->lb})
        dfree(p);
    delete B;
}

KktArgs kkt_args(const hn_batch* B, const double* lam, const double* b, const double* c) {
    return KktArgs{lam,    b,      c,      B->ru,  B->cu,       B->offset, B->kkt,
                   B->kkt_ref, B->xb, B->zb, B->lb, B->ref_iter, B->kkt_tol, B->kkt_extra};
}

SpmvMat n_mat(const hn_batch* B, const double* nval) {
    return SpmvMat{(int)B->m, (int)B->P->nnz, B->nrp, B->P->ci, nval, B->tile_row, B->tile_nz, B->carry_row,
                   B->carry_val, B->head_row, B->head_val, B->ntiles};
}

void solve_all(hn_batch* B, const int32_t* status, const int32_t* refine, double* x, cudaStream_t s) {
    for (int64_t st = 0; st < B->nsteps; ++st) {
        const int cnt = B->step_cnt[st];
        batch_fwd_diag_kernel<<<cnt, kFb, 0, s>>>((int)st, B->row_off, B->dn_off, B->order, status, refine, B->dense, x);
        launched("batch_fwd_diag_kernel");
        const int64_t nc = B->step_chunks_h[st];
        if (nc > 0) {
            batch_fwd_gemv_kernel<<<(unsigned)nc, kT, 0, s>>>((int)st, cnt, B->step_chunks + B->chunk_off_h[st],
                                                              B->row_off, B->dn_off, B->order, status, refine,
                                                              B->dense, x);
            launched("batch_fwd_gemv_kernel");
        }
    }
    batch_scale_kernel<<<(unsigned)((B->m + 255) / 256), 256, 0, s>>>(B->m, B->row_inst, status, refine, B->dD, x);
    launched("batch_scale_kernel");
    for (int64_t st = B->nsteps - 1; st >= 0; --st) {
        const int cnt = B->step_cnt[st];
        const int64_t nc = B->step_chunks_h[st];
        const int64_t* ch = B->step_chunks + B->chunk_off_h[st];
        if (nc > 0) {
            batch_bwd_gemv_kernel<<<(unsigned)nc, kT, 0, s>>>((int)st, cnt, ch, B->row_off, B->dn_off, B->order,
                                                              status, refine, B->dense, x, B->solve_part);
            launched("batch_bwd_gemv_kernel");
        }
        batch_bwd_diag_kernel<<<cnt, kFb, 0, s>>>((int)st, ch, B->row_off, B->dn_off, B->order, status, refine,
                                                  B->dense, B->solve_part, x);
        launched("batch_bwd_diag_kernel");
    }
}

}  // namespace
}  // namespace hn

using namespace hn;

extern "C" {

int hn_batch_create(int64_t K, const int64_t* row_off_host, const int64_t* col_off_host, const hn_pattern* P,
                    hn_batch** out) {
    return guard("hn_batch_create", [&] {
        require_init();
        if (K <= 0 || !row_off_host || !col_off_host || !P || !out) fail(HN_ERR_INVALID_ARG, "bad arguments");
        *out = nullptr;
        const int64_t m = row_off_host[K], n = col_off_host[K];
        if (m != P->m) fail(HN_ERR_INVALID_ARG, "row offsets do not match the pattern");
        std::vector<int64_t> dn(K + 1, 0);
        std::vector<int32_t> order(K);
        for (int64_t i = 0; i < K; ++i) {
            const int64_t mi = row_off_host[i + 1] - row_off_host[i];
            const int64_t ni = col_off_host[i + 1] - col_off_host[i];
            if (mi < 1 || ni < 1) fail(HN_ERR_INVALID_ARG, "every instance needs a row and a column");
            dn[i + 1] = dn[i] + mi * dense_ld(static_cast<int>(mi));
            order[i] = static_cast<int32_t>(i);
        }
        std::stable_sort(order.begin(), order.end(), [&](int32_t a, int32_t b) {
            return row_off_host[a + 1] - row_off_host[a] > row_off_host[b + 1] - row_off_host[b];
        });
        hn_batch* B = new hn_batch();
        cudaStream_t s = nullptr;
        try {
            B->K = K;
            B->m = m;
            B->n = n;
            B->P = P;
            B->row_off = dmalloc<int64_t>(K + 1);
            B->col_off = dmalloc<int64_t>(K + 1);
            B->dn_off = dmalloc<int64_t>(K + 1);
            B->order = dmalloc<int32_t>(K);
            B->row_inst = dmalloc<int32_t>(m);
            B->dense = dmalloc<double>(dn[K]);
            B->dD = dmalloc<double>(m);
            B->refine = dmalloc<int32_t>(K);
            B->nref = dmalloc<int32_t>(1);
            B->r = dmalloc<double>(m);
            B->ax = dmalloc<double>(m);
            B->nrp = dmalloc<int32_t>(m + 1);
            check_cuda(cudaFuncSetAttribute(batch_ldlt_update_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)kUpdSmem),
                       "update smem attribute");
            check_cuda(cudaFuncSetAttribute(batch_ldlt_diag_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)kPanelSmem),
                       "diagonal-block smem attribute");
            B->ref_iter = dmalloc<int32_t>(K);
            B->kkt = dmalloc<double>(4 * K);
            B->kkt_ref = dmalloc<double>(4 * K);
            check_cuda(cudaMemsetAsync(B->ref_iter, 0xff, sizeof(int32_t) * K, s), "memset");  // -1
            check_cuda(cudaMemsetAsync(B->kkt, 0, sizeof(double) * 4 * K, s), "memset");
            check_cuda(cudaMemsetAsync(B->kkt_ref, 0, sizeof(double) * 4 * K, s), "memset");
            check_cuda(cudaMemcpy(B->row_off, row_off_host, sizeof(int64_t) * (K + 1), cudaMemcpyHostToDevice), "H2D");
            check_cuda(cudaMemcpy(B->col_off, col_off_host, sizeof(int64_t) * (K + 1), cudaMemcpyHostToDevice), "H2D");
            check_cuda(cudaMemcpy(B->dn_off, dn.data(), sizeof(int64_t) * (K + 1), cudaMemcpyHostToDevice), "H2D");
            check_cuda(cudaMemcpy(B->order, order.data(), sizeof(int32_t) * K, cudaMemcpyHostToDevice), "H2D");
            row_inst_kernel<<<(unsigned)K, 256, 0, s>>>(K, B->row_off, B->row_inst);
            launched("row_inst_kernel");
            narrow_rp_kernel<<<(unsigned)((m + 1 + 255) / 256), 256, 0, s>>>(m + 1, P->rp, B->nrp);
            launched("narrow_rp_kernel");
            make_tile_table(B->nrp, m, P->nnz, &B->ntiles, &B->tile_row, &B->tile_nz, &B->carry_row, &B->carry_val,
                            &B->head_row, &B->head_val, s);
            // level schedule (instances in decreasing size: the ones with a block
            // at step s form a prefix of `order`)
            const int64_t mmax = row_off_host[order[0] + 1] - row_off_host[order[0]];
            B->nsteps = (mmax + kFb - 1) / kFb;
            B->pair_off_h.assign(1, 0);
            B->chunk_off_h.assign(1, 0);
            std::vector<int64_t> flat, cflat;
            for (int64_t st = 0; st < B->nsteps; ++st) {
                int32_t cnt = 0;
                int64_t acc = 0, cacc = 0;
                for (int64_t b = 0; b < K; ++b) {
                    const int64_t mi = row_off_host[order[b] + 1] - row_off_host[order[b]];
                    if (mi <= st * kFb) break;
                    const int64_t rest = mi - std::min<int64_t>(mi, (st + 1) * kFb);
                    const int64_t T = (rest + kFb - 1) / kFb;
                    acc += T * (T + 1) / 2;
                    flat.push_back(acc);
                    cacc += (rest + kT - 1) / kT;
                    cflat.push_back(cacc);
                    ++cnt;
                }
                B->step_cnt.push_back(cnt);
                B->step_pairs_h.push_back(acc);
                B->pair_off_h.push_back((int64_t)flat.size());
                B->step_chunks_h.push_back(cacc);
                B->chunk_off_h.push_back((int64_t)cflat.size());
            }
            B->step_pairs = dmalloc<int64_t>(flat.size());
            B->step_chunks = dmalloc<int64_t>(cflat.size());
            int64_t maxc = 1;
            for (int64_t c : B->step_chunks_h) maxc = std::max(maxc, c);
            B->solve_part = dmalloc<double>(maxc * kFb);
            check_cuda(cudaMemcpy(B->step_chunks, cflat.data(), sizeof(int64_t) * cflat.size(),
                                  cudaMemcpyHostToDevice),
                       "H2D chunks");
            check_cuda(cudaMemcpy(B->step_pairs, flat.data(), sizeof(int64_t) * flat.size(), cudaMemcpyHostToDevice),
                       "H2D schedule");
            check_cuda(cudaStreamSynchronize(s), "batch create sync");
        } catch (...) {
            free_batch(B);
            throw;
        }
        *out = B;
    });
}

int hn_batch_destroy(hn_batch* B) {
    return guard("hn_batch_destroy", [&] {
        if (!B) return;
        require_init();
        cudaDeviceSynchronize();
        free_batch(B);
    });
}

int hn_batch_residuals(hn_batch* B, const hn_csr* M, const double* x, const double* lam, const double* z,
                       const double* b, const double* c, double* mx, double* rp, double* rd, double* D, double* Drd,
                       double* scal, int32_t* status, int32_t* iters, int iter, double tol, double ctol,
                       void* stream) {
    return guard("hn_batch_residuals", [&] {
        require_init();
        if (!B || !M || !M->has_t) fail(HN_ERR_INVALID_ARG, "bad arguments");
        cudaStream_t s = as_stream(stream);
        spmv_launch(spmv_mat(M, 0), x, EpiResidual{b, mx, rp}, s);
        spmv_launch(spmv_mat(M, 1), lam, EpiDualResidual{z, c, rd}, s);
        batch_prep_kernel<<<(unsigned)B->K, kT, 0, s>>>(B->row_off, B->col_off, x, z, rd, rp, D, Drd, scal, status,
                                                        iters, iter, tol, ctol, kkt_args(B, lam, b, c));
        launched("batch_prep_kernel");
    });
}

int hn_batch_set_kkt(hn_batch* B, const double* ru, const double* cu, const double* offset, double kkt_tol,
                     int extra_iterations) {
    return guard("hn_batch_set_kkt", [&] {
        require_init();
        if (!B || (ru == nullptr) != (cu == nullptr) || (ru && !offset) || extra_iterations < 0)
            fail(HN_ERR_INVALID_ARG, "bad arguments");
        if (kkt_tol > 0.0 && !ru) fail(HN_ERR_INVALID_ARG, "tightening needs the unscale factors");
        B->ru = ru;
        B->cu = cu;
        B->offset = offset;
        B->kkt_tol = kkt_tol > 0.0 ? kkt_tol : 0.0;
        B->kkt_extra = extra_iterations;
        if (B->kkt_tol > 0.0 && !B->xb) {
            B->xb = dmalloc<double>(B->n);
            B->zb = dmalloc<double>(B->n);
            B->lb = dmalloc<double>(B->m);
        }
        check_cuda(cudaMemset(B->ref_iter, 0xff, sizeof(int32_t) * B->K), "memset");
        check_cuda(cudaMemset(B->kkt, 0, sizeof(double) * 4 * B->K), "memset");
        check_cuda(cudaMemset(B->kkt_ref, 0, sizeof(double) * 4 * B->K), "memset");
    });
}

int hn_batch_kkt(const hn_batch* B, double* kkt_host, int32_t* ref_iter_host) {
    return guard("hn_batch_kkt", [&] {
        require_init();
        if (!B) fail(HN_ERR_INVALID_ARG, "null batch");
        check_cuda(cudaDeviceSynchronize(), "sync");
        if (kkt_host)
            check_cuda(cudaMemcpy(kkt_host, B->kkt, sizeof(double) * 4 * B->K, cudaMemcpyDeviceToHost), "D2H kkt");
        if (ref_iter_host)
            check_cuda(cudaMemcpy(ref_iter_host, B->ref_iter, sizeof(int32_t) * B->K, cudaMemcpyDeviceToHost),
                       "D2H ref_iter");
    });
}

int hn_batch_finish(hn_batch* B, double* x, double* z, double* lam, int32_t* status, int32_t* iters, void* stream) {
    return guard("hn_batch_finish", [&] {
        require_init();
        if (!B || !x || !z || !lam || !status || !iters) fail(HN_ERR_INVALID_ARG, "bad arguments");
        cudaStream_t s = as_stream(stream);
        batch_finish_kernel<<<(unsigned)B->K, kT, 0, s>>>(B->row_off, B->col_off, x, z, lam, status, iters,
                                                          kkt_args(B, lam, nullptr, nullptr));
        launched("batch_finish_kernel");
    });
}

int hn_batch_factor(hn_batch* B, const double* D, double reg, double singular_tol, double* nval,
                    const int32_t* status, void* stream) {
    return guard("hn_batch_factor", [&] {
        require_init();
        if (!B || !D || !nval || !status) fail(HN_ERR_INVALID_ARG, "bad arguments");
        cudaStream_t s = as_stream(stream);
        ada_numeric_unregularised(B->P, D, nval, s);
        batch_reg_kernel<<<(unsigned)B->K, kT, 0, s>>>(B->row_off, B->P->diag_pos, reg, status, nval);
        launched("batch_reg_kernel");
        batch_dense_kernel<<<(unsigned)((B->m * 32 + 255) / 256), 256, 0, s>>>(
            B->m, B->row_off, B->row_inst, B->dn_off, status, B->P->rp, B->P->ci, nval, B->dense);
        launched("batch_dense_kernel");
        for (int64_t st = 0; st < B->nsteps; ++st) {
            const int cnt = B->step_cnt[st];
            batch_ldlt_diag_kernel<<<cnt, kT, kPanelSmem, s>>>((int)st, B->row_off, B->dn_off, B->order, status,
                                                               B->dense, B->dD, singular_tol);
            launched("batch_ldlt_diag_kernel");
            const int64_t nc = B->step_chunks_h[st];
            if (nc > 0) {
                batch_ldlt_panel_kernel<<<(unsigned)nc, kT, 0, s>>>((int)st, cnt, B->step_chunks + B->chunk_off_h[st],
                                                                    B->row_off, B->dn_off, B->order, status,
                                                                    B->dense, B->dD);
                launched("batch_ldlt_panel_kernel");
            }
            const int64_t np = B->step_pairs_h[st];
            if (np > 0) {
                const int grid = (int)std::min<int64_t>(np, (int64_t)ctx().sm_count * 2);
                batch_ldlt_update_kernel<<<grid, kT, kUpdSmem, s>>>((int)st, cnt, np, B->step_pairs + B->pair_off_h[st],
                                                             B->row_off, B->dn_off, B->order, status, B->dense,
                                                             B->dD);
                launched("batch_ldlt_update_kernel");
            }
        }
    });
}

int hn_batch_solve(hn_batch* B, const double* nval, const double* rhs, double* x, const int32_t* status,
                   void* stream) {
    return guard("hn_batch_solve", [&] {
        require_init();
        if (!B || !nval || !rhs || !x || !status) fail(HN_ERR_INVALID_ARG, "bad arguments");
        cudaStream_t s = as_stream(stream);
        check_cuda(cudaMemcpyAsync(x, rhs, sizeof(double) * B->m, cudaMemcpyDeviceToDevice, s), "copy rhs");
        solve_all(B, status, nullptr, x, s);
        batch_refine_start_kernel<<<(unsigned)B->K, kT, 0, s>>>(B->row_off, status, rhs, B->refine);
        launched("batch_refine_start_kernel");
        const SpmvMat N = n_mat(B, nval);
        for (int sweep = 0; sweep < 5; ++sweep) {
            spmv_launch(N, x, EpiAxpby{1.0, 0.0, B->ax}, s);
            check_cuda(cudaMemsetAsync(B->nref, 0, sizeof(int32_t), s), "memset");
            batch_refine_check_kernel<<<(unsigned)B->K, kT, 0, s>>>(B->row_off, status, rhs, B->ax, B->r, B->refine,
                                                                    B->nref);
            launched("batch_refine_check_kernel");
            int32_t left = 0;
            check_cuda(cudaMemcpyAsync(&left, B->nref, sizeof(left), cudaMemcpyDeviceToHost, s), "D2H");
            check_cuda(cudaStreamSynchronize(s), "refine sync");
            if (left == 0) break;
            solve_all(B, status, B->refine, B->r, s);
            batch_axpy_masked_kernel<<<(unsigned)((B->m + 255) / 256), 256, 0, s>>>(B->m, B->row_inst, status,
                                                                                    B->refine, B->r, x);
            launched("batch_axpy_masked_kernel");
        }
    });
}

int hn_batch_steps(hn_batch* B, const double* x, const double* dx, const double* z, const double* dz,
                   const double* dlam, double* scal, int32_t* status, void* stream) {
    return guard("hn_batch_steps", [&] {
        require_init();
        if (!B) fail(HN_ERR_INVALID_ARG, "null batch");
        cudaStream_t s = as_stream(stream);
        batch_steps_kernel<<<(unsigned)B->K, kT, 0, s>>>(B->row_off, B->col_off, x, dx, z, dz, dlam, scal, status);
        launched("batch_steps_kernel");
    });
}

int hn_batch_corrector(hn_batch* B, const hn_csr* M, const double* x, const double* dx, const double* z,
                       const double* dz, const double* rhs_pred, double* zs, double* rhs, double* scal,
                       const int32_t* status, void* stream) {
    return guard("hn_batch_corrector", [&] {
        require_init();
        if (!B || !M) fail(HN_ERR_INVALID_ARG, "bad arguments");
        cudaStream_t s = as_stream(stream);
        batch_corr_kernel<<<(unsigned)B->K, kT, 0, s>>>(B->col_off, x, dx, z, dz, scal, status, zs);
        launched("batch_corr_kernel");
        spmv_launch(spmv_mat(M, 0), zs, EpiCorrRhs{rhs_pred, rhs}, s);
    });
}

int hn_batch_update(hn_batch* B, double* x, const double* dx, double* z, const double* dz, double* lam,
                    const double* dlam, const double* scal, int32_t* status, int32_t* iters, int iter,
                    void* stream) {
    return guard("hn_batch_update", [&] {
        require_init();
        if (!B) fail(HN_ERR_INVALID_ARG, "null batch");
        cudaStream_t s = as_stream(stream);
        batch_update_kernel<<<(unsigned)B->K, kT, 0, s>>>(B->row_off, B->col_off, x, dx, z, dz, lam, dlam, scal,
                                                          status, iters, iter);
        launched("batch_update_kernel");
    });
}

}  // extern "C"
