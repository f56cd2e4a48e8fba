// Fused device kernels of one Mehrotra predictor-corrector iteration
// (core/lp/interior_point.cpp:507-708). Each SpMV carries its elementwise
// follow-up in the epilogue, so the vectors of the iteration are streamed as
// few times as possible:
//
//   residuals : mx = M x, rp = mx - b (:507-512);  rd = M^T lam + z - c (:514-515)
//               then one pass: mu = x^T z / n, ||rp||_inf, ||rd||_inf (:517-530),
//               D = x / z clamped to (0, 1e10] (:532-539), Drd = D rd (:584)
//   rhs       : rhs = -rp - M(Drd) + mx (:585-600; M x reuses mx)
//   direction : t = M^T dlam; dx = D (t + rd) - x (+ corr); dz = -(t + rd) (:607-615, :666-673)
//   steps     : alpha_p = max_step(x, dx), alpha_d = max_step(z, dz) (:134-142),
//               plus the non-finite guards of :617-627
//   corrector : mu_aff (:632-636), sigma (:638-643), zs = (sigma mu - dx dz) (1/z)
//               (:645-651), rhs = rhs_pred - M zs (:652-659)
//   update    : x += ap dx, z += ad dz, lam += ad dlam and the guard of :698-708
//
// Scalars stay on the device in a double[HN_IPM_NSCAL] block; the host reads
// it once per decision (convergence, guards). Reductions are deterministic
// (fixed per-block trees, partials folded in block order by the last block).
#include <cmath>

#include "hn_spmv.cuh"

namespace hn {
namespace {

constexpr int kT = 256;

__device__ __forceinline__ bool finite(double v) { return isfinite(v); }

__device__ __forceinline__ unsigned long long* flags_of(double* scal) {
    return reinterpret_cast<unsigned long long*>(scal + HN_IPM_FLAGS);
}

// Last-block-done helper: returns true in every thread of the block that
// finished last (partials of all blocks are then visible).
__device__ __forceinline__ bool last_block(unsigned* counter) {
    __shared__ bool last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = (atomicAdd(counter, 1u) == gridDim.x - 1);
    __syncthreads();
    if (last) __threadfence();
    return last;
}

__global__ void __launch_bounds__(kT) prep_kernel(int64_t n, int64_t m, const double* __restrict__ x,
                                                  const double* __restrict__ z, const double* __restrict__ rd,
                                                  const double* __restrict__ rp, double* __restrict__ D,
                                                  double* __restrict__ Drd, double* partials, unsigned* counter,
                                                  double* scal) {
    __shared__ double sh[32];
    double smu = 0.0, mrd = 0.0, mrp = 0.0;
    const int64_t stride = (int64_t)gridDim.x * kT;
    for (int64_t j = blockIdx.x * (int64_t)kT + threadIdx.x; j < n; j += stride) {
        const double xj = x[j], zj = z[j], r = rd[j];
        smu += xj * zj;
        mrd = fmax(mrd, fabs(r));
        double d = xj / zj;
        if (!(d >= 0.0) || !finite(d) || d > 1e10) d = 1e10;
        D[j] = d;
        Drd[j] = d * r;
    }
    for (int64_t i = blockIdx.x * (int64_t)kT + threadIdx.x; i < m; i += stride) mrp = fmax(mrp, fabs(rp[i]));
    const double bs = block_sum<kT>(smu, sh);
    const double bd = block_max<kT>(mrd, sh);
    const double bp = block_max<kT>(mrp, sh);
    const int G = gridDim.x;
    if (threadIdx.x == 0) {
        partials[blockIdx.x] = bs;
        partials[G + blockIdx.x] = bd;
        partials[2 * G + blockIdx.x] = bp;
    }
    if (!last_block(counter)) return;
    double s = 0.0, a = 0.0, c = 0.0;
    for (int i = threadIdx.x; i < G; i += kT) {
        s += __ldcg(partials + i);
        a = fmax(a, __ldcg(partials + G + i));
        c = fmax(c, __ldcg(partials + 2 * G + i));
    }
    s = block_sum<kT>(s, sh);
    a = block_max<kT>(a, sh);
    c = block_max<kT>(c, sh);
    if (threadIdx.x == 0) {
        scal[HN_IPM_MU] = s / static_cast<double>(n);
        scal[HN_IPM_NRD] = a;
        scal[HN_IPM_NRP] = c;
        *counter = 0u;
    }
}

__global__ void __launch_bounds__(kT) steps_kernel(int64_t n, int64_t m, const double* __restrict__ x,
                                                   const double* __restrict__ dx, const double* __restrict__ z,
                                                   const double* __restrict__ dz, const double* __restrict__ dlam,
                                                   double* partials, unsigned* counter, double* scal) {
    __shared__ double sh[32];
    __shared__ int s_bad;
    if (threadIdx.x == 0) s_bad = 0;
    __syncthreads();
    double ap = 1.0, ad = 1.0;
    bool bad = false;
    const int64_t stride = (int64_t)gridDim.x * kT;
    for (int64_t j = blockIdx.x * (int64_t)kT + threadIdx.x; j < n; j += stride) {
        const double a = dx[j], b = dz[j];
        if (a < 0.0) ap = fmin(ap, -x[j] / a);
        if (b < 0.0) ad = fmin(ad, -z[j] / b);
        bad |= !finite(a) || !finite(b);
    }
    for (int64_t i = blockIdx.x * (int64_t)kT + threadIdx.x; i < m; i += stride) bad |= !finite(dlam[i]);
    if (bad) s_bad = 1;
    const double bp = block_min<kT>(ap, sh);
    const double bq = block_min<kT>(ad, sh);
    const int G = gridDim.x;
    if (threadIdx.x == 0) {
        partials[blockIdx.x] = bp;
        partials[G + blockIdx.x] = bq;
        if (s_bad) atomicOr(flags_of(scal), 1ull);
    }
    if (!last_block(counter)) return;
    double p = 1.0, q = 1.0;
    for (int i = threadIdx.x; i < G; i += kT) {
        p = fmin(p, __ldcg(partials + i));
        q = fmin(q, __ldcg(partials + G + i));
    }
    p = block_min<kT>(p, sh);
    q = block_min<kT>(q, sh);
    if (threadIdx.x == 0) {
        const double sp = 0.99 * p, sq = 0.99 * q;
        scal[HN_IPM_AP] = sp < 1.0 ? sp : 1.0;  // std::min(1.0, 0.99 * alpha)
        scal[HN_IPM_AD] = sq < 1.0 ? sq : 1.0;
        *counter = 0u;
    }
}

__global__ void __launch_bounds__(kT) mu_aff_kernel(int64_t n, const double* __restrict__ x,
                                                    const double* __restrict__ dx, const double* __restrict__ z,
                                                    const double* __restrict__ dz, double* partials,
                                                    unsigned* counter, double* scal) {
    __shared__ double sh[32];
    const double ap = scal[HN_IPM_AP], ad = scal[HN_IPM_AD];
    double s = 0.0;
    const int64_t stride = (int64_t)gridDim.x * kT;
    for (int64_t j = blockIdx.x * (int64_t)kT + threadIdx.x; j < n; j += stride)
        s += (x[j] + ap * dx[j]) * (z[j] + ad * dz[j]);
    s = block_sum<kT>(s, sh);
    if (threadIdx.x == 0) partials[blockIdx.x] = s;
    if (!last_block(counter)) return;
    double t = 0.0;
    for (int i = threadIdx.x; i < (int)gridDim.x; i += kT) t += __ldcg(partials + i);
    t = block_sum<kT>(t, sh);
    if (threadIdx.x == 0) {
        const double mu_aff = t / static_cast<double>(n);
        const double mu = scal[HN_IPM_MU];
        double sigma;
        if (!finite(mu_aff) || mu_aff < 0.0 || !(mu > 0.0)) {
            sigma = 0.5;
        } else {
            const double r = pow(mu_aff / fmax(mu, 1e-300), 3.0);
            sigma = r < 0.1 ? 0.1 : (r > 0.9 ? 0.9 : r);  // std::clamp
        }
        scal[HN_IPM_MUAFF] = mu_aff;
        scal[HN_IPM_SIGMA] = sigma;
        *counter = 0u;
    }
}

__global__ void corr_term_kernel(int64_t n, const double* __restrict__ dx, const double* __restrict__ dz,
                                 const double* __restrict__ z, const double* __restrict__ scal,
                                 double* __restrict__ zs) {
    const double sm = scal[HN_IPM_SIGMA] * scal[HN_IPM_MU];
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n; j += stride) {
        const double zinv = 1.0 / z[j];
        zs[j] = (sm - dx[j] * dz[j]) * zinv;
    }
}

__global__ void __launch_bounds__(kT) update_kernel(int64_t n, int64_t m, double* __restrict__ x,
                                                    const double* __restrict__ dx, double* __restrict__ z,
                                                    const double* __restrict__ dz, double* __restrict__ lam,
                                                    const double* __restrict__ dlam, double* scal) {
    __shared__ int s_bad;
    if (threadIdx.x == 0) s_bad = 0;
    __syncthreads();
    const double ap = scal[HN_IPM_AP], ad = scal[HN_IPM_AD];
    bool bad = false;
    const int64_t stride = (int64_t)gridDim.x * kT;
    for (int64_t j = blockIdx.x * (int64_t)kT + threadIdx.x; j < n; j += stride) {
        const double xn = x[j] + ap * dx[j];
        const double zn = z[j] + ad * dz[j];
        x[j] = xn;
        z[j] = zn;
        bad |= xn < 0.0 || zn < 0.0 || !finite(xn) || !finite(zn);
    }
    for (int64_t i = blockIdx.x * (int64_t)kT + threadIdx.x; i < m; i += stride) lam[i] += ad * dlam[i];
    if (bad) s_bad = 1;
    __syncthreads();
    if (threadIdx.x == 0 && s_bad) atomicOr(flags_of(scal), 2ull);
}

__global__ void __launch_bounds__(kT) max_step_kernel(int64_t n, const double* __restrict__ v,
                                                      const double* __restrict__ d, double* partials,
                                                      unsigned* counter, double* out) {
    __shared__ double sh[32];
    double a = 1.0;
    const int64_t stride = (int64_t)gridDim.x * kT;
    for (int64_t j = blockIdx.x * (int64_t)kT + threadIdx.x; j < n; j += stride)
        if (d[j] < 0.0) a = fmin(a, -v[j] / d[j]);
    a = block_min<kT>(a, sh);
    if (threadIdx.x == 0) partials[blockIdx.x] = a;
    if (!last_block(counter)) return;
    double p = 1.0;
    for (int i = threadIdx.x; i < (int)gridDim.x; i += kT) p = fmin(p, __ldcg(partials + i));
    p = block_min<kT>(p, sh);
    if (threadIdx.x == 0) {
        const double s = 0.99 * p;
        *out = s < 1.0 ? s : 1.0;
        *counter = 0u;
    }
}

// Relative KKT residual of the iterate with the scaling undone: per block the
// maxima of |rp| ru, |b| ru, |rd| cu, |c| cu and the sums c^T x, b^T lam; the
// last block folds the partials in block order (deterministic).
constexpr int kKktMaxBlocks = 592;  // 6 partial arrays fit the workspace's 4 x kMaxReduceBlocks
static_assert(6 * kKktMaxBlocks <= 4 * kMaxReduceBlocks, "kkt partials exceed the workspace");

__global__ void __launch_bounds__(kT) kkt_kernel(int64_t n, int64_t m, const double* __restrict__ x,
                                                 const double* __restrict__ lam, const double* __restrict__ b,
                                                 const double* __restrict__ c, const double* __restrict__ rp,
                                                 const double* __restrict__ rd, const double* __restrict__ ru,
                                                 const double* __restrict__ cu, double offset, double* partials,
                                                 unsigned* counter, double* out) {
    __shared__ double sh[32];
    double pr = 0.0, bn = 0.0, du = 0.0, cn = 0.0, cx = 0.0, by = 0.0;
    const int64_t stride = (int64_t)gridDim.x * kT;
    for (int64_t j = blockIdx.x * (int64_t)kT + threadIdx.x; j < n; j += stride) {
        const double u = cu[j], cj = c[j];
        const double t = fabs(rd[j]) * u;
        du = fmax(du, t <= 1.7976931348623157e308 ? t : INFINITY);  // NaN or inf counts as infinite
        cn = fmax(cn, fabs(cj) * u);
        cx += cj * x[j];
    }
    for (int64_t i = blockIdx.x * (int64_t)kT + threadIdx.x; i < m; i += stride) {
        const double u = ru[i], bi = b[i];
        const double t = fabs(rp[i]) * u;
        pr = fmax(pr, t <= 1.7976931348623157e308 ? t : INFINITY);
        bn = fmax(bn, fabs(bi) * u);
        by += bi * lam[i];
    }
    const int G = gridDim.x;
    const double v0 = block_max<kT>(pr, sh), v1 = block_max<kT>(bn, sh), v2 = block_max<kT>(du, sh),
                 v3 = block_max<kT>(cn, sh), v4 = block_sum<kT>(cx, sh), v5 = block_sum<kT>(by, sh);
    if (threadIdx.x == 0) {
        partials[blockIdx.x] = v0;
        partials[G + blockIdx.x] = v1;
        partials[2 * G + blockIdx.x] = v2;
        partials[3 * G + blockIdx.x] = v3;
        partials[4 * G + blockIdx.x] = v4;
        partials[5 * G + blockIdx.x] = v5;
    }
    if (!last_block(counter)) return;
    double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0, a4 = 0.0, a5 = 0.0;
    for (int k = threadIdx.x; k < G; k += kT) {
        a0 = fmax(a0, __ldcg(partials + k));
        a1 = fmax(a1, __ldcg(partials + G + k));
        a2 = fmax(a2, __ldcg(partials + 2 * G + k));
        a3 = fmax(a3, __ldcg(partials + 3 * G + k));
        a4 += __ldcg(partials + 4 * G + k);
        a5 += __ldcg(partials + 5 * G + k);
    }
    a0 = block_max<kT>(a0, sh);
    a1 = block_max<kT>(a1, sh);
    a2 = block_max<kT>(a2, sh);
    a3 = block_max<kT>(a3, sh);
    a4 = block_sum<kT>(a4, sh);
    a5 = block_sum<kT>(a5, sh);
    if (threadIdx.x == 0) {
        const double P = a0 / (1.0 + a1), Dl = a2 / (1.0 + a3), Gp = fabs(a4 - a5) / (1.0 + fabs(a4 + offset));
        // NaN in any part makes the whole residual NaN (never "converged")
        out[0] = (P != P || Dl != Dl || Gp != Gp) ? nan("") : fmax(P, fmax(Dl, Gp));
        out[1] = P;
        out[2] = Dl;
        out[3] = Gp;
        *counter = 0u;
    }
}

int red_grid(int64_t n) { return grid_for(n, kT * 4, kMaxReduceBlocks); }

void need_t(const hn_csr* A) {
    if (!A) fail(HN_ERR_INVALID_ARG, "null matrix handle");
    if (!A->has_t) fail(HN_ERR_INVALID_ARG, "IPM kernels need a handle with A^T");
}

}  // namespace
}  // namespace hn

using namespace hn;

extern "C" {

int hn_ipm_residuals(const hn_csr* A, const double* x, const double* lam, const double* z, const double* b,
                     const double* c, double* mx, double* rp, double* rd, double* D, double* Drd, double* scal,
                     void* stream) {
    return guard("hn_ipm_residuals", [&] {
        require_init();
        need_t(A);
        cudaStream_t s = as_stream(stream);
        spmv_launch(spmv_mat(A, 0), x, EpiResidual{b, mx, rp}, s);
        spmv_launch(spmv_mat(A, 1), lam, EpiDualResidual{z, c, rd}, s);
        Workspace& w = workspace(s);
        const int64_t big = A->n > A->m ? A->n : A->m;
        prep_kernel<<<red_grid(big), kT, 0, s>>>(A->n, A->m, x, z, rd, rp, D, Drd, w.partials, w.counter, scal);
        launched("prep_kernel");
    });
}

int hn_ipm_rhs(const hn_csr* A, const double* Drd, const double* rp, const double* mx, double* rhs,
               void* stream) {
    return guard("hn_ipm_rhs", [&] {
        require_init();
        need_t(A);
        spmv_launch(spmv_mat(A, 0), Drd, EpiRhs{rp, mx, rhs}, as_stream(stream));
    });
}

int hn_ipm_direction(const hn_csr* A, const double* dlam, const double* D, const double* rd, const double* x,
                     const double* corr, double* dx, double* dz, void* stream) {
    return guard("hn_ipm_direction", [&] {
        require_init();
        need_t(A);
        spmv_launch(spmv_mat(A, 1), dlam, EpiDirection{D, rd, x, corr, dx, dz}, as_stream(stream));
    });
}

int hn_ipm_step_lengths(int64_t n, int64_t m, const double* x, const double* dx, const double* z,
                        const double* dz, const double* dlam, double* scal, void* stream) {
    return guard("hn_ipm_step_lengths", [&] {
        require_init();
        cudaStream_t s = as_stream(stream);
        Workspace& w = workspace(s);
        steps_kernel<<<red_grid(n > m ? n : m), kT, 0, s>>>(n, m, x, dx, z, dz, dlam, w.partials, w.counter, scal);
        launched("steps_kernel");
    });
}

int hn_ipm_corrector(const hn_csr* A, const double* x, const double* dx, const double* z, const double* dz,
                     const double* rhs_pred, double* zs, double* rhs, double* scal, void* stream) {
    return guard("hn_ipm_corrector", [&] {
        require_init();
        need_t(A);
        cudaStream_t s = as_stream(stream);
        Workspace& w = workspace(s);
        const int64_t n = A->n;
        mu_aff_kernel<<<red_grid(n), kT, 0, s>>>(n, x, dx, z, dz, w.partials, w.counter, scal);
        launched("mu_aff_kernel");
        corr_term_kernel<<<grid_for(n, kT, ctx().sm_count * 16), kT, 0, s>>>(n, dx, dz, z, scal, zs);
        launched("corr_term_kernel");
        spmv_launch(spmv_mat(A, 0), zs, EpiCorrRhs{rhs_pred, rhs}, s);
    });
}

int hn_ipm_update(int64_t n, int64_t m, double* x, const double* dx, double* z, const double* dz, double* lam,
                  const double* dlam, double* scal, void* stream) {
    return guard("hn_ipm_update", [&] {
        require_init();
        cudaStream_t s = as_stream(stream);
        update_kernel<<<grid_for(n > m ? n : m, kT, ctx().sm_count * 16), kT, 0, s>>>(n, m, x, dx, z, dz, lam,
                                                                                     dlam, scal);
        launched("update_kernel");
    });
}

int hn_ipm_kkt(int64_t n, int64_t m, const double* x, const double* lam, const double* b, const double* c,
               const double* rp, const double* rd, const double* ru, const double* cu, double offset, double* kkt,
               void* stream) {
    return guard("hn_ipm_kkt", [&] {
        require_init();
        if (n < 1 || m < 0 || !x || !c || !rd || !cu || !kkt || (m > 0 && (!lam || !b || !rp || !ru)))
            fail(HN_ERR_INVALID_ARG, "bad arguments");
        cudaStream_t s = as_stream(stream);
        Workspace& w = workspace(s);
        kkt_kernel<<<grid_for(n > m ? n : m, kT * 4, kKktMaxBlocks), kT, 0, s>>>(n, m, x, lam, b, c, rp, rd, ru, cu,
                                                                                  offset, w.partials, w.counter, kkt);
        launched("kkt_kernel");
    });
}

int hn_max_step(int64_t n, const double* v, const double* d, double* result, void* stream) {
    return guard("hn_max_step", [&] {
        require_init();
        if (n < 0 || !result) fail(HN_ERR_INVALID_ARG, "bad arguments");
        cudaStream_t s = as_stream(stream);
        Workspace& w = workspace(s);
        max_step_kernel<<<red_grid(n), kT, 0, s>>>(n, v, d, w.partials, w.counter, result);
        launched("max_step_kernel");
    });
}

}  // extern "C"
