// Revised-simplex pricing on the device: the per-iteration O(nnz + n) work of
// HyperNova's SimplexSolver (core/lp/simplex.cpp), over the matrix's device
// A^T. The basis factorisation (FTRAN/BTRAN) stays on the host.
//
//   hn_price_reduced_costs  rc = c - A^T y                    (compute_reduced_costs, :1225-1233)
//   hn_price_devex_update   alpha = A^T u; s = max |alpha_j| over nonbasic j;
//                           w_j = max(w_j, (alpha_j / s)^2)    (update_devex_weights, :1235-1271)
//   hn_price_select         Bland: first improving column;
//                           ranked: the k best by |rc_j|/sqrt(w_j), index
//                           ascending on ties                  (select_entering_variable,
//                                                               ranked_candidates, :1283-1361)
//   hn_price_columns        dense columns a_j of A             (extract_column, :25-35)
//
// A^T x sums each column's contributions in increasing row order, which is
// the order of SparseMatrix::transpose_multiply's and update_devex_weights's
// scatters, so reduced costs and Devex rows are bit-identical to the
// reference's. Selection reduces with atomic max/min on integer keys, whose
// result does not depend on the order the blocks arrive in.
#include <algorithm>
#include <climits>

#include "hn_spmv.cuh"

namespace hn {
namespace {

constexpr int kPT = 256;
constexpr int kPriceBlocks = 148 * 4;

// workspace select words
constexpr int W_COUNT = 0, W_FIRST = 1, W_PREV_S = 2, W_PREV_I = 3, W_BEST_S = 4, W_BEST_I = 5, W_HAVE_PREV = 6;

struct EpiReducedCost {
    const double* cost;
    double* rc;
    __device__ __forceinline__ void operator()(int j, double s) const { rc[j] = cost[j] - s; }
};

// s = max over nonbasic j of |alpha_j| (std::max from 0.0, NaN-ignoring).
__global__ void __launch_bounds__(kPT) devex_scale_kernel(int64_t n, const double* __restrict__ alpha,
                                                          const int32_t* __restrict__ nonbasis,
                                                          double* __restrict__ partials,
                                                          unsigned* __restrict__ counter, double* __restrict__ out) {
    __shared__ double sh[32];
    __shared__ bool last;
    double v = 0.0;
    for (int64_t j = blockIdx.x * (int64_t)kPT + threadIdx.x; j < n; j += (int64_t)gridDim.x * kPT)
        if (nonbasis[j] >= 0) v = fmax(v, fabs(alpha[j]));
    double r = block_max<kPT>(v, sh);
    if (threadIdx.x == 0) {
        partials[blockIdx.x] = r;
        __threadfence();
        last = atomicAdd(counter, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    double t = 0.0;
    for (int i = threadIdx.x; i < (int)gridDim.x; i += kPT) t = fmax(t, __ldcg(partials + i));
    r = block_max<kPT>(t, sh);
    if (threadIdx.x == 0) {
        *out = r;
        *counter = 0u;
    }
}

__global__ void __launch_bounds__(kPT) devex_apply_kernel(int64_t n, const double* __restrict__ alpha,
                                                          const int32_t* __restrict__ nonbasis,
                                                          const double* __restrict__ scale,
                                                          double* __restrict__ w) {
    const double s = *scale;
    if (s == 0.0) return;
    for (int64_t j = blockIdx.x * (int64_t)kPT + threadIdx.x; j < n; j += (int64_t)gridDim.x * kPT) {
        if (nonbasis[j] < 0) continue;
        const double t = alpha[j] / s;
        const double q = t * t;
        if (q > w[j]) w[j] = q;
    }
}

struct PriceArgs {
    int64_t n;
    const double* rc;
    const double* w;
    const int32_t* nonbasis;
    const uint8_t* artificial;
    int phase1, maximize;
    double tol;
};

// Improving nonbasic column j (the filters of ranked_candidates and of the
// Bland scan); score = |rc_j| / sqrt(w_j) with w guarded to 1.
__device__ __forceinline__ bool eligible(const PriceArgs& a, int64_t j, double& score) {
    if (a.nonbasis[j] < 0) return false;
    if (!a.phase1 && a.artificial && a.artificial[j]) return false;
    double rc = a.rc[j];
    if (a.maximize) rc = -rc;
    if (!(rc < -a.tol)) return false;
    double w = a.w ? a.w[j] : 1.0;
    if (!(w > 0.0) || !isfinite(w)) w = 1.0;
    score = fabs(rc) / sqrt(w);
    return true;
}

__device__ __forceinline__ unsigned long long warp_max_u64(unsigned long long v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long u = __shfl_xor_sync(0xffffffffu, v, o);
        v = u > v ? u : v;
    }
    return v;
}
__device__ __forceinline__ unsigned long long warp_min_u64(unsigned long long v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long u = __shfl_xor_sync(0xffffffffu, v, o);
        v = u < v ? u : v;
    }
    return v;
}

__global__ void price_init_kernel(unsigned long long* sel) {
    if (threadIdx.x == 0) {
        sel[W_COUNT] = 0ull;
        sel[W_FIRST] = ULLONG_MAX;
        sel[W_PREV_S] = 0ull;
        sel[W_PREV_I] = 0ull;
        sel[W_BEST_S] = 0ull;
        sel[W_BEST_I] = ULLONG_MAX;
        sel[W_HAVE_PREV] = 0ull;
    }
}

// Count of improving columns and the first one (Bland).
__global__ void __launch_bounds__(kPT) price_count_kernel(PriceArgs a, unsigned long long* sel) {
    unsigned long long cnt = 0, first = ULLONG_MAX;
    for (int64_t j = blockIdx.x * (int64_t)kPT + threadIdx.x; j < a.n; j += (int64_t)gridDim.x * kPT) {
        double sc;
        if (eligible(a, j, sc)) {
            ++cnt;
            if ((unsigned long long)j < first) first = (unsigned long long)j;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
    first = warp_min_u64(first);
    if ((threadIdx.x & 31) == 0) {
        if (cnt) atomicAdd(sel + W_COUNT, cnt);
        if (first != ULLONG_MAX) atomicMin(sel + W_FIRST, first);
    }
}

// The previous pick of the ranking; (score, j) is eligible for this round when
// it comes after it in the order (score desc, index asc).
struct Prev {
    bool have;
    unsigned long long s, i;
    __device__ __forceinline__ explicit Prev(const unsigned long long* sel)
        : have(sel[W_HAVE_PREV] != 0ull), s(sel[W_PREV_S]), i(sel[W_PREV_I]) {}
    __device__ __forceinline__ bool admits(unsigned long long sb, int64_t j) const {
        return !have || sb < s || (sb == s && (unsigned long long)j > i);
    }
};

// Round stage 1: the best score among columns after the previous pick.
// Scores are positive doubles, whose bit patterns order like their values.
__global__ void __launch_bounds__(kPT) price_best_score_kernel(PriceArgs a, unsigned long long* sel) {
    const Prev prev(sel);
    unsigned long long best = 0ull;
    for (int64_t j = blockIdx.x * (int64_t)kPT + threadIdx.x; j < a.n; j += (int64_t)gridDim.x * kPT) {
        double sc;
        if (!eligible(a, j, sc)) continue;
        const unsigned long long sb = (unsigned long long)__double_as_longlong(sc);
        if (prev.admits(sb, j) && sb > best) best = sb;
    }
    best = warp_max_u64(best);
    if ((threadIdx.x & 31) == 0 && best) atomicMax(sel + W_BEST_S, best);
}

// Round stage 2: the lowest index holding that score.
__global__ void __launch_bounds__(kPT) price_best_index_kernel(PriceArgs a, unsigned long long* sel) {
    const unsigned long long target = sel[W_BEST_S];
    if (!target) return;
    const Prev prev(sel);
    unsigned long long bi = ULLONG_MAX;
    for (int64_t j = blockIdx.x * (int64_t)kPT + threadIdx.x; j < a.n; j += (int64_t)gridDim.x * kPT) {
        double sc;
        if (!eligible(a, j, sc)) continue;
        const unsigned long long sb = (unsigned long long)__double_as_longlong(sc);
        if (sb == target && prev.admits(sb, j) && (unsigned long long)j < bi) bi = (unsigned long long)j;
    }
    bi = warp_min_u64(bi);
    if ((threadIdx.x & 31) == 0 && bi != ULLONG_MAX) atomicMin(sel + W_BEST_I, bi);
}

// Round close: record the pick (or -1) and make it the new "previous".
__global__ void price_round_close_kernel(unsigned long long* sel, int64_t* out, int64_t r) {
    if (threadIdx.x != 0) return;
    if (sel[W_BEST_S]) {
        out[1 + r] = (int64_t)sel[W_BEST_I];
        sel[W_PREV_S] = sel[W_BEST_S];
        sel[W_PREV_I] = sel[W_BEST_I];
        sel[W_HAVE_PREV] = 1ull;
    } else {
        out[1 + r] = -1;
        sel[W_PREV_S] = 0ull;  // nothing sorts after a score of 0: later rounds find nothing
        sel[W_PREV_I] = ULLONG_MAX;
        sel[W_HAVE_PREV] = 1ull;
    }
    sel[W_BEST_S] = 0ull;
    sel[W_BEST_I] = ULLONG_MAX;
}

__global__ void price_bland_close_kernel(const unsigned long long* sel, int64_t* out) {
    if (threadIdx.x != 0) return;
    out[0] = (int64_t)sel[W_COUNT];
    out[1] = sel[W_FIRST] == ULLONG_MAX ? -1 : (int64_t)sel[W_FIRST];
}

__global__ void price_count_close_kernel(const unsigned long long* sel, int64_t* out) {
    if (threadIdx.x == 0) out[0] = (int64_t)sel[W_COUNT];
}

// Columns outside [0, n) are left zero and counted in *bad.
__global__ void __launch_bounds__(kPT) column_gather_kernel(int64_t m, int64_t n, const int32_t* __restrict__ rpT,
                                                            const int32_t* __restrict__ ciT,
                                                            const double* __restrict__ valT,
                                                            const int64_t* __restrict__ cols, double* __restrict__ out,
                                                            unsigned long long* bad) {
    const int64_t r = blockIdx.x;
    const int64_t j = cols[r];
    if (j < 0 || j >= n) {
        if (threadIdx.x == 0) atomicAdd(bad, 1ull);
        return;
    }
    double* o = out + r * m;
    for (int32_t e = rpT[j] + threadIdx.x; e < rpT[j + 1]; e += kPT) o[ciT[e]] = valT[e];
}

int price_grid(int64_t n) {
    const int64_t b = (n + kPT - 1) / kPT;
    return (int)std::max<int64_t>(1, std::min<int64_t>(b, kPriceBlocks));
}

}  // namespace
}  // namespace hn

using namespace hn;

extern "C" {

int hn_price_reduced_costs(const hn_csr* A, const double* y, const double* cost, double* rc, void* stream) {
    return guard("hn_price_reduced_costs", [&] {
        require_init();
        if (!A || !y || !cost || !rc) fail(HN_ERR_INVALID_ARG, "null argument");
        if (!A->has_t) fail(HN_ERR_INVALID_ARG, "matrix was created without its transpose");
        spmv_launch(spmv_mat(A, 1), y, EpiReducedCost{cost, rc}, as_stream(stream));
    });
}

int hn_price_devex_update(const hn_csr* A, const double* u, const int32_t* nonbasis, double* weights,
                          double* alpha, void* stream) {
    return guard("hn_price_devex_update", [&] {
        require_init();
        if (!A || !u || !nonbasis || !weights || !alpha) fail(HN_ERR_INVALID_ARG, "null argument");
        if (!A->has_t) fail(HN_ERR_INVALID_ARG, "matrix was created without its transpose");
        cudaStream_t s = as_stream(stream);
        Workspace& w = workspace(s);
        spmv_launch(spmv_mat(A, 1), u, EpiAxpby{1.0, 0.0, alpha}, s);
        const int g = price_grid(A->n);
        double* scale = w.partials + 4 * kMaxReduceBlocks;
        devex_scale_kernel<<<g, kPT, 0, s>>>(A->n, alpha, nonbasis, w.partials, w.counter, scale);
        launched("devex_scale_kernel");
        devex_apply_kernel<<<g, kPT, 0, s>>>(A->n, alpha, nonbasis, scale, weights);
        launched("devex_apply_kernel");
    });
}

int hn_price_select(int64_t n, const double* rc, const double* weights, const int32_t* nonbasis,
                    const uint8_t* artificial, int phase1, int maximize, double optimality_tol, int rule, int64_t k,
                    int64_t* out, void* stream) {
    return guard("hn_price_select", [&] {
        require_init();
        if (n < 0 || !out || (n > 0 && (!rc || !nonbasis))) fail(HN_ERR_INVALID_ARG, "bad arguments");
        if (rule != HN_PRICE_BLAND && rule != HN_PRICE_RANKED) fail(HN_ERR_INVALID_ARG, "unknown pricing rule");
        if (rule == HN_PRICE_RANKED && (k < 1 || k > HN_PRICE_MAX_K)) fail(HN_ERR_INVALID_ARG, "k out of range");
        cudaStream_t s = as_stream(stream);
        Workspace& w = workspace(s);
        const PriceArgs a{n, rc, weights, nonbasis, artificial, phase1, maximize, optimality_tol};
        const int g = price_grid(n);
        price_init_kernel<<<1, 32, 0, s>>>(w.select);
        launched("price_init_kernel");
        price_count_kernel<<<g, kPT, 0, s>>>(a, w.select);
        launched("price_count_kernel");
        if (rule == HN_PRICE_BLAND) {
            price_bland_close_kernel<<<1, 32, 0, s>>>(w.select, out);
            launched("price_bland_close_kernel");
            return;
        }
        price_count_close_kernel<<<1, 32, 0, s>>>(w.select, out);
        launched("price_count_close_kernel");
        for (int64_t r = 0; r < k; ++r) {
            price_best_score_kernel<<<g, kPT, 0, s>>>(a, w.select);
            launched("price_best_score_kernel");
            price_best_index_kernel<<<g, kPT, 0, s>>>(a, w.select);
            launched("price_best_index_kernel");
            price_round_close_kernel<<<1, 32, 0, s>>>(w.select, out, r);
            launched("price_round_close_kernel");
        }
    });
}

int hn_price_columns(const hn_csr* A, int64_t k, const int64_t* cols, double* out, void* stream) {
    return guard("hn_price_columns", [&] {
        require_init();
        if (!A || k < 0 || (k > 0 && (!cols || !out))) fail(HN_ERR_INVALID_ARG, "bad arguments");
        if (!A->has_t) fail(HN_ERR_INVALID_ARG, "matrix was created without its transpose");
        if (k == 0) return;
        cudaStream_t s = as_stream(stream);
        Workspace& w = workspace(s);
        check_cuda(cudaMemsetAsync(out, 0, sizeof(double) * (size_t)A->m * (size_t)k, s), "memset columns");
        check_cuda(cudaMemsetAsync(w.select + W_COUNT, 0, sizeof(unsigned long long), s), "memset flag");
        column_gather_kernel<<<(unsigned)k, kPT, 0, s>>>(A->m, A->n, A->rpT, A->ciT, A->valT, cols, out,
                                                         w.select + W_COUNT);
        launched("column_gather_kernel");
        unsigned long long bad = 0;
        check_cuda(cudaMemcpyAsync(&bad, w.select + W_COUNT, sizeof(bad), cudaMemcpyDeviceToHost, s), "D2H flag");
        check_cuda(cudaStreamSynchronize(s), "column gather sync");
        if (bad) fail(HN_ERR_INVALID_ARG, "column index out of range");
    });
}

}  // extern "C"
