// Merge-path FP64 CSR SpMV with a fused per-row epilogue.
//
// The merge path is the interleaving of the m row ends (rp[1..m]) with the
// nnz nonzero indices; it is cut into tiles of kSpmvTile items so every CTA
// does the same amount of work whatever the row-length distribution (the
// Zipf-skewed A^T rows of the large configuration and the Poisson rows of A
// alike). Inside a tile each thread walks kSpmvIpt consecutive items.
//
// Per tile: the row ends go to shared memory; each thread finds where the
// path enters and leaves its items (two binary searches), loads the products
// of its contiguous nonzeros straight into registers (col_idx, values, then
// the x gathers -- through L1, so a warp's neighbouring ranges share sectors),
// and walks its items, finishing rows that end in its range; partial rows are
// combined through a shared carry array in thread order. A row that
// began in an earlier tile leaves its in-tile part in head_val and is
// finished by a second, tiny kernel that adds the earlier tiles' carries in
// tile order. Every row's sum therefore has a fixed association order, so
// results are deterministic run to run.
//
// Epilogues receive (row, sum) exactly once per row and write the outputs
// (y = alpha*s + beta*y, residuals, IPM directions ...).
#pragma once

#include "hn_internal.cuh"

namespace hn {

constexpr int kSpmvThreads = 256;
constexpr int kSpmvIpt = 7;
constexpr int kSpmvTile = kSpmvThreads * kSpmvIpt;

struct SpmvMat {
    int m, nnz;
    const int32_t* rp;
    const int32_t* ci;
    const double* val;
    const int32_t* tile_row;
    const int32_t* tile_nz;
    int32_t* carry_row;
    double* carry_val;
    int32_t* head_row;
    double* head_val;
    int64_t ntiles;
    int kind = 0;  // 0: merge path; 1: binned vector CSR
    const int32_t* perm = nullptr;
    SpmvBins bins = {};
};

inline SpmvMat spmv_mat(const hn_csr* A, int trans) {
    SpmvMat M;
    if (!trans) {
        M = SpmvMat{(int)A->m, (int)A->nnz, A->rp, A->ci, A->val, A->tile_row, A->tile_nz,
                    A->carry_row, A->carry_val, A->head_row, A->head_val, A->ntiles};
    } else {
        M = SpmvMat{(int)A->n, (int)A->nnz_t, A->rpT, A->ciT, A->valT, A->tile_row_t, A->tile_nz_t,
                    A->carry_row_t, A->carry_val_t, A->head_row_t, A->head_val_t, A->ntiles_t};
    }
    const int d = trans ? 1 : 0;
    if (A->spmv_kind[d] == 1 && A->perm[d]) {
        M.kind = 1;
        M.perm = A->perm[d];
        M.bins = A->bins[d];
    }
    return M;
}

// Merge-path coordinate of tile-local diagonal `diag`: rows consumed (return)
// and nonzeros consumed (diag - return), from the tile's row ends in shared memory.
__device__ __forceinline__ int tile_search(const int32_t* s_rowend, int k0, int diag, int nrows_t, int nnz_t) {
    int lo = diag - nnz_t > 0 ? diag - nnz_t : 0;
    int hi = diag < nrows_t ? diag : nrows_t;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (s_rowend[mid] <= k0 + diag - mid - 1)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

template <class Epi>
__global__ void __launch_bounds__(kSpmvThreads) spmv_tile_kernel(SpmvMat a, const double* __restrict__ x,
                                                                 Epi epi) {
    __shared__ int32_t s_rowend[kSpmvTile + 1];
    __shared__ int32_t s_crow[kSpmvThreads];
    __shared__ double s_cval[kSpmvThreads];
    __shared__ int32_t s_rowstart0;

    const int tid = threadIdx.x;
    const int tile = blockIdx.x;
    const int r0 = a.tile_row[tile], k0 = a.tile_nz[tile];
    const int r1 = a.tile_row[tile + 1], k1 = a.tile_nz[tile + 1];
    const int nrows_t = r1 - r0;
    const int nnz_t = k1 - k0;

    if (tid == 0) {
        s_rowstart0 = (r0 < a.m) ? a.rp[r0] : a.nnz;
        a.head_row[tile] = -1;
    }
    for (int i = tid; i <= nrows_t; i += kSpmvThreads) {
        const int r = r0 + i;
        s_rowend[i] = (r < a.m) ? __ldg(a.rp + r + 1) : INT_MAX;
    }
    __syncthreads();

    // this thread's kSpmvIpt merge items: its nonzeros are the contiguous
    // range [nz, nz_e) of the tile, found from the path at both ends
    const int total_t = nrows_t + nnz_t;
    const int diag = min(tid * kSpmvIpt, total_t);
    const int diag_end = min(diag + kSpmvIpt, total_t);
    int row = tile_search(s_rowend, k0, diag, nrows_t, nnz_t);
    int nz = diag - row;
    const int row_e = tile_search(s_rowend, k0, diag_end, nrows_t, nnz_t);
    const int cnt = (diag_end - row_e) - nz;

    // products of those nonzeros, straight into registers (no shared buffer):
    // column indices first, then values, then the gathers of x
    double v[kSpmvIpt];
    {
        int c[kSpmvIpt];
#pragma unroll
        for (int u = 0; u < kSpmvIpt; ++u) c[u] = (u < cnt) ? __ldg(a.ci + k0 + nz + u) : 0;
        double w[kSpmvIpt];
#pragma unroll
        for (int u = 0; u < kSpmvIpt; ++u) w[u] = (u < cnt) ? __ldg(a.val + k0 + nz + u) : 0.0;
#pragma unroll
        for (int u = 0; u < kSpmvIpt; ++u) v[u] = (u < cnt) ? w[u] * __ldcg(x + c[u]) : 0.0;
    }

    double sum = 0.0;
    int first_row = -1;
    double first_val = 0.0;
#pragma unroll
    for (int it = 0; it < kSpmvIpt; ++it) {
        if (diag + it < diag_end) {
            const bool take_nz = (nz < nnz_t) && (k0 + nz < s_rowend[row]);
            if (take_nz) {
                sum += v[0];
#pragma unroll
                for (int q = 0; q < kSpmvIpt - 1; ++q) v[q] = v[q + 1];
                ++nz;
            } else if (row < nrows_t) {
                if (first_row < 0) {
                    first_row = row;
                    first_val = sum;
                } else {
                    epi(r0 + row, sum);
                }
                sum = 0.0;
                ++row;
            }
        }
    }
    s_crow[tid] = row;
    s_cval[tid] = sum;
    __syncthreads();

    if (first_row >= 0) {
        int t = tid - 1;
        while (t >= 0 && s_crow[t] == first_row) --t;
        double acc = 0.0;
        for (int u = t + 1; u < tid; ++u) acc += s_cval[u];
        acc += first_val;
        if (t < 0 && first_row == 0 && k0 > s_rowstart0) {
            a.head_row[tile] = r0;
            a.head_val[tile] = acc;
        } else {
            epi(r0 + first_row, acc);
        }
    }
    if (tid == kSpmvThreads - 1) {
        const int crow = s_crow[tid];
        if (r0 + crow < a.m) {
            int t = tid;
            while (t >= 0 && s_crow[t] == crow) --t;
            double acc = 0.0;
            for (int u = t + 1; u <= tid; ++u) acc += s_cval[u];
            a.carry_row[tile] = r0 + crow;
            a.carry_val[tile] = acc;
        } else {
            a.carry_row[tile] = -1;
        }
    }
}

template <class Epi>
__global__ void spmv_fixup_kernel(SpmvMat a, Epi epi) {
    const int64_t tile = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (tile >= a.ntiles) return;
    const int r = a.head_row[tile];
    if (r < 0) return;
    int64_t s = tile - 1;
    while (s >= 0 && a.carry_row[s] == r) --s;
    double acc = 0.0;
    for (int64_t u = s + 1; u < tile; ++u) acc += a.carry_val[u];
    acc += a.head_val[tile];
    epi(r, acc);
}

// ---- binned vector CSR ----
// A group of G lanes sums one row: lane l takes the row's nonzeros l, l + G,
// ... in order (kVecUnroll loads in flight), then the group combines its
// lanes by a fixed shuffle tree; every row's association order is fixed, so
// results are deterministic. Rows are grouped by G (bins); one launch covers
// all bins.
constexpr int kVecUnroll = 4;

template <int G, class Epi>
__device__ __forceinline__ void vec_rows(const SpmvMat& a, int bin, int unit, const double* __restrict__ x,
                                         const Epi& epi) {
    const int lane = threadIdx.x & 31, sub = lane / G, l = lane % G;
    const int idx = a.bins.row_off[bin] + unit * (32 / G) + sub;
    const bool valid = idx < a.bins.row_off[bin + 1];
    const int r = valid ? a.perm[idx] : 0;
    const int k0 = valid ? __ldg(a.rp + r) : 0, k1 = valid ? __ldg(a.rp + r + 1) : 0;
    double sum = 0.0;
    for (int k = k0 + l; k < k1; k += kVecUnroll * G) {
        int c[kVecUnroll];
        double w[kVecUnroll];
#pragma unroll
        for (int u = 0; u < kVecUnroll; ++u) {
            const int kk = k + u * G;
            c[u] = kk < k1 ? __ldg(a.ci + kk) : 0;
            w[u] = kk < k1 ? __ldg(a.val + kk) : 0.0;
        }
        double p[kVecUnroll];
#pragma unroll
        for (int u = 0; u < kVecUnroll; ++u) p[u] = (k + u * G < k1) ? w[u] * __ldcg(x + c[u]) : 0.0;
#pragma unroll
        for (int u = 0; u < kVecUnroll; ++u)
            if (k + u * G < k1) sum += p[u];
    }
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) sum += __shfl_down_sync(0xffffffffu, sum, o, G);
    if (valid && l == 0) epi(r, sum);
}

template <class Epi>
__global__ void __launch_bounds__(kSpmvThreads) spmv_vec_kernel(SpmvMat a, const double* __restrict__ x, Epi epi) {
    const int w = (int)((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5);
    if (w >= a.bins.unit_off[a.bins.nbins]) return;  // whole warps leave together
    int bin = 0;
    while (w >= a.bins.unit_off[bin + 1]) ++bin;
    const int unit = w - a.bins.unit_off[bin];
    switch (a.bins.lg[bin]) {
        case 0: vec_rows<1>(a, bin, unit, x, epi); break;
        case 1: vec_rows<2>(a, bin, unit, x, epi); break;
        case 2: vec_rows<4>(a, bin, unit, x, epi); break;
        case 3: vec_rows<8>(a, bin, unit, x, epi); break;
        case 4: vec_rows<16>(a, bin, unit, x, epi); break;
        default: vec_rows<32>(a, bin, unit, x, epi); break;
    }
}

// Launches one product on `s`: the binned vector kernel, or the merge-path
// tile kernel and its fix-up.
template <class Epi>
void spmv_launch(const SpmvMat& M, const double* x, const Epi& epi, cudaStream_t s) {
    if (M.kind == 1) {
        const int64_t units = M.bins.unit_off[M.bins.nbins];
        if (units == 0) return;
        spmv_vec_kernel<Epi><<<(unsigned)((units * 32 + kSpmvThreads - 1) / kSpmvThreads), kSpmvThreads, 0, s>>>(
            M, x, epi);
        launched("spmv_vec_kernel");
        return;
    }
    if (M.ntiles == 0) return;
    spmv_tile_kernel<Epi><<<(unsigned)M.ntiles, kSpmvThreads, 0, s>>>(M, x, epi);
    launched("spmv_tile_kernel");
    if (M.ntiles > 1) {
        spmv_fixup_kernel<Epi><<<(unsigned)((M.ntiles + 255) / 256), 256, 0, s>>>(M, epi);
        launched("spmv_fixup_kernel");
    }
}

// ---- epilogues ----
struct EpiAxpby {
    double alpha, beta;
    double* y;
    __device__ __forceinline__ void operator()(int r, double s) const {
        y[r] = (beta == 0.0) ? alpha * s : alpha * s + beta * y[r];
    }
};

// y = s - b (a residual op(A) x - b in one pass)
struct EpiSub {
    const double* b;
    double* y;
    __device__ __forceinline__ void operator()(int r, double s) const { y[r] = s - b[r]; }
};

// IPM epilogues (core/lp/interior_point.cpp line numbers in hn_ipm.cu)
struct EpiResidual {
    const double* b;
    double* mx;
    double* rp;
    __device__ __forceinline__ void operator()(int r, double s) const {
        mx[r] = s;
        rp[r] = s - b[r];
    }
};

struct EpiDualResidual {
    const double* z;
    const double* c;
    double* rd;
    __device__ __forceinline__ void operator()(int j, double s) const { rd[j] = (s + z[j]) - c[j]; }
};

struct EpiRhs {
    const double* rp;
    const double* mx;
    double* rhs;
    __device__ __forceinline__ void operator()(int i, double s) const { rhs[i] = ((-rp[i]) - s) + mx[i]; }
};

struct EpiCorrRhs {
    const double* pred;
    double* rhs;
    __device__ __forceinline__ void operator()(int i, double s) const { rhs[i] = pred[i] - s; }
};

struct EpiDirection {
    const double* D;
    const double* rd;
    const double* x;
    const double* corr;
    double* dx;
    double* dz;
    __device__ __forceinline__ void operator()(int j, double s) const {
        const double u = s + rd[j];
        double v = D[j] * u - x[j];
        if (corr) v = v + corr[j];
        dx[j] = v;
        dz[j] = -u;
    }
};

}  // namespace hn
