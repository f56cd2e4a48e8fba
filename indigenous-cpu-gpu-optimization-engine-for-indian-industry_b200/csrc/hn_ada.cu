// Normal-equation assembly N = A diag(d) A^T + dyn_reg I
// (build_normal_equations, core/lp/interior_point.cpp:144-200).
//
// Symbolic (once per A): one CTA per row i marks, in a shared-memory bitmap
// of m bits, every k reachable through a nonzero A_ij (the rows of column j,
// read from the device A^T) plus k = i; a popcount gives the row length, a
// second pass writes the column indices in ascending order by scanning the
// bitmap. Integer work only: the pattern is exact.
//
// Numeric (every IPM iteration): one warp per row of N, taking the row in
// slices of kSlice pattern positions held in shared memory (keys + FP64
// accumulators). For each nonzero A_ij in row order, with d_j > 0, the warp
// binary-searches the part of column j inside the slice's key range and adds
// (A_ij * A_kj) * d_j to the slot of k (lanes touch distinct k, so no atomics;
// the j loop is sequential so each entry sums in column order -- the
// reference's order for the diagonal). The slice is then stored coalesced.
// HBM traffic is the N write (12 B per entry incl. the key read); column
// reads of A^T hit L2.
#include <algorithm>
#include <vector>

#include "hn_internal.cuh"

namespace hn {
namespace {

constexpr int kSymThreads = 256;
constexpr int kMaxBitmapWords = 50000;  // m <= 1.6M rows (200 KB of shared memory)
constexpr int kSlice = 512;
constexpr int kNumWarps = 8;

__device__ __forceinline__ void mark_row(int i, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                                         const double* __restrict__ val, const int32_t* __restrict__ rpT,
                                         const int32_t* __restrict__ ciT, uint32_t* bm) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) atomicOr(&bm[i >> 5], 1u << (i & 31));
    for (int e = rp[i] + warp; e < rp[i + 1]; e += kSymThreads / 32) {
        if (val[e] == 0.0) continue;
        const int j = ci[e];
        for (int p = rpT[j] + lane; p < rpT[j + 1]; p += 32) {
            const int k = ciT[p];
            atomicOr(&bm[k >> 5], 1u << (k & 31));
        }
    }
}

__global__ void __launch_bounds__(kSymThreads) ada_count_kernel(int m, const int32_t* __restrict__ rp,
                                                                const int32_t* __restrict__ ci,
                                                                const double* __restrict__ val,
                                                                const int32_t* __restrict__ rpT,
                                                                const int32_t* __restrict__ ciT, int W,
                                                                int64_t* __restrict__ counts) {
    extern __shared__ uint32_t bm[];
    __shared__ int64_t sh[32];
    for (int i = blockIdx.x; i < m; i += gridDim.x) {
        for (int w = threadIdx.x; w < W; w += kSymThreads) bm[w] = 0u;
        __syncthreads();
        mark_row(i, rp, ci, val, rpT, ciT, bm);
        __syncthreads();
        int64_t c = 0;
        for (int w = threadIdx.x; w < W; w += kSymThreads) c += __popc(bm[w]);
        c = block_sum_i64<kSymThreads>(c, sh);
        if (threadIdx.x == 0) counts[i] = c;
        __syncthreads();
    }
}

__global__ void __launch_bounds__(kSymThreads) ada_fill_kernel(int m, const int32_t* __restrict__ rp,
                                                               const int32_t* __restrict__ ci,
                                                               const double* __restrict__ val,
                                                               const int32_t* __restrict__ rpT,
                                                               const int32_t* __restrict__ ciT, int W,
                                                               const int64_t* __restrict__ rpN,
                                                               int32_t* __restrict__ ciN,
                                                               int64_t* __restrict__ diag_pos) {
    extern __shared__ uint32_t bm[];
    __shared__ int64_t sh[32];
    const int wpt = (W + kSymThreads - 1) / kSymThreads;
    for (int i = blockIdx.x; i < m; i += gridDim.x) {
        for (int w = threadIdx.x; w < W; w += kSymThreads) bm[w] = 0u;
        __syncthreads();
        mark_row(i, rp, ci, val, rpT, ciT, bm);
        __syncthreads();
        const int w0 = threadIdx.x * wpt;
        const int w1 = min(W, w0 + wpt);
        int64_t c = 0;
        for (int w = w0; w < w1; ++w) c += __popc(bm[w]);
        int64_t total;
        int64_t off = rpN[i] + block_exclusive_scan_i64<kSymThreads>(c, sh, &total);
        for (int w = w0; w < w1; ++w) {
            uint32_t bits = bm[w];
            while (bits) {
                const int b = __ffs(bits) - 1;
                const int k = w * 32 + b;
                if (k == i) diag_pos[i] = off;
                ciN[off++] = k;
                bits &= bits - 1;
            }
        }
        __syncthreads();
    }
}

__global__ void __launch_bounds__(kNumWarps * 32) ada_numeric_kernel(
    int m, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci, const double* __restrict__ val,
    const int32_t* __restrict__ rpT, const int32_t* __restrict__ ciT, const double* __restrict__ valT,
    const double* __restrict__ d, const int64_t* __restrict__ rpN, const int32_t* __restrict__ ciN,
    const int64_t* __restrict__ diag_pos, double* __restrict__ nval, unsigned long long* maxdiag) {
    __shared__ int32_t s_key_all[kNumWarps][kSlice];
    __shared__ double s_acc_all[kNumWarps][kSlice];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int32_t* s_key = s_key_all[warp];
    double* s_acc = s_acc_all[warp];
    const int64_t gw = blockIdx.x * (int64_t)kNumWarps + warp;
    const int64_t nw = (int64_t)gridDim.x * kNumWarps;
    for (int64_t i = gw; i < m; i += nw) {
        const int64_t pe0 = rpN[i + 1];
        const int e_beg = rp[i], e_end = rp[i + 1];
        for (int64_t ps = rpN[i]; ps < pe0; ps += kSlice) {
            const int len = (int)min((int64_t)kSlice, pe0 - ps);
            for (int q = lane; q < len; q += 32) {
                s_key[q] = ciN[ps + q];
                s_acc[q] = 0.0;
            }
            __syncwarp();
            const int klo = s_key[0], khi = s_key[len - 1];
            for (int e0 = e_beg; e0 < e_end; e0 += 32) {
                const int e = e0 + lane;
                int my_j = 0;
                double my_a = 0.0, my_d = 0.0;
                if (e < e_end) {
                    my_j = ci[e];
                    my_a = val[e];
                    my_d = d[my_j];
                }
                const int cnt = min(32, e_end - e0);
                for (int u = 0; u < cnt; ++u) {
                    const int j = __shfl_sync(0xffffffffu, my_j, u);
                    const double a = __shfl_sync(0xffffffffu, my_a, u);
                    const double dj = __shfl_sync(0xffffffffu, my_d, u);
                    if (dj <= 0.0 || a == 0.0) continue;
                    int cs = rpT[j];
                    const int ce = rpT[j + 1];
                    if (ce - cs > 32) {
                        int lo = cs, hi = ce;
                        while (lo < hi) {
                            const int mid = (lo + hi) >> 1;
                            if (__ldg(ciT + mid) < klo)
                                lo = mid + 1;
                            else
                                hi = mid;
                        }
                        cs = lo;
                    }
                    for (int p = cs + lane; p < ce; p += 32) {
                        const int k = __ldg(ciT + p);
                        if (k > khi) break;
                        if (k < klo) continue;
                        int lo = 0, hi = len - 1;
                        while (lo < hi) {
                            const int mid = (lo + hi) >> 1;
                            if (s_key[mid] < k)
                                lo = mid + 1;
                            else
                                hi = mid;
                        }
                        if (s_key[lo] == k) s_acc[lo] += (a * __ldg(valT + p)) * dj;
                    }
                    __syncwarp();
                }
            }
            __syncwarp();
            for (int q = lane; q < len; q += 32) nval[ps + q] = s_acc[q];
            if (lane == 0 && klo <= i && i <= khi) {
                const double v = s_acc[diag_pos[i] - ps];
                if (v > 0.0) atomicMax(maxdiag, static_cast<unsigned long long>(__double_as_longlong(v)));
            }
            __syncwarp();
        }
    }
}

__global__ void ada_reg_kernel(int m, const int64_t* __restrict__ diag_pos, double reg,
                               const unsigned long long* __restrict__ maxdiag, double* __restrict__ nval,
                               double* dyn_out) {
    const double md = __longlong_as_double(static_cast<long long>(*maxdiag));
    double dyn = 1e-12 * md;
    dyn = (reg < dyn) ? dyn : reg;  // std::max(regularization, 1e-12 * max_diag)
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < m) nval[diag_pos[i]] += dyn;
    if (i == 0 && dyn_out) *dyn_out = dyn;
}

void free_pattern(hn_pattern* P) {
    if (!P) return;
    dfree(P->rp);
    dfree(P->ci);
    dfree(P->diag_pos);
    dfree(P->maxdiag);
    delete P;
}

}  // namespace
}  // namespace hn

using namespace hn;

extern "C" {

int hn_ada_symbolic(const hn_csr* A, hn_pattern** out) {
    return guard("hn_ada_symbolic", [&] {
        require_init();
        if (!A || !out) fail(HN_ERR_INVALID_ARG, "bad arguments");
        if (!A->has_t) fail(HN_ERR_INVALID_ARG, "hn_ada_symbolic needs a handle with A^T");
        *out = nullptr;
        const int64_t m = A->m;
        const int64_t W = (m + 31) / 32;
        if (W > kMaxBitmapWords)
            fail(HN_ERR_UNSUPPORTED, "m = " + std::to_string(m) + " exceeds the 1.6M-row bitmap limit");
        hn_pattern* P = new hn_pattern();
        cudaStream_t s = nullptr;
        try {
            P->m = m;
            P->A = A;
            P->rp = dmalloc<int64_t>(m + 1);
            P->diag_pos = dmalloc<int64_t>(m);
            P->maxdiag = dmalloc<unsigned long long>(1);
            check_cuda(cudaMemsetAsync(P->rp, 0, sizeof(int64_t) * (m + 1), s), "memset rp");
            const size_t smem = sizeof(uint32_t) * (size_t)(W > 0 ? W : 1);
            check_cuda(cudaFuncSetAttribute(ada_count_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)smem),
                       "smem attribute");
            check_cuda(cudaFuncSetAttribute(ada_fill_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)smem),
                       "smem attribute");
            const int grid = (int)std::min<int64_t>(std::max<int64_t>(m, 1), (int64_t)ctx().sm_count * 8);
            if (m > 0) {
                ada_count_kernel<<<grid, kSymThreads, smem, s>>>((int)m, A->rp, A->ci, A->val, A->rpT, A->ciT,
                                                                 (int)W, P->rp);
                launched("ada_count_kernel");
            }
            scan_exclusive_i64(P->rp, P->rp, m + 1, s);
            check_cuda(cudaMemcpyAsync(&P->nnz, P->rp + m, sizeof(int64_t), cudaMemcpyDeviceToHost, s),
                       "D2H nnz");
            check_cuda(cudaStreamSynchronize(s), "symbolic sync");
            P->ci = dmalloc<int32_t>(P->nnz);
            if (m > 0) {
                ada_fill_kernel<<<grid, kSymThreads, smem, s>>>((int)m, A->rp, A->ci, A->val, A->rpT, A->ciT,
                                                                (int)W, P->rp, P->ci, P->diag_pos);
                launched("ada_fill_kernel");
            }
            check_cuda(cudaStreamSynchronize(s), "symbolic sync");
        } catch (...) {
            free_pattern(P);
            throw;
        }
        *out = P;
    });
}

int hn_pattern_info(const hn_pattern* P, int64_t* m, int64_t* nnz) {
    return guard("hn_pattern_info", [&] {
        if (!P) fail(HN_ERR_INVALID_ARG, "null pattern");
        if (m) *m = P->m;
        if (nnz) *nnz = P->nnz;
    });
}

int hn_pattern_export(const hn_pattern* P, uint64_t* rp, uint64_t* ci) {
    return guard("hn_pattern_export", [&] {
        require_init();
        if (!P) fail(HN_ERR_INVALID_ARG, "null pattern");
        std::vector<int64_t> r(P->m + 1);
        std::vector<int32_t> c(P->nnz);
        check_cuda(cudaMemcpy(r.data(), P->rp, sizeof(int64_t) * (P->m + 1), cudaMemcpyDeviceToHost), "D2H");
        if (P->nnz > 0)
            check_cuda(cudaMemcpy(c.data(), P->ci, sizeof(int32_t) * P->nnz, cudaMemcpyDeviceToHost), "D2H");
        if (rp)
            for (int64_t i = 0; i <= P->m; ++i) rp[i] = (uint64_t)r[i];
        if (ci)
            for (int64_t k = 0; k < P->nnz; ++k) ci[k] = (uint64_t)c[k];
    });
}

int hn_pattern_device(const hn_pattern* P, const int64_t** rp, const int32_t** ci, const int64_t** dp) {
    return guard("hn_pattern_device", [&] {
        if (!P) fail(HN_ERR_INVALID_ARG, "null pattern");
        if (rp) *rp = P->rp;
        if (ci) *ci = P->ci;
        if (dp) *dp = P->diag_pos;
    });
}

int hn_ada_numeric(const hn_pattern* P, const double* d, double reg, double* nval, double* dyn_out,
                   void* stream) {
    return guard("hn_ada_numeric", [&] {
        require_init();
        if (!P || !d || (P->nnz > 0 && !nval)) fail(HN_ERR_INVALID_ARG, "bad arguments");
        const hn_csr* A = P->A;
        cudaStream_t s = as_stream(stream);
        if (P->m == 0) return;
        check_cuda(cudaMemsetAsync(P->maxdiag, 0, sizeof(unsigned long long), s), "memset maxdiag");
        const int grid = (int)std::min<int64_t>((P->m + kNumWarps - 1) / kNumWarps, (int64_t)ctx().sm_count * 4);
        ada_numeric_kernel<<<grid, kNumWarps * 32, 0, s>>>((int)P->m, A->rp, A->ci, A->val, A->rpT, A->ciT,
                                                           A->valT, d, P->rp, P->ci, P->diag_pos, nval,
                                                           P->maxdiag);
        launched("ada_numeric_kernel");
        ada_reg_kernel<<<(unsigned)((P->m + 255) / 256), 256, 0, s>>>((int)P->m, P->diag_pos, reg, P->maxdiag,
                                                                      nval, dyn_out);
        launched("ada_reg_kernel");
    });
}

int hn_pattern_destroy(hn_pattern* P) {
    return guard("hn_pattern_destroy", [&] {
        if (!P) return;
        require_init();
        cudaDeviceSynchronize();
        free_pattern(P);
    });
}

}  // extern "C"
