// Normal-equation assembly N = A diag(d) A^T + dyn_reg I
// (build_normal_equations, core/lp/interior_point.cpp:144-200).
//
// A "contribution" is one term (A_ij * A_kj) * d_j: row i of N, entry e of
// row i of A (column j), row k of column j. Contributions are numbered q in
// a fixed structural order -- rows i ascending, entries e of row i in CSR
// order, then the rows k of column j (A^T row j) ascending.
//
// Symbolic (once per A; integer work only, exact):
//   one CTA per row i builds two shared-memory bitmaps over the m columns of
//   N: b1 = k reached at least once (plus k = i), b2 = k reached twice or more
//   (plus k = i). popcounts give the row length, the number of contributions,
//   of "multi" slots (b2) and of contributions into multi slots; after scans,
//   a second pass writes the sorted pattern (scanning b1), the table of multi
//   slots, and the scatter map: map[q] = the N position of a slot reached
//   once, or kMulti | the scratch index of the contribution inside its multi
//   slot's range, numbered in q order.
// Numeric (every IPM iteration), three kernels, all streaming:
//   stage  : one CTA per row; every contribution of the row is computed in
//            parallel and stored once -- into a shared-memory copy of the row
//            (then written out coalesced) or, for a multi slot, into scratch.
//            Single-contribution slots (~98% of N for random LPs) need no
//            accumulation, no search and no atomics.
//   combine: one thread per multi slot sums its scratch range in q order --
//            column order, the order the reference accumulates the diagonal
//            (:188-191) -- and takes the max diagonal.
//   reg    : N_ii += dyn_reg = max(reg, 1e-12 * max diag) (:193-196).
// HBM traffic per numeric call: the 4-byte map entry per contribution, the
// 8-byte N value per entry, plus the small multi-slot tables.
#include <algorithm>
#include <vector>

#include "hn_internal.cuh"

namespace hn {
namespace {

constexpr int kT = 256;
constexpr int64_t kMaxBitmapWords = 12500;  // m <= 400,000: four W-word arrays in 200 KB of shared memory
constexpr uint32_t kMulti = 0x80000000u;
constexpr int64_t kDiagFlag = int64_t(1) << 62;
constexpr int kEntryChunk = 512;  // row entries of A staged per pass of the numeric kernel
constexpr int kStage = 6144;      // N row slots staged in shared memory (longer rows write directly)
constexpr int kUnroll = 8;        // contributions per thread per trip of the numeric kernel

__device__ __forceinline__ uint32_t bit_of(int k) { return 1u << (k & 31); }

// Marks every contribution of row i: b1 |= bit(k); if it was set already, b2 |= bit(k).
__device__ __forceinline__ void mark_contributions(int i, const int32_t* __restrict__ rp,
                                                   const int32_t* __restrict__ ci, const double* __restrict__ val,
                                                   const int32_t* __restrict__ rpT, const int32_t* __restrict__ ciT,
                                                   uint32_t* b1, uint32_t* b2, int64_t* nq_local) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) {
        atomicOr(&b1[i >> 5], bit_of(i));
        atomicOr(&b2[i >> 5], bit_of(i));  // the diagonal is always a multi slot (it gets dyn_reg)
    }
    int64_t cnt = 0;
    for (int e = rp[i] + warp; e < rp[i + 1]; e += kT / 32) {
        if (val[e] == 0.0) continue;
        const int j = ci[e];
        for (int p = rpT[j] + lane; p < rpT[j + 1]; p += 32) {
            const int k = ciT[p];
            const uint32_t old = atomicOr(&b1[k >> 5], bit_of(k));
            if (old & bit_of(k)) atomicOr(&b2[k >> 5], bit_of(k));
            ++cnt;
        }
    }
    *nq_local = cnt;
}

__global__ void __launch_bounds__(kT) ada_count_kernel(int m, const int32_t* __restrict__ rp,
                                                       const int32_t* __restrict__ ci,
                                                       const double* __restrict__ val,
                                                       const int32_t* __restrict__ rpT,
                                                       const int32_t* __restrict__ ciT, int W,
                                                       int64_t* __restrict__ len, int64_t* __restrict__ nq,
                                                       int64_t* __restrict__ nms, int64_t* __restrict__ nmq) {
    extern __shared__ uint32_t smem[];
    uint32_t* b1 = smem;
    uint32_t* b2 = smem + W;
    __shared__ int64_t sh[32];
    for (int i = blockIdx.x; i < m; i += gridDim.x) {
        for (int w = threadIdx.x; w < W; w += kT) {
            b1[w] = 0u;
            b2[w] = 0u;
        }
        __syncthreads();
        int64_t q;
        mark_contributions(i, rp, ci, val, rpT, ciT, b1, b2, &q);
        __syncthreads();
        int64_t L = 0, MS = 0, D1 = 0;
        for (int w = threadIdx.x; w < W; w += kT) {
            L += __popc(b1[w]);
            MS += __popc(b2[w]);
            D1 += __popc(b1[w] & ~b2[w]);
        }
        L = block_sum_i64<kT>(L, sh);
        MS = block_sum_i64<kT>(MS, sh);
        D1 = block_sum_i64<kT>(D1, sh);
        q = block_sum_i64<kT>(q, sh);
        if (threadIdx.x == 0) {
            len[i] = L;
            nq[i] = q;
            nms[i] = MS;
            nmq[i] = q - D1;
        }
        __syncthreads();
    }
}

__device__ __forceinline__ int rank_of(const uint32_t* b, const int32_t* pre, int k) {
    return pre[k >> 5] + __popc(b[k >> 5] & (bit_of(k) - 1u));
}

__global__ void __launch_bounds__(kT) ada_fill_kernel(
    int m, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci, const double* __restrict__ val,
    const int32_t* __restrict__ rpT, const int32_t* __restrict__ ciT, int W, const int64_t* __restrict__ rpN,
    const int64_t* __restrict__ qrow, const int64_t* __restrict__ msrow, const int64_t* __restrict__ mqrow,
    int32_t* __restrict__ ciN, int64_t* __restrict__ diag_pos, int64_t* __restrict__ mpos, int32_t* mcnt,
    int32_t* __restrict__ mbeg, uint32_t* __restrict__ map) {
    extern __shared__ uint32_t smem[];
    uint32_t* b1 = smem;
    uint32_t* b2 = smem + W;
    int32_t* pre1 = reinterpret_cast<int32_t*>(smem + 2 * W);
    int32_t* pre2 = reinterpret_cast<int32_t*>(smem + 3 * W);
    __shared__ int64_t sh[32];
    const int wpt = (W + kT - 1) / kT;
    for (int i = blockIdx.x; i < m; i += gridDim.x) {
        for (int w = threadIdx.x; w < W; w += kT) {
            b1[w] = 0u;
            b2[w] = 0u;
        }
        __syncthreads();
        int64_t unused;
        mark_contributions(i, rp, ci, val, rpT, ciT, b1, b2, &unused);
        __syncthreads();
        // word prefix popcounts; pattern, diagonal position and the multi-slot table
        const int w0 = min(W, threadIdx.x * wpt);
        const int w1 = min(W, w0 + wpt);
        int64_t c1 = 0, c2 = 0;
        for (int w = w0; w < w1; ++w) {
            c1 += __popc(b1[w]);
            c2 += __popc(b2[w]);
        }
        int64_t t1, t2;
        int64_t o1 = block_exclusive_scan_i64<kT>(c1, sh, &t1);
        int64_t o2 = block_exclusive_scan_i64<kT>(c2, sh, &t2);
        const int64_t row0 = rpN[i], ms0 = msrow[i];
        for (int w = w0; w < w1; ++w) {
            pre1[w] = static_cast<int32_t>(o1);
            pre2[w] = static_cast<int32_t>(o2);
            uint32_t bits = b1[w];
            const uint32_t bits2 = b2[w];
            while (bits) {
                const int b = __ffs(bits) - 1;
                const int k = w * 32 + b;
                const int64_t pos = row0 + o1;
                ciN[pos] = k;
                if (k == i) diag_pos[i] = pos;
                if ((bits2 >> b) & 1u) {
                    mpos[ms0 + o2] = pos | (k == i ? kDiagFlag : 0);
                    mcnt[ms0 + o2] = 0;
                    ++o2;
                }
                ++o1;
                bits &= bits - 1;
            }
        }
        __syncthreads();
        // contributions per multi slot
        {
            const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
            for (int e = rp[i] + warp; e < rp[i + 1]; e += kT / 32) {
                if (val[e] == 0.0) continue;
                const int j = ci[e];
                for (int p = rpT[j] + lane; p < rpT[j + 1]; p += 32) {
                    const int k = ciT[p];
                    if (b2[k >> 5] & bit_of(k)) atomicAdd(&mcnt[ms0 + rank_of(b2, pre2, k)], 1);
                }
            }
        }
        __syncthreads();
        // scratch ranges of this row's multi slots (then mcnt becomes a cursor)
        {
            const int64_t MS = msrow[i + 1] - ms0;
            int64_t carry = mqrow[i];
            for (int64_t t0 = 0; t0 < MS; t0 += kT) {
                const int64_t t = t0 + threadIdx.x;
                const int64_t v = t < MS ? mcnt[ms0 + t] : 0;
                int64_t tot;
                const int64_t ex = block_exclusive_scan_i64<kT>(v, sh, &tot);
                if (t < MS) {
                    mbeg[ms0 + t] = static_cast<int32_t>(carry + ex);
                    mcnt[ms0 + t] = 0;
                }
                carry += tot;
            }
        }
        __syncthreads();
        // scatter map in contribution order; entries e go one after the other so
        // the ordinals inside each multi slot follow the column order
        int64_t q = qrow[i];
        for (int e = rp[i]; e < rp[i + 1]; ++e) {
            if (val[e] == 0.0) continue;
            const int j = ci[e];
            const int cs = rpT[j], ce = rpT[j + 1];
            for (int p = cs + threadIdx.x; p < ce; p += kT) {
                const int k = ciT[p];
                const int64_t qq = q + (p - cs);
                if (b2[k >> 5] & bit_of(k)) {
                    const int64_t ms = ms0 + rank_of(b2, pre2, k);
                    const int ord = atomicAdd(&mcnt[ms], 1);
                    map[qq] = kMulti | static_cast<uint32_t>(mbeg[ms] + ord);
                } else {
                    map[qq] = static_cast<uint32_t>(row0 + rank_of(b1, pre1, k));
                }
            }
            q += ce - cs;
            __syncthreads();
        }
        __syncthreads();
    }
}

// ---- numeric ----
struct StageSmem {
    int32_t j[kEntryChunk];
    int32_t pc[kEntryChunk];
    int32_t cs[kEntryChunk + 1];
    double a[kEntryChunk];
    double d[kEntryChunk];
};

__global__ void __launch_bounds__(kT) ada_stage_kernel(
    int m, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci, const double* __restrict__ val,
    const int32_t* __restrict__ rpT, const double* __restrict__ valT, const double* __restrict__ d,
    const int64_t* __restrict__ rpN, const int64_t* __restrict__ qrow, const uint32_t* __restrict__ map,
    double* __restrict__ nval, double* __restrict__ scratch) {
    extern __shared__ double stage[];
    __shared__ StageSmem s;
    __shared__ int64_t sh[32];
    for (int i = blockIdx.x; i < m; i += gridDim.x) {
        const int64_t row0 = rpN[i];
        const int64_t L = rpN[i + 1] - row0;
        const bool staged = L <= kStage;
        int64_t q0 = qrow[i];
        for (int e0 = rp[i]; e0 < rp[i + 1]; e0 += kEntryChunk) {
            const int ne = min(kEntryChunk, rp[i + 1] - e0);
            // entries of this chunk: column, value, d_j, column start, contribution count
            int64_t cnt_local = 0;
            int cntv[kEntryChunk / kT];
#pragma unroll
            for (int u = 0; u < kEntryChunk / kT; ++u) {
                const int t = threadIdx.x * (kEntryChunk / kT) + u;
                int c = 0;
                if (t < ne) {
                    const int e = e0 + t;
                    const double a = val[e];
                    const int j = ci[e];
                    const int p0 = rpT[j];
                    c = (a == 0.0) ? 0 : rpT[j + 1] - p0;
                    s.j[t] = j;
                    s.pc[t] = p0;
                    s.a[t] = a;
                    s.d[t] = d[j];
                }
                cntv[u] = c;
                cnt_local += c;
            }
            int64_t total;
            int64_t pre = block_exclusive_scan_i64<kT>(cnt_local, sh, &total);
#pragma unroll
            for (int u = 0; u < kEntryChunk / kT; ++u) {
                const int t = threadIdx.x * (kEntryChunk / kT) + u;
                if (t < ne) s.cs[t] = static_cast<int32_t>(pre);
                pre += cntv[u];
            }
            if (threadIdx.x == 0) s.cs[ne] = static_cast<int32_t>(total);
            __syncthreads();
            const int Qc = static_cast<int>(total);
            // kUnroll contributions per thread per trip: all their loads are
            // issued before any is used, so each thread keeps 2*kUnroll loads
            // in flight instead of one dependent pair
            for (int base = 0; base < Qc; base += kT * kUnroll) {
                uint32_t tgt[kUnroll];
                double aT[kUnroll], coef[kUnroll], dd[kUnroll];
#pragma unroll
                for (int u = 0; u < kUnroll; ++u) {
                    const int qq = base + u * kT + threadIdx.x;
                    tgt[u] = 0u;
                    aT[u] = 0.0;
                    coef[u] = 0.0;
                    dd[u] = 0.0;
                    if (qq < Qc) {
                        // entry of contribution qq: last t with cs[t] <= qq
                        int lo = 0, hi = ne - 1;
                        while (lo < hi) {
                            const int mid = (lo + hi + 1) >> 1;
                            if (s.cs[mid] <= qq)
                                lo = mid;
                            else
                                hi = mid - 1;
                        }
                        const int p = s.pc[lo] + (qq - s.cs[lo]);
                        tgt[u] = __ldcs(map + q0 + qq);
                        aT[u] = __ldg(valT + p);
                        coef[u] = s.a[lo];
                        dd[u] = s.d[lo];
                    }
                }
#pragma unroll
                for (int u = 0; u < kUnroll; ++u) {
                    const int qq = base + u * kT + threadIdx.x;
                    if (qq >= Qc) continue;
                    const double v = (dd[u] <= 0.0) ? 0.0 : (coef[u] * aT[u]) * dd[u];
                    if (tgt[u] & kMulti)
                        scratch[tgt[u] & ~kMulti] = v;
                    else if (staged)
                        stage[static_cast<int64_t>(tgt[u]) - row0] = v;
                    else
                        nval[tgt[u]] = v;
                }
            }
            q0 += total;
            __syncthreads();
        }
        if (staged)
            for (int t = threadIdx.x; t < L; t += kT) nval[row0 + t] = stage[t];
        __syncthreads();
    }
}

__global__ void ada_combine_kernel(int64_t nms, const int64_t* __restrict__ mpos, const int32_t* __restrict__ mbeg,
                                   const double* __restrict__ scratch, double* __restrict__ nval,
                                   unsigned long long* maxdiag) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= nms) return;
    double s = 0.0;
    for (int32_t u = mbeg[t]; u < mbeg[t + 1]; ++u) s += scratch[u];
    const int64_t mp = mpos[t];
    nval[mp & ~kDiagFlag] = s;
    if ((mp & kDiagFlag) && s > 0.0) atomicMax(maxdiag, static_cast<unsigned long long>(__double_as_longlong(s)));
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
    dfree(P->qrow);
    dfree(P->map);
    dfree(P->mpos);
    dfree(P->mbeg);
    dfree(P->scratch);
    delete P;
}

int64_t d2h_i64(const int64_t* p, cudaStream_t s) {
    int64_t v = 0;
    check_cuda(cudaMemcpyAsync(&v, p, sizeof(v), cudaMemcpyDeviceToHost, s), "D2H scalar");
    check_cuda(cudaStreamSynchronize(s), "D2H sync");
    return v;
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
            fail(HN_ERR_UNSUPPORTED, "m = " + std::to_string(m) + " exceeds the 400,000-row symbolic limit");
        hn_pattern* P = new hn_pattern();
        cudaStream_t s = nullptr;
        int64_t *len = nullptr, *nms = nullptr, *nmq = nullptr;
        int32_t* mcnt = nullptr;
        try {
            P->m = m;
            P->A = A;
            P->rp = dmalloc<int64_t>(m + 1);
            P->qrow = dmalloc<int64_t>(m + 1);
            P->diag_pos = dmalloc<int64_t>(m);
            P->maxdiag = dmalloc<unsigned long long>(1);
            nms = dmalloc<int64_t>(m + 1);
            nmq = dmalloc<int64_t>(m + 1);
            for (int64_t* a : {P->rp, P->qrow, nms, nmq})
                check_cuda(cudaMemsetAsync(a, 0, sizeof(int64_t) * (m + 1), s), "memset");
            const size_t smem_count = 2 * sizeof(uint32_t) * (size_t)(W > 0 ? W : 1);
            const size_t smem_fill = 4 * sizeof(uint32_t) * (size_t)(W > 0 ? W : 1);
            check_cuda(cudaFuncSetAttribute(ada_count_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)smem_count),
                       "smem attribute");
            check_cuda(cudaFuncSetAttribute(ada_fill_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)smem_fill),
                       "smem attribute");
            const int grid = (int)std::min<int64_t>(std::max<int64_t>(m, 1), (int64_t)ctx().sm_count * 8);
            if (m > 0) {
                ada_count_kernel<<<grid, kT, smem_count, s>>>((int)m, A->rp, A->ci, A->val, A->rpT, A->ciT, (int)W,
                                                              P->rp, P->qrow, nms, nmq);
                launched("ada_count_kernel");
            }
            scan_exclusive_i64(P->rp, P->rp, m + 1, s);
            scan_exclusive_i64(P->qrow, P->qrow, m + 1, s);
            scan_exclusive_i64(nms, nms, m + 1, s);
            scan_exclusive_i64(nmq, nmq, m + 1, s);
            P->nnz = d2h_i64(P->rp + m, s);
            P->nq = d2h_i64(P->qrow + m, s);
            P->nms = d2h_i64(nms + m, s);
            P->nmq = d2h_i64(nmq + m, s);
            if (P->nnz >= (int64_t(1) << 31) || P->nmq >= (int64_t(1) << 31))
                fail(HN_ERR_UNSUPPORTED, "nnz(N) = " + std::to_string(P->nnz) + " exceeds the 2^31 slot limit");
            P->ci = dmalloc<int32_t>(P->nnz);
            P->map = dmalloc<uint32_t>(P->nq);
            P->mpos = dmalloc<int64_t>(P->nms);
            P->mbeg = dmalloc<int32_t>(P->nms + 1);
            P->scratch = dmalloc<double>(P->nmq);
            mcnt = dmalloc<int32_t>(P->nms);
            const int32_t last = static_cast<int32_t>(P->nmq);
            check_cuda(cudaMemcpyAsync(P->mbeg + P->nms, &last, sizeof(last), cudaMemcpyHostToDevice, s), "H2D");
            if (m > 0) {
                ada_fill_kernel<<<grid, kT, smem_fill, s>>>((int)m, A->rp, A->ci, A->val, A->rpT, A->ciT, (int)W,
                                                            P->rp, P->qrow, nms, nmq, P->ci, P->diag_pos, P->mpos,
                                                            mcnt, P->mbeg, P->map);
                launched("ada_fill_kernel");
            }
            // opt in above the 48 KB default: dynamic stage buffer + the static entry tables
            check_cuda(cudaFuncSetAttribute(ada_stage_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)(sizeof(double) * kStage + 16384)),
                       "smem attribute");
            check_cuda(cudaStreamSynchronize(s), "symbolic sync");
        } catch (...) {
            dfree(nms);
            dfree(nmq);
            dfree(mcnt);
            free_pattern(P);
            throw;
        }
        dfree(nms);
        dfree(nmq);
        dfree(mcnt);
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
        const int grid = (int)std::min<int64_t>(P->m, (int64_t)ctx().sm_count * 3);
        ada_stage_kernel<<<grid, kT, sizeof(double) * kStage, s>>>((int)P->m, A->rp, A->ci, A->val, A->rpT,
                                                                   A->valT, d, P->rp, P->qrow, P->map, nval,
                                                                   P->scratch);
        launched("ada_stage_kernel");
        if (P->nms > 0) {
            ada_combine_kernel<<<(unsigned)((P->nms + 255) / 256), 256, 0, s>>>(P->nms, P->mpos, P->mbeg,
                                                                                P->scratch, nval, P->maxdiag);
            launched("ada_combine_kernel");
        }
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
