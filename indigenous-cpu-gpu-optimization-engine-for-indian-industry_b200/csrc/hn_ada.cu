// Normal-equation assembly N = A diag(d) A^T + dyn_reg I
// (build_normal_equations, core/lp/interior_point.cpp:144-200).
//
// A "contribution" is one term (A_ij * A_kj) * d_j: row i of N, entry e of
// row i of A (column j), row k of column j. Contributions are numbered q in
// a fixed structural order -- rows i ascending, entries e of row i in CSR
// order, then the rows k of column j (A^T row j) ascending.
//
// Symbolic (once per A; integer work only, exact):
//   one CTA per row i builds two shared-memory bitmaps over the columns of N
//   that row i can reach (its window, from the first and last row of each of
//   its columns in A^T): b1 = k reached at least once (plus k = i), b2 = k
//   reached twice or more (plus k = i). popcounts give the row length, the
//   number of terms, of "multi" slots (b2) and of terms into multi slots;
//   after scans, a second pass writes the sorted pattern (scanning b1), the
//   table of multi slots and the gather map: for each slot of N, the A^T and
//   A positions of its single term, or the multi-slot index; the terms of a
//   multi slot are listed in column order.
// Numeric (every IPM iteration), three streaming kernels:
//   slot   : one thread per slot of N, in slot order: reads its (p, e) pair,
//            gathers A_ij, A_kj, d_j (L2-resident) and writes the value --
//            fully coalesced, no search, no atomics, no shared memory.
//            Single-term slots are ~98% of N for random LPs.
//   combine: one thread per multi slot sums its terms in column order -- the
//            order the reference accumulates the diagonal (:188-191) -- and
//            takes the max diagonal.
//   reg    : N_ii += dyn_reg = max(reg, 1e-12 * max diag) (:193-196).
// HBM traffic per numeric call: 8 bytes of map + 8 bytes of N per slot.
#include <algorithm>
#include <vector>

#include "hn_internal.cuh"

namespace hn {
namespace {

constexpr int kT = 256;
constexpr int64_t kMaxBitmapWords = 12500;  // row reach <= 400,000 columns: four W-word arrays in 200 KB of shared memory
constexpr uint32_t kMulti = 0x80000000u;
constexpr int64_t kDiagFlag = int64_t(1) << 62;
constexpr int kSlotsPerThread = 4;  // slots per thread per trip of the numeric kernel
constexpr uint16_t kSlotMulti = 0xFFFFu;
constexpr int kRowThreads = 256;     // row-mode numeric kernel
constexpr int kRowWindow = 8192;     // row mode: slots of a row of N assembled per pass (64 KB)
constexpr int kRowMaxSlots = 65534;  // row mode: slot offsets fit 16 bits
constexpr int kRowMaxEntries = 256;  // row mode: entries of a row of A staged in shared memory

__device__ __forceinline__ uint32_t bit_of(int k) { return 1u << (k & 31); }

// Reach of row i: the smallest and largest k it touches (its own index
// included), as a first bitmap word and a word count. Block-diagonal batches
// have reaches of one block, so their bitmaps stay small whatever m is.
__global__ void ada_window_kernel(int m, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                                  const double* __restrict__ val, const int32_t* __restrict__ rpT,
                                  const int32_t* __restrict__ ciT, int32_t* __restrict__ wbase,
                                  int32_t* __restrict__ wcount, unsigned* __restrict__ wmax) {
    const int64_t i = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (i >= m) return;
    int lo = (int)i, hi = (int)i;
    for (int e = rp[i] + lane; e < rp[i + 1]; e += 32) {
        if (val[e] == 0.0) continue;
        const int j = ci[e];
        if (rpT[j + 1] > rpT[j]) {
            lo = min(lo, ciT[rpT[j]]);
            hi = max(hi, ciT[rpT[j + 1] - 1]);
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
        hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    }
    if (lane == 0) {
        wbase[i] = lo >> 5;
        const int wc = (hi >> 5) - (lo >> 5) + 1;
        wcount[i] = wc;
        atomicMax(wmax, (unsigned)wc);
    }
}

// Marks every contribution of row i: b1 |= bit(k); if it was set already,
// b2 |= bit(k). Bitmap word w covers k in [(wb + w) * 32, (wb + w) * 32 + 32).
__device__ __forceinline__ void mark_contributions(int i, int wb, const int32_t* __restrict__ rp,
                                                   const int32_t* __restrict__ ci, const double* __restrict__ val,
                                                   const int32_t* __restrict__ rpT, const int32_t* __restrict__ ciT,
                                                   uint32_t* b1, uint32_t* b2, int64_t* nq_local) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) {
        atomicOr(&b1[(i >> 5) - wb], bit_of(i));
        atomicOr(&b2[(i >> 5) - wb], bit_of(i));  // the diagonal is always a multi slot (it gets dyn_reg)
    }
    int64_t cnt = 0;
    for (int e = rp[i] + warp; e < rp[i + 1]; e += kT / 32) {
        if (val[e] == 0.0) continue;
        const int j = ci[e];
        for (int p = rpT[j] + lane; p < rpT[j + 1]; p += 32) {
            const int k = ciT[p];
            const uint32_t old = atomicOr(&b1[(k >> 5) - wb], bit_of(k));
            if (old & bit_of(k)) atomicOr(&b2[(k >> 5) - wb], bit_of(k));
            ++cnt;
        }
    }
    *nq_local = cnt;
}

__global__ void __launch_bounds__(kT) ada_count_kernel(int m, const int32_t* __restrict__ rp,
                                                       const int32_t* __restrict__ ci,
                                                       const double* __restrict__ val,
                                                       const int32_t* __restrict__ rpT,
                                                       const int32_t* __restrict__ ciT, int Wmax,
                                                       const int32_t* __restrict__ wbase,
                                                       const int32_t* __restrict__ wcount,
                                                       int64_t* __restrict__ len, int64_t* __restrict__ nq,
                                                       int64_t* __restrict__ nms, int64_t* __restrict__ nmq,
                                                       unsigned* __restrict__ maxes) {
    extern __shared__ uint32_t smem[];
    uint32_t* b1 = smem;
    uint32_t* b2 = smem + Wmax;
    __shared__ int64_t sh[32];
    for (int i = blockIdx.x; i < m; i += gridDim.x) {
        const int W = wcount[i];
        for (int w = threadIdx.x; w < W; w += kT) {
            b1[w] = 0u;
            b2[w] = 0u;
        }
        __syncthreads();
        int64_t q;
        mark_contributions(i, wbase[i], rp, ci, val, rpT, ciT, b1, b2, &q);
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
            atomicMax(maxes + 1, (unsigned)L);
            atomicMax(maxes + 2, (unsigned)(rp[i + 1] - rp[i]));
        }
        __syncthreads();
    }
}

__device__ __forceinline__ int rank_of(const uint32_t* b, const int32_t* pre, int k, int wb) {
    return pre[(k >> 5) - wb] + __popc(b[(k >> 5) - wb] & (bit_of(k) - 1u));
}

__global__ void __launch_bounds__(kT) ada_fill_kernel(
    int m, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci, const double* __restrict__ val,
    const int32_t* __restrict__ rpT, const int32_t* __restrict__ ciT, int Wmax, const int32_t* __restrict__ wbase,
    const int32_t* __restrict__ wcount, const int64_t* __restrict__ rpN, const int64_t* __restrict__ msrow,
    const int64_t* __restrict__ mqrow, int32_t* __restrict__ ciN, int64_t* __restrict__ diag_pos,
    int64_t* __restrict__ mpos, int32_t* mcnt, int32_t* __restrict__ mbeg, uint2* __restrict__ gmap,
    uint2* __restrict__ mlist, const int64_t* __restrict__ tq, uint16_t* __restrict__ smap,
    uint32_t* __restrict__ rmap, int qbits) {
    extern __shared__ uint32_t smem[];
    uint32_t* b1 = smem;
    uint32_t* b2 = smem + Wmax;
    int32_t* pre1 = reinterpret_cast<int32_t*>(smem + 2 * Wmax);
    int32_t* pre2 = reinterpret_cast<int32_t*>(smem + 3 * Wmax);
    __shared__ int64_t sh[32];
    for (int i = blockIdx.x; i < m; i += gridDim.x) {
        const int W = wcount[i], wb = wbase[i];
        const int wpt = (W + kT - 1) / kT;
        for (int w = threadIdx.x; w < W; w += kT) {
            b1[w] = 0u;
            b2[w] = 0u;
        }
        __syncthreads();
        int64_t unused;
        mark_contributions(i, wb, rp, ci, val, rpT, ciT, b1, b2, &unused);
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
                const int k = (wb + w) * 32 + b;
                const int64_t pos = row0 + o1;
                ciN[pos] = k;
                if (k == i) diag_pos[i] = pos;
                if ((bits2 >> b) & 1u) {
                    mpos[ms0 + o2] = pos | (k == i ? kDiagFlag : 0);
                    mcnt[ms0 + o2] = 0;
                    if (gmap) gmap[pos] = make_uint2(kMulti | static_cast<uint32_t>(ms0 + o2), 0u);
                    if (rmap) rmap[pos] = kMulti | static_cast<uint32_t>(o2);
                    ++o2;
                }
                ++o1;
                bits &= bits - 1;
            }
        }
        __syncthreads();
        // terms per multi slot
        {
            const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
            for (int e = rp[i] + warp; e < rp[i + 1]; e += kT / 32) {
                if (val[e] == 0.0) continue;
                const int j = ci[e];
                for (int p = rpT[j] + lane; p < rpT[j + 1]; p += 32) {
                    const int k = ciT[p];
                    if (b2[(k >> 5) - wb] & bit_of(k)) atomicAdd(&mcnt[ms0 + rank_of(b2, pre2, k, wb)], 1);
                }
            }
        }
        __syncthreads();
        // term ranges of this row's multi slots (then mcnt becomes a cursor)
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
        // gather map (or slot map); entries e go one after the other so the
        // terms of each multi slot are listed in column order
        int64_t tloc = smap ? tq[i] : 0;
        for (int e = rp[i]; e < rp[i + 1]; ++e) {
            if (val[e] == 0.0) continue;
            const int j = ci[e];
            const int cs = rpT[j], ce = rpT[j + 1];
            for (int p = cs + threadIdx.x; p < ce; p += kT) {
                const int k = ciT[p];
                const uint2 pe = make_uint2(static_cast<uint32_t>(p), static_cast<uint32_t>(e));
                const bool multi = b2[(k >> 5) - wb] & bit_of(k);
                if (multi) {
                    const int64_t ms = ms0 + rank_of(b2, pre2, k, wb);
                    const int ord = atomicAdd(&mcnt[ms], 1);
                    mlist[mbeg[ms] + ord] = pe;
                } else if (gmap) {
                    gmap[row0 + rank_of(b1, pre1, k, wb)] = pe;
                } else if (rmap) {
                    rmap[row0 + rank_of(b1, pre1, k, wb)] =
                        (static_cast<uint32_t>(e - rp[i]) << qbits) | static_cast<uint32_t>(p - cs);
                }
                if (smap) smap[tloc + (p - cs)] = multi ? kSlotMulti : static_cast<uint16_t>(rank_of(b1, pre1, k, wb));
            }
            tloc += ce - cs;
            __syncthreads();
        }
        __syncthreads();
    }
}

// ---- numeric ----
// vd[e] = (A value e, d of its column): one 16-byte gather per term instead of
// a value load plus a dependent column-index -> d chain.
__global__ void ada_vd_kernel(int64_t nnz, const double* __restrict__ val, const int32_t* __restrict__ ci,
                              const double* __restrict__ d, double2* __restrict__ vd) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nnz; e += (int64_t)gridDim.x * blockDim.x)
        vd[e] = make_double2(val[e], __ldg(d + ci[e]));
}

__device__ __forceinline__ double term(uint2 pe, const double2* __restrict__ vd, const double* __restrict__ valT) {
    const double2 q = __ldg(vd + pe.y);
    return (q.y <= 0.0) ? 0.0 : (q.x * __ldg(valT + pe.x)) * q.y;  // columns with D_j <= 0 skipped
}

// Numeric phase, two kernels per call:
//   ada_combine_kernel sums every multi slot's terms in column order (the
//     order from_triplets' stable sort leaves them in) into the compact mval;
//   ada_slot_kernel then writes every slot of N once, in slot order: a single
//     term (A value x A^T value) x d, or the multi slot's mval entry.
// In the slot kernel each thread handles kSlotsPerThread slots per trip; all
// gathers of a trip are issued before any use (a multi slot reads mval and
// gathers entry 0, which always exists), and the next trip's map entries are
// loaded before this trip's gathers, so the map stream from HBM overlaps the
// gathers from L2.
__global__ void __launch_bounds__(kT, 4) ada_slot_kernel(int64_t nnz, const uint2* __restrict__ gmap,
                                                         const double2* __restrict__ vd,
                                                         const double* __restrict__ valT,
                                                         const double* __restrict__ mval, double* __restrict__ nval) {
    const int64_t stride = (int64_t)gridDim.x * kT * kSlotsPerThread;
    int64_t t0 = blockIdx.x * (int64_t)kT * kSlotsPerThread + threadIdx.x;
    uint2 g[kSlotsPerThread];
#pragma unroll
    for (int u = 0; u < kSlotsPerThread; ++u) {
        const int64_t t = t0 + (int64_t)u * kT;
        g[u] = t < nnz ? __ldcs(gmap + t) : make_uint2(kMulti, 0u);
    }
    for (; t0 < nnz; t0 += stride) {
        uint2 gn[kSlotsPerThread];
#pragma unroll
        for (int u = 0; u < kSlotsPerThread; ++u) {
            const int64_t t = t0 + stride + (int64_t)u * kT;
            gn[u] = t < nnz ? __ldcs(gmap + t) : make_uint2(kMulti, 0u);
        }
        double2 q[kSlotsPerThread];
        double b[kSlotsPerThread];
#pragma unroll
        for (int u = 0; u < kSlotsPerThread; ++u) {
            const bool multi = g[u].x & kMulti;
            const int64_t t = t0 + (int64_t)u * kT;
            q[u] = __ldg(vd + (multi ? 0u : g[u].y));
            b[u] = (multi && t < nnz) ? __ldcs(mval + (g[u].x & ~kMulti)) : __ldg(valT + (multi ? 0u : g[u].x));
        }
#pragma unroll
        for (int u = 0; u < kSlotsPerThread; ++u) {
            const int64_t t = t0 + (int64_t)u * kT;
            if (t >= nnz) continue;
            const double v = (g[u].x & kMulti) ? b[u]
                             : (q[u].y <= 0.0) ? 0.0  // columns with D_j <= 0 skipped
                                               : (q[u].x * b[u]) * q[u].y;
            __stcs(nval + t, v);
        }
#pragma unroll
        for (int u = 0; u < kSlotsPerThread; ++u) g[u] = gn[u];
    }
}

// Relative map: one warp per row of N at a time (rows handed out longest
// first), kRmapU slots per lane per trip, the next trip's map words loaded
// before this trip's gathers. A single-term slot's word gives its A entry
// within row i (high bits: e - rp_A[i]) and its A^T entry within row j of
// A^T (low bits: p - rp_AT[j]). The warp first stages its row's A entries --
// (A value, d) and the start of the A^T row of their column -- in its own
// shared-memory slice (rows of A are at most kRmapTerms long in this
// layout), so a slot costs one 4-byte map word from HBM, two shared loads
// and one A^T value gathered through L1 (the slots of a row walk each of its
// A^T rows in order, so neighbouring values share lines). (A value x A^T
// value) x d is the slot kernel's arithmetic, so the layouts give the same
// bits. Every index read from the map is clamped into its table, so a
// corrupt map gives wrong values, never an access outside the buffers.
constexpr int kRmapU = 8;
constexpr int kRmapT = 256;      // threads (8 warps, one row each)
constexpr int kRmapTerms = 256;  // longest row of A this layout takes
constexpr int64_t kRmapMinRow = 2048;  // mean slots per row of N above which it is the default
__global__ void __launch_bounds__(kRmapT, 3) ada_rmap_kernel(int m, const int32_t* __restrict__ order,
                                                             unsigned* __restrict__ row_next,
                                                             const int32_t* __restrict__ rpA,
                                                             const double2* __restrict__ vd,
                                                             const int32_t* __restrict__ ecs,
                                                             const double* __restrict__ valT, int64_t nnzA,
                                                             const int64_t* __restrict__ rpN,
                                                             const int64_t* __restrict__ msrow, int64_t nms,
                                                             const uint32_t* __restrict__ rmap, int qbits,
                                                             const double* __restrict__ mval,
                                                             double* __restrict__ nval) {
    __shared__ double2 s_q[kRmapT / 32][kRmapTerms];
    __shared__ int32_t s_cs[kRmapT / 32][kRmapTerms];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double2* sq = s_q[warp];
    int32_t* scs = s_cs[warp];
    const uint32_t qmask = (1u << qbits) - 1u;
    constexpr int64_t kStep = 32 * kRmapU;
    for (;;) {
        unsigned idx = 0;
        if (lane == 0) idx = atomicAdd(row_next, 1u);
        idx = __shfl_sync(0xffffffffu, idx, 0);
        if (idx >= static_cast<unsigned>(m)) return;
        const int i = __ldg(order + idx);
        const int64_t r0 = __ldg(rpN + i), r1 = __ldg(rpN + i + 1);
        const int e0 = __ldg(rpA + i);
        const int ne = min(__ldg(rpA + i + 1) - e0, kRmapTerms);
        const int64_t ms0 = __ldg(msrow + i);
        __syncwarp();  // the previous row's slots are done with the slice
        for (int t = lane; t < ne; t += 32) {
            sq[t] = __ldg(vd + e0 + t);
            scs[t] = __ldg(ecs + e0 + t);
        }
        __syncwarp();
        uint32_t g[kRmapU];
#pragma unroll
        for (int u = 0; u < kRmapU; ++u) {
            const int64_t t = r0 + lane + u * 32;
            g[u] = t < r1 ? __ldcs(rmap + t) : kMulti;
        }
        for (int64_t t0 = r0 + lane; t0 < r1; t0 += kStep) {
            uint32_t gn[kRmapU];
#pragma unroll
            for (int u = 0; u < kRmapU; ++u) {
                const int64_t t = t0 + kStep + u * 32;
                gn[u] = t < r1 ? __ldcs(rmap + t) : kMulti;
            }
            double2 q[kRmapU];
            double b[kRmapU];
#pragma unroll
            for (int u = 0; u < kRmapU; ++u) {
                const int64_t t = t0 + u * 32;
                if (g[u] & kMulti) {
                    const int64_t ms = min(ms0 + (int64_t)(g[u] & ~kMulti), nms - 1);
                    q[u] = make_double2(0.0, 0.0);
                    b[u] = t < r1 ? __ldcs(mval + ms) : 0.0;
                } else {
                    const int eo = min(static_cast<int>(g[u] >> qbits), kRmapTerms - 1);
                    q[u] = sq[eo];
                    int64_t pT = (int64_t)scs[eo] + (int64_t)(g[u] & qmask);
                    pT = pT < nnzA ? pT : 0;
                    b[u] = __ldg(valT + pT);
                }
            }
#pragma unroll
            for (int u = 0; u < kRmapU; ++u) {
                const int64_t t = t0 + u * 32;
                if (t >= r1) continue;
                const double v = (g[u] & kMulti) ? b[u]
                                 : (q[u].y <= 0.0) ? 0.0  // columns with D_j <= 0 skipped
                                                   : (q[u].x * b[u]) * q[u].y;
                __stcs(nval + t, v);
            }
#pragma unroll
            for (int u = 0; u < kRmapU; ++u) g[u] = gn[u];
        }
    }
}

__global__ void ada_ecs_kernel(int64_t nnz, const int32_t* __restrict__ ci, const int32_t* __restrict__ rpT,
                               int32_t* __restrict__ ecs) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nnz; e += (int64_t)gridDim.x * blockDim.x)
        ecs[e] = rpT[ci[e]];
}

// The first kBatch terms of a slot are gathered together; longer lists
// continue one term at a time.
constexpr int kBatch = 4;
__global__ void ada_combine_kernel(int64_t nms, const int64_t* __restrict__ mpos, const int32_t* __restrict__ mbeg,
                                   const uint2* __restrict__ mlist, const double2* __restrict__ vd,
                                   const double* __restrict__ valT, double* __restrict__ mval,
                                   unsigned long long* maxdiag) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= nms) return;
    const int32_t u0 = mbeg[t], u1 = mbeg[t + 1];
    uint2 pe[kBatch];
#pragma unroll
    for (int k = 0; k < kBatch; ++k) pe[k] = (u0 + k < u1) ? __ldg(mlist + u0 + k) : make_uint2(0u, 0u);
    double2 q[kBatch];
    double b[kBatch];
#pragma unroll
    for (int k = 0; k < kBatch; ++k) {
        q[k] = __ldg(vd + pe[k].y);
        b[k] = __ldg(valT + pe[k].x);
    }
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < kBatch; ++k)
        if (u0 + k < u1) s += (q[k].y <= 0.0) ? 0.0 : (q[k].x * b[k]) * q[k].y;
    for (int32_t u = u0 + kBatch; u < u1; ++u) s += term(mlist[u], vd, valT);
    mval[t] = s;
    if ((mpos[t] & kDiagFlag) && s > 0.0)
        atomicMax(maxdiag, static_cast<unsigned long long>(__double_as_longlong(s)));
}

// Row mode: one CTA per row of N at a time, the row assembled in shared
// memory in windows of kRowWindow slots. The row's A entries (value, d,
// A^T row start, term offset) are staged in shared memory; then each warp
// takes whole entries e (column j) and its lanes walk the entry's terms --
// row j of A^T and the matching run of 2-byte slot offsets -- contiguously,
// kRowU terms per lane in flight, so A^T values and offsets arrive in
// coalesced lines instead of one random 32-byte sector per slot. A
// single-term slot in the window gets (A value x A^T value) x d at its
// offset, the window's multi slots take their combined sums from mval, and
// the window leaves in one coalesced streaming store; a row longer than the
// window walks its terms once per window. The arithmetic of each slot is the
// slot kernel's, so every layout gives the same bits.
constexpr int kRowU = 4;
constexpr size_t kRowSmem = sizeof(double) * kRowWindow + sizeof(double2) * kRowMaxEntries +
                            sizeof(int32_t) * (2 * kRowMaxEntries + 1);
__global__ void __launch_bounds__(kRowThreads, 3) ada_row_kernel(
    int m, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci, const double2* __restrict__ vd,
    const int32_t* __restrict__ rpT, const double* __restrict__ valT, const int64_t* __restrict__ tq,
    const uint16_t* __restrict__ smap, const int64_t* __restrict__ rpN, const int64_t* __restrict__ msrow,
    const int64_t* __restrict__ mpos, const double* __restrict__ mval, double* __restrict__ nval) {
    extern __shared__ __align__(16) double row_smem[];
    double* srow = row_smem;
    double2* s_vd = reinterpret_cast<double2*>(row_smem + kRowWindow);
    int32_t* s_cs = reinterpret_cast<int32_t*>(s_vd + kRowMaxEntries);
    int32_t* s_to = s_cs + kRowMaxEntries;
    __shared__ int64_t sh[32];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    constexpr int kWarps = kRowThreads / 32;
    for (int i = blockIdx.x; i < m; i += gridDim.x) {
        const int e0 = rp[i], ne = rp[i + 1] - e0;
        // term counts per entry (0 for an explicit zero of A), exclusive scan
        int64_t cnt = 0;
        if (tid < ne) {
            const double2 q = vd[e0 + tid];
            const int j = ci[e0 + tid];
            const int cs = rpT[j];
            s_vd[tid] = q;
            s_cs[tid] = cs;
            cnt = (q.x == 0.0) ? 0 : rpT[j + 1] - cs;
        }
        int64_t tot;
        const int64_t ex = block_exclusive_scan_i64<kRowThreads>(cnt, sh, &tot);
        if (tid < ne) s_to[tid] = static_cast<int32_t>(ex);
        if (tid == 0) s_to[ne] = static_cast<int32_t>(tot);
        __syncthreads();
        const uint16_t* sm = smap + tq[i];
        const int64_t r0 = rpN[i];
        const int L = static_cast<int>(rpN[i + 1] - r0);
        const int64_t ms0 = msrow[i], ms1 = msrow[i + 1];
        for (int w0 = 0; w0 < L; w0 += kRowWindow) {
            const int w1 = min(L, w0 + kRowWindow);
            for (int e = warp; e < ne; e += kWarps) {
                const int t0 = s_to[e], c = s_to[e + 1] - t0;
                if (c == 0) continue;
                const double2 q = s_vd[e];
                const double* vT = valT + s_cs[e];
                const uint16_t* se = sm + t0;
                for (int p0 = lane; p0 < c; p0 += 32 * kRowU) {
                    uint16_t slot[kRowU];
                    double b[kRowU];
#pragma unroll
                    for (int u = 0; u < kRowU; ++u) {
                        const int p = p0 + 32 * u;
                        slot[u] = p < c ? __ldcs(se + p) : kSlotMulti;
                        b[u] = p < c ? __ldcg(vT + p) : 0.0;
                    }
#pragma unroll
                    for (int u = 0; u < kRowU; ++u) {
                        const int sl = slot[u];
                        if (sl != kSlotMulti && sl >= w0 && sl < w1)
                            srow[sl - w0] = (q.y <= 0.0) ? 0.0 : (q.x * b[u]) * q.y;  // columns with D_j <= 0 skipped
                    }
                }
            }
            for (int64_t ms = ms0 + tid; ms < ms1; ms += kRowThreads) {
                const int64_t k = (mpos[ms] & ~kDiagFlag) - r0;
                if (k >= w0 && k < w1) srow[k - w0] = __ldcs(mval + ms);
            }
            __syncthreads();
            for (int k = w0 + tid; k < w1; k += kRowThreads) __stcs(nval + r0 + k, srow[k - w0]);
            __syncthreads();
        }
    }
}

// term counts of a row rounded up to whole 16-byte chunks of the slot map
__global__ void pad8_kernel(int64_t m, const int64_t* __restrict__ nq, int64_t* __restrict__ out) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < m) out[i] = (nq[i] + 7) & ~int64_t(7);
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
    for (void* p : {(void*)P->rp, (void*)P->ci, (void*)P->diag_pos, (void*)P->maxdiag, (void*)P->gmap,
                    (void*)P->mpos, (void*)P->mbeg, (void*)P->mlist, (void*)P->vd, (void*)P->mval, (void*)P->tq,
                    (void*)P->smap, (void*)P->msrow, (void*)P->rmap, (void*)P->ecs, (void*)P->order,
                    (void*)P->row_next})
        dfree(p);
    delete P;
}

int64_t d2h_i64(const int64_t* p, cudaStream_t s) {
    int64_t v = 0;
    check_cuda(cudaMemcpyAsync(&v, p, sizeof(v), cudaMemcpyDeviceToHost, s), "D2H scalar");
    check_cuda(cudaStreamSynchronize(s), "D2H sync");
    return v;
}

void launch_numeric(const hn_pattern* P, const double* d, double* nval, cudaStream_t s) {
    const hn_csr* A = P->A;
    if (A->nnz > 0) {
        const int gv = (int)std::min<int64_t>((A->nnz + kT - 1) / kT, (int64_t)ctx().sm_count * 16);
        ada_vd_kernel<<<gv, kT, 0, s>>>(A->nnz, A->val, A->ci, d, P->vd);
        launched("ada_vd_kernel");
    }
    check_cuda(cudaMemsetAsync(P->maxdiag, 0, sizeof(unsigned long long), s), "memset maxdiag");
    if (P->nms > 0) {
        ada_combine_kernel<<<(unsigned)((P->nms + 255) / 256), 256, 0, s>>>(P->nms, P->mpos, P->mbeg, P->mlist,
                                                                            P->vd, A->valT, P->mval, P->maxdiag);
        launched("ada_combine_kernel");
    }
    if (P->row_mode) {
        static int row_attr_device = -1;
        if (row_attr_device != ctx().device) {
            check_cuda(cudaFuncSetAttribute(ada_row_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)kRowSmem),
                       "row kernel smem attribute");
            row_attr_device = ctx().device;
        }
        const int grid = (int)std::min<int64_t>(P->m, (int64_t)ctx().sm_count * 3);
        ada_row_kernel<<<grid, kRowThreads, kRowSmem, s>>>((int)P->m, A->rp, A->ci, P->vd, A->rpT, A->valT, P->tq,
                                                       P->smap, P->rp, P->msrow, P->mpos, P->mval, nval);
        launched("ada_row_kernel");
        return;
    }
    if (P->rmap) {
        check_cuda(cudaMemsetAsync(P->row_next, 0, sizeof(unsigned), s), "memset row counter");
        const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((P->m + 7) / 8, (int64_t)ctx().sm_count * 3));
        ada_rmap_kernel<<<grid, kRmapT, 0, s>>>((int)P->m, P->order, P->row_next, A->rp, P->vd, P->ecs, A->valT,
                                                A->nnz, P->rp, P->msrow, P->nms, P->rmap, P->qbits, P->mval, nval);
        launched("ada_rmap_kernel");
        return;
    }
    const int64_t per_block = (int64_t)kT * kSlotsPerThread;
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((P->nnz + per_block - 1) / per_block,
                                                                 (int64_t)ctx().sm_count * 4));
    ada_slot_kernel<<<grid, kT, 0, s>>>(P->nnz, P->gmap, P->vd, A->valT, P->mval, nval);
    launched("ada_slot_kernel");
}

}  // namespace

void ada_numeric_unregularised(const hn_pattern* P, const double* d, double* nval, cudaStream_t s) {
    if (P->m == 0) return;
    launch_numeric(P, d, nval, s);
}

}  // namespace hn

using namespace hn;

extern "C" {

int hn_ada_symbolic(const hn_csr* A, hn_pattern** out) { return hn_ada_symbolic_ex(A, 0u, out); }

int hn_pattern_mode(const hn_pattern* P, int* row_mode, int64_t* max_row) {
    return guard("hn_pattern_mode", [&] {
        if (!P) fail(HN_ERR_INVALID_ARG, "null pattern");
        if (row_mode) *row_mode = P->row_mode ? 1 : (P->rmap ? 2 : 0);
        if (max_row) *max_row = P->max_row;
    });
}

int hn_ada_symbolic_ex(const hn_csr* A, unsigned flags, hn_pattern** out) {
    return guard("hn_ada_symbolic", [&] {
        require_init();
        if (!A || !out) fail(HN_ERR_INVALID_ARG, "bad arguments");
        if (!A->has_t) fail(HN_ERR_INVALID_ARG, "hn_ada_symbolic needs a handle with A^T");
        *out = nullptr;
        const int64_t m = A->m;
        hn_pattern* P = new hn_pattern();
        cudaStream_t s = nullptr;
        int64_t *nq = nullptr, *nms = nullptr, *nmq = nullptr, *tqa = nullptr;
        int32_t *mcnt = nullptr, *wbase = nullptr, *wcount = nullptr;
        unsigned* wmax_d = nullptr;
        try {
            // row reaches -> bitmap width
            wbase = dmalloc<int32_t>(m);
            wcount = dmalloc<int32_t>(m);
            wmax_d = dmalloc<unsigned>(3);  // widest bitmap, longest row of N, longest row of A
            check_cuda(cudaMemsetAsync(wmax_d, 0, 3 * sizeof(unsigned), s), "memset");
            if (m > 0) {
                ada_window_kernel<<<(unsigned)((m * 32 + 255) / 256), 256, 0, s>>>((int)m, A->rp, A->ci, A->val,
                                                                                  A->rpT, A->ciT, wbase, wcount,
                                                                                  wmax_d);
                launched("ada_window_kernel");
            }
            unsigned wmax_h = 0;
            check_cuda(cudaMemcpyAsync(&wmax_h, wmax_d, sizeof(unsigned), cudaMemcpyDeviceToHost, s), "D2H");
            check_cuda(cudaStreamSynchronize(s), "window sync");
            const int64_t W = std::max<int64_t>(wmax_h, 1);
            if (W > kMaxBitmapWords)
                fail(HN_ERR_UNSUPPORTED, "a row of N reaches " + std::to_string(W * 32) +
                                             " columns; the symbolic bitmaps hold 400,000");
            P->m = m;
            P->A = A;
            P->rp = dmalloc<int64_t>(m + 1);
            P->diag_pos = dmalloc<int64_t>(m);
            P->maxdiag = dmalloc<unsigned long long>(1);
            P->vd = dmalloc<double2>(A->nnz > 0 ? A->nnz : 1);
            nq = dmalloc<int64_t>(m + 1);
            nms = dmalloc<int64_t>(m + 1);
            nmq = dmalloc<int64_t>(m + 1);
            for (int64_t* a : {P->rp, nq, nms, nmq})
                check_cuda(cudaMemsetAsync(a, 0, sizeof(int64_t) * (m + 1), s), "memset");
            const size_t smem_count = 2 * sizeof(uint32_t) * (size_t)W;
            const size_t smem_fill = 4 * sizeof(uint32_t) * (size_t)W;
            check_cuda(cudaFuncSetAttribute(ada_count_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)smem_count),
                       "smem attribute");
            check_cuda(cudaFuncSetAttribute(ada_fill_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)smem_fill),
                       "smem attribute");
            const int grid = (int)std::min<int64_t>(std::max<int64_t>(m, 1), (int64_t)ctx().sm_count * 8);
            if (m > 0) {
                ada_count_kernel<<<grid, kT, smem_count, s>>>((int)m, A->rp, A->ci, A->val, A->rpT, A->ciT, (int)W,
                                                              wbase, wcount, P->rp, nq, nms, nmq, wmax_d);
                launched("ada_count_kernel");
            }
            tqa = dmalloc<int64_t>(m + 1);
            check_cuda(cudaMemsetAsync(tqa, 0, sizeof(int64_t) * (m + 1), s), "memset");
            if (m > 0) {
                pad8_kernel<<<(unsigned)((m + 255) / 256), 256, 0, s>>>(m, nq, tqa);
                launched("pad8_kernel");
            }
            scan_exclusive_i64(tqa, tqa, m + 1, s);
            scan_exclusive_i64(P->rp, P->rp, m + 1, s);
            scan_exclusive_i64(nq, nq, m + 1, s);
            scan_exclusive_i64(nms, nms, m + 1, s);
            scan_exclusive_i64(nmq, nmq, m + 1, s);
            P->nnz = d2h_i64(P->rp + m, s);
            P->nq = d2h_i64(nq + m, s);
            P->nms = d2h_i64(nms + m, s);
            P->nmq = d2h_i64(nmq + m, s);
            if (P->nnz >= (int64_t(1) << 31) || P->nmq >= (int64_t(1) << 31))
                fail(HN_ERR_UNSUPPORTED, "nnz(N) = " + std::to_string(P->nnz) + " exceeds the 2^31 slot limit");
            unsigned maxes[3] = {0, 0, 0};
            check_cuda(cudaMemcpyAsync(maxes, wmax_d, sizeof(maxes), cudaMemcpyDeviceToHost, s), "D2H");
            check_cuda(cudaStreamSynchronize(s), "count sync");
            P->max_row = static_cast<int32_t>(maxes[1]);
            P->row_mode = (flags & HN_ADA_COMPACT) && m > 0 && maxes[1] <= (unsigned)kRowMaxSlots &&
                          maxes[1] < kSlotMulti &&
                          maxes[2] <= (unsigned)kRowMaxEntries && P->nq < (int64_t(1) << 31);
            // relative map: offsets within a row of A (maxes[2] entries) and
            // within a row of A^T must share 31 bits
            int qbits = 0;
            bool rel = false;
            if (!P->row_mode && m > 0 && !(flags & HN_ADA_GATHER8)) {
                std::vector<int32_t> rpT(A->n + 1);
                check_cuda(cudaMemcpy(rpT.data(), A->rpT, sizeof(int32_t) * (A->n + 1), cudaMemcpyDeviceToHost),
                           "D2H rpT");
                int64_t maxcol = 1;
                for (int64_t j = 0; j < A->n; ++j) maxcol = std::max<int64_t>(maxcol, rpT[j + 1] - rpT[j]);
                while ((int64_t(1) << qbits) < maxcol) ++qbits;
                const bool fits = qbits < 31 && (int64_t)std::max(maxes[2], 1u) <= (int64_t(1) << (31 - qbits)) &&
                                  maxes[2] <= (unsigned)kRmapTerms;
                // without a request: the relative map when the rows of N are
                // long enough for a warp per row to amortise its set-up
                const bool long_rows = P->nnz >= kRmapMinRow * m;
                rel = fits && ((flags & HN_ADA_RELATIVE) || (!(flags & HN_ADA_COMPACT) && long_rows));
            }
            P->ci = dmalloc<int32_t>(P->nnz);
            if (P->row_mode) {
                P->smap = dmalloc<uint16_t>(d2h_i64(tqa + m, s));
                P->tq = tqa;
                P->msrow = nms;
                tqa = nms = nullptr;  // owned by the pattern now
            } else if (rel) {
                P->qbits = qbits;
                P->rmap = dmalloc<uint32_t>(P->nnz);
                P->ecs = dmalloc<int32_t>(A->nnz > 0 ? A->nnz : 1);
                P->order = dmalloc<int32_t>(m);
                P->row_next = dmalloc<unsigned>(1);
                P->msrow = nms;
                nms = nullptr;  // owned by the pattern now
                if (A->nnz > 0) {
                    const int ge = (int)std::min<int64_t>((A->nnz + kT - 1) / kT, (int64_t)ctx().sm_count * 16);
                    ada_ecs_kernel<<<ge, kT, 0, s>>>(A->nnz, A->ci, A->rpT, P->ecs);
                    launched("ada_ecs_kernel");
                }
                // rows of N longest first: the counter hands the long rows out early
                std::vector<int64_t> rpn(m + 1);
                check_cuda(cudaMemcpy(rpn.data(), P->rp, sizeof(int64_t) * (m + 1), cudaMemcpyDeviceToHost),
                           "D2H rp");
                std::vector<int32_t> ord(m);
                for (int64_t i = 0; i < m; ++i) ord[i] = static_cast<int32_t>(i);
                std::stable_sort(ord.begin(), ord.end(), [&](int32_t a, int32_t b) {
                    return rpn[a + 1] - rpn[a] > rpn[b + 1] - rpn[b];
                });
                check_cuda(cudaMemcpy(P->order, ord.data(), sizeof(int32_t) * m, cudaMemcpyHostToDevice), "H2D");
            } else {
                P->gmap = dmalloc<uint2>(P->nnz);
            }
            P->mpos = dmalloc<int64_t>(P->nms);
            P->mval = dmalloc<double>(P->nms);
            P->mbeg = dmalloc<int32_t>(P->nms + 1);
            P->mlist = dmalloc<uint2>(P->nmq);
            mcnt = dmalloc<int32_t>(P->nms);
            const int32_t last = static_cast<int32_t>(P->nmq);
            check_cuda(cudaMemcpyAsync(P->mbeg + P->nms, &last, sizeof(last), cudaMemcpyHostToDevice, s), "H2D");
            if (m > 0) {
                ada_fill_kernel<<<grid, kT, smem_fill, s>>>((int)m, A->rp, A->ci, A->val, A->rpT, A->ciT, (int)W,
                                                            wbase, wcount, P->rp, P->msrow ? P->msrow : nms, nmq,
                                                            P->ci, P->diag_pos, P->mpos, mcnt, P->mbeg, P->gmap,
                                                            P->mlist, P->tq, P->smap, P->rmap, P->qbits);
                launched("ada_fill_kernel");
            }
            check_cuda(cudaStreamSynchronize(s), "symbolic sync");
        } catch (...) {
            for (void* p : {(void*)nq, (void*)nms, (void*)nmq, (void*)mcnt, (void*)wbase, (void*)wcount,
                            (void*)wmax_d, (void*)tqa})
                dfree(p);
            free_pattern(P);
            throw;
        }
        for (void* p : {(void*)nq, (void*)nms, (void*)nmq, (void*)mcnt, (void*)wbase, (void*)wcount, (void*)wmax_d,
                        (void*)tqa})
            dfree(p);
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
        cudaStream_t s = as_stream(stream);
        if (P->m == 0) return;
        launch_numeric(P, d, nval, s);
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
