// Device CSR handles: upload + validation, merge-path tile tables (the row
// binning), and the device-built A^T.
//
// A^T is produced by a stable LSD radix sort of the column indices (4-bit
// digits) carrying each entry's CSR position, so entries of equal column keep
// their CSR order -- exactly the order SparseMatrix::transposed() yields
// (sparse_matrix.cpp:84-96 -> from_triplets :8-53 -> sum_duplicates :230-262):
// (column,row) ascending; equal (column,row) keys summed in input order; exact
// zero sums dropped. All of it is integer work except the duplicate sums, so
// the output is bit-identical to the reference.
#include <cstring>
#include <vector>

#include "hn_internal.cuh"
#include "hn_spmv.cuh"

namespace hn {
namespace {

constexpr int kSortThreads = 256;
constexpr int kSortItems = 8;
constexpr int kSortTile = kSortThreads * kSortItems;
constexpr int kRadixBits = 4;
constexpr int kRadix = 1 << kRadixBits;

__global__ void __launch_bounds__(kSortThreads) radix_upsweep(const int32_t* __restrict__ keys,
                                                              int64_t n, int shift,
                                                              int32_t* __restrict__ counts,
                                                              int64_t ntiles) {
    __shared__ int hist[kRadix];
    if (threadIdx.x < kRadix) hist[threadIdx.x] = 0;
    __syncthreads();
    const int64_t base = blockIdx.x * (int64_t)kSortTile + threadIdx.x * kSortItems;
#pragma unroll
    for (int i = 0; i < kSortItems; ++i)
        if (base + i < n) atomicAdd(&hist[(keys[base + i] >> shift) & (kRadix - 1)], 1);
    __syncthreads();
    if (threadIdx.x < kRadix) counts[threadIdx.x * ntiles + blockIdx.x] = hist[threadIdx.x];
}

// Stable scatter of one tile: a key's destination is the global offset of
// (digit, tile) plus the number of same-digit keys before it in the tile.
__global__ void __launch_bounds__(kSortThreads) radix_downsweep(
    const int32_t* __restrict__ kin, const int32_t* __restrict__ vin, int32_t* __restrict__ kout,
    int32_t* __restrict__ vout, int64_t n, int shift, const int32_t* __restrict__ offsets,
    int64_t ntiles) {
    __shared__ int32_t s_cnt[kRadix * kSortThreads];  // digit-major, thread-minor
    __shared__ int64_t s_scan[32];
    const int t = threadIdx.x;
    const int64_t base = blockIdx.x * (int64_t)kSortTile + t * kSortItems;
    int32_t k[kSortItems], v[kSortItems], d[kSortItems], rank[kSortItems];
#pragma unroll
    for (int i = 0; i < kSortItems; ++i) {
        const bool ok = base + i < n;
        k[i] = ok ? kin[base + i] : 0;
        v[i] = ok ? vin[base + i] : 0;
        d[i] = ok ? ((k[i] >> shift) & (kRadix - 1)) : kRadix;  // kRadix = no key
    }
#pragma unroll
    for (int i = 0; i < kSortItems; ++i) {
        int r = 0;
#pragma unroll
        for (int j = 0; j < i; ++j) r += (d[j] == d[i]);
        rank[i] = r;
    }
#pragma unroll
    for (int dg = 0; dg < kRadix; ++dg) {
        int c = 0;
#pragma unroll
        for (int i = 0; i < kSortItems; ++i) c += (d[i] == dg);
        s_cnt[dg * kSortThreads + t] = c;
    }
    __syncthreads();
    // exclusive scan over the kRadix*kSortThreads counters: thread t owns the
    // 16 consecutive counters [16t, 16t+16)
    constexpr int per = kRadix * kSortThreads / kSortThreads;
    int32_t loc[per];
    int64_t sum = 0;
#pragma unroll
    for (int i = 0; i < per; ++i) {
        loc[i] = s_cnt[t * per + i];
        sum += loc[i];
    }
    int64_t total;
    int64_t pre = block_exclusive_scan_i64<kSortThreads>(sum, s_scan, &total);
    __syncthreads();
#pragma unroll
    for (int i = 0; i < per; ++i) {
        s_cnt[t * per + i] = static_cast<int32_t>(pre);
        pre += loc[i];
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < kSortItems; ++i) {
        if (d[i] >= kRadix) continue;
        const int dg = d[i];
        const int64_t local = s_cnt[dg * kSortThreads + t] + rank[i] - s_cnt[dg * kSortThreads];
        const int64_t dst = offsets[dg * ntiles + blockIdx.x] + local;
        kout[dst] = k[i];
        vout[dst] = v[i];
    }
}

__global__ void iota_kernel(int32_t* p, int64_t n) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) p[i] = static_cast<int32_t>(i);
}

// One warp per row writes the row id over the row's nonzeros.
__global__ void row_of_kernel(const int32_t* __restrict__ rp, int64_t m, int32_t* __restrict__ row_of) {
    const int64_t w = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= m) return;
    for (int32_t k = rp[w] + lane; k < rp[w + 1]; k += 32) row_of[k] = static_cast<int32_t>(w);
}

__global__ void gather_t_kernel(int64_t nnz, const int32_t* __restrict__ perm,
                                const int32_t* __restrict__ row_of, const double* __restrict__ val,
                                int32_t* __restrict__ ci_raw, double* __restrict__ val_raw) {
    const int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (p >= nnz) return;
    const int32_t k = perm[p];
    ci_raw[p] = row_of[k];
    val_raw[p] = val[k];
}

// Heads of (column,row) runs sum their run in order; keep = head && sum != 0.
__global__ void runs_kernel(int64_t nnz, const int32_t* __restrict__ key,
                            const int32_t* __restrict__ ci_raw, const double* __restrict__ val_raw,
                            double* __restrict__ run_sum, int32_t* __restrict__ keep) {
    const int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (p >= nnz) return;
    const bool head = (p == 0) || key[p - 1] != key[p] || ci_raw[p - 1] != ci_raw[p];
    if (!head) {
        keep[p] = 0;
        return;
    }
    double s = val_raw[p];
    for (int64_t q = p + 1; q < nnz && key[q] == key[p] && ci_raw[q] == ci_raw[p]; ++q) s += val_raw[q];
    run_sum[p] = s;
    keep[p] = (s != 0.0) ? 1 : 0;
}

__global__ void compact_kernel(int64_t nnz, const int32_t* __restrict__ keep,
                               const int32_t* __restrict__ pos, const int32_t* __restrict__ key,
                               const int32_t* __restrict__ ci_raw, const double* __restrict__ run_sum,
                               int32_t* __restrict__ ciT, double* __restrict__ valT,
                               int32_t* __restrict__ keyT) {
    const int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (p >= nnz || !keep[p]) return;
    const int32_t q = pos[p];
    ciT[q] = ci_raw[p];
    valT[q] = run_sum[p];
    keyT[q] = key[p];
}

__global__ void histogram_kernel(int64_t n, const int32_t* __restrict__ key, int32_t* __restrict__ cnt) {
    const int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (p < n) atomicAdd(&cnt[key[p]], 1);
}

__global__ void sum_i32_kernel(int64_t n, const int32_t* __restrict__ v, unsigned long long* out) {
    __shared__ int64_t sh[32];
    int64_t acc = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        acc += v[i];
    acc = block_sum_i64<256>(acc, sh);
    if (threadIdx.x == 0) atomicAdd(out, static_cast<unsigned long long>(acc));
}

// Merge-path coordinates of diagonals t*items (t = 0..ntiles) over the list
// of m row ends (rp[1..m]) and nnz nonzero indices.
__global__ void tiles_kernel(const int32_t* __restrict__ rp, int64_t m, int64_t nnz, int64_t items,
                             int64_t ntiles, int32_t* __restrict__ tile_row,
                             int32_t* __restrict__ tile_nz) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t > ntiles) return;
    int64_t diag = t * items;
    if (diag > m + nnz) diag = m + nnz;
    int64_t lo = diag - nnz > 0 ? diag - nnz : 0;
    int64_t hi = diag < m ? diag : m;
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if ((int64_t)rp[mid + 1] <= diag - mid - 1)
            lo = mid + 1;
        else
            hi = mid;
    }
    tile_row[t] = static_cast<int32_t>(lo);
    tile_nz[t] = static_cast<int32_t>(diag - lo);
}

inline unsigned blocks(int64_t n, int t = 256) { return static_cast<unsigned>((n + t - 1) / t); }

void build_tiles(const int32_t* rp, int64_t m, int64_t nnz, int64_t& ntiles, int32_t*& trow,
                 int32_t*& tnz, int32_t*& crow, double*& cval, int32_t*& hrow, double*& hval,
                 cudaStream_t s) {
    ntiles = (m + nnz + kSpmvTile - 1) / kSpmvTile;
    trow = dmalloc<int32_t>(ntiles + 1);
    tnz = dmalloc<int32_t>(ntiles + 1);
    crow = dmalloc<int32_t>(ntiles);
    cval = dmalloc<double>(ntiles);
    hrow = dmalloc<int32_t>(ntiles);
    hval = dmalloc<double>(ntiles);
    tiles_kernel<<<blocks(ntiles + 1), 256, 0, s>>>(rp, m, nnz, kSpmvTile, ntiles, trow, tnz);
    launched("tiles_kernel");
}

void free_transpose(hn_csr* A) {
    dfree(A->rpT);
    dfree(A->ciT);
    dfree(A->valT);
    dfree(A->permT);
    dfree(A->tile_row_t);
    dfree(A->tile_nz_t);
    dfree(A->carry_row_t);
    dfree(A->carry_val_t);
    dfree(A->head_row_t);
    dfree(A->head_val_t);
    A->rpT = A->ciT = A->permT = A->tile_row_t = A->tile_nz_t = A->carry_row_t = A->head_row_t =
        nullptr;
    A->valT = A->carry_val_t = A->head_val_t = nullptr;
    A->has_t = false;
    dfree(A->perm[1]);
    A->perm[1] = nullptr;
}

// Stable LSD radix sort of nnz (key, value) pairs on the keys' low bits
// (keys in [0, range)); kA/vA hold the result, kB/vB are scratch.
void radix_sort_pairs(int32_t*& kA, int32_t*& vA, int32_t*& kB, int32_t*& vB, int64_t nnz, int64_t range,
                      cudaStream_t s) {
    int bits = 0;
    while (bits < 31 && (int64_t(1) << bits) < range) ++bits;
    const int64_t ntiles = (nnz + kSortTile - 1) / kSortTile;
    if (nnz == 0 || bits == 0) return;
    int32_t* counts = dmalloc<int32_t>(kRadix * ntiles);
    for (int shift = 0; shift < bits; shift += kRadixBits) {
        radix_upsweep<<<(unsigned)ntiles, kSortThreads, 0, s>>>(kA, nnz, shift, counts, ntiles);
        launched("radix_upsweep");
        scan_exclusive_i32(counts, counts, kRadix * ntiles, s);
        radix_downsweep<<<(unsigned)ntiles, kSortThreads, 0, s>>>(kA, vA, kB, vB, nnz, shift, counts, ntiles);
        launched("radix_downsweep");
        std::swap(kA, kB);
        std::swap(vA, vB);
    }
    check_cuda(cudaStreamSynchronize(s), "radix sort sync");
    dfree(counts);
}

__global__ void gather_i32_kernel(int64_t nnz, const int32_t* __restrict__ perm, const int32_t* __restrict__ src,
                                  int32_t* __restrict__ dst) {
    const int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (p < nnz) dst[p] = src[perm[p]];
}

void build_transpose(hn_csr* A, cudaStream_t s) {
    const int64_t nnz = A->nnz, m = A->m, n = A->n;
    A->rpT = dmalloc<int32_t>(n + 1);
    int32_t* kA = dmalloc<int32_t>(nnz);
    int32_t* kB = dmalloc<int32_t>(nnz);
    int32_t* vA = dmalloc<int32_t>(nnz);
    int32_t* vB = dmalloc<int32_t>(nnz);
    check_cuda(cudaMemcpyAsync(kA, A->ci, sizeof(int32_t) * nnz, cudaMemcpyDeviceToDevice, s), "copy keys");
    if (nnz > 0) {
        iota_kernel<<<blocks(nnz), 256, 0, s>>>(vA, nnz);
        launched("iota_kernel");
    }
    radix_sort_pairs(kA, vA, kB, vB, nnz, n, s);
    // kA: sorted column keys, vA: CSR position of each sorted entry
    int32_t* row_of = dmalloc<int32_t>(nnz);
    if (m > 0 && nnz > 0) {
        row_of_kernel<<<blocks(m * 32), 256, 0, s>>>(A->rp, m, row_of);
        launched("row_of_kernel");
    }
    int32_t* ci_raw = kB;  // reuse
    double* val_raw = dmalloc<double>(nnz);
    double* run_sum = dmalloc<double>(nnz);
    int32_t* keep = vB;  // reuse
    unsigned long long* kept_d = dmalloc<unsigned long long>(1);
    unsigned long long kept = 0;
    if (nnz > 0) {
        gather_t_kernel<<<blocks(nnz), 256, 0, s>>>(nnz, vA, row_of, A->val, ci_raw, val_raw);
        launched("gather_t_kernel");
        runs_kernel<<<blocks(nnz), 256, 0, s>>>(nnz, kA, ci_raw, val_raw, run_sum, keep);
        launched("runs_kernel");
        check_cuda(cudaMemsetAsync(kept_d, 0, sizeof(unsigned long long), s), "memset");
        sum_i32_kernel<<<grid_for(nnz, 256, 1024), 256, 0, s>>>(nnz, keep, kept_d);
        launched("sum_i32_kernel");
        check_cuda(cudaMemcpyAsync(&kept, kept_d, sizeof(kept), cudaMemcpyDeviceToHost, s), "D2H kept");
        check_cuda(cudaStreamSynchronize(s), "transpose sync");
    }
    int32_t* cnt = dmalloc<int32_t>(n + 1);
    check_cuda(cudaMemsetAsync(cnt, 0, sizeof(int32_t) * (n + 1), s), "memset cnt");
    if (static_cast<int64_t>(kept) == nnz) {
        // nothing merged or dropped: the permutation carries values directly
        A->nnz_t = nnz;
        A->ciT = ci_raw;
        A->valT = val_raw;
        A->permT = vA;
        A->t_compacted = false;
        if (nnz > 0) {
            histogram_kernel<<<blocks(nnz), 256, 0, s>>>(nnz, kA, cnt);
            launched("histogram_kernel");
        }
        dfree(run_sum);
        dfree(keep);
        dfree(kA);
    } else {
        int32_t* pos = dmalloc<int32_t>(nnz);
        scan_exclusive_i32(keep, pos, nnz, s);
        A->nnz_t = static_cast<int64_t>(kept);
        A->ciT = dmalloc<int32_t>(A->nnz_t);
        A->valT = dmalloc<double>(A->nnz_t);
        int32_t* keyT = dmalloc<int32_t>(A->nnz_t);
        compact_kernel<<<blocks(nnz), 256, 0, s>>>(nnz, keep, pos, kA, ci_raw, run_sum, A->ciT, A->valT,
                                                   keyT);
        launched("compact_kernel");
        if (A->nnz_t > 0) {
            histogram_kernel<<<blocks(A->nnz_t), 256, 0, s>>>(A->nnz_t, keyT, cnt);
            launched("histogram_kernel");
        }
        check_cuda(cudaStreamSynchronize(s), "transpose sync");
        A->permT = nullptr;
        A->t_compacted = true;
        dfree(pos);
        dfree(keyT);
        dfree(ci_raw);
        dfree(val_raw);
        dfree(run_sum);
        dfree(keep);
        dfree(kA);
        dfree(vA);
    }
    scan_exclusive_i32(cnt, A->rpT, n + 1, s);
    check_cuda(cudaStreamSynchronize(s), "transpose sync");
    dfree(cnt);
    dfree(row_of);
    dfree(kept_d);
    build_tiles(A->rpT, n, A->nnz_t, A->ntiles_t, A->tile_row_t, A->tile_nz_t, A->carry_row_t,
                A->carry_val_t, A->head_row_t, A->head_val_t, s);
    check_cuda(cudaStreamSynchronize(s), "tiles sync");
    A->has_t = true;
}

void free_csr(hn_csr* A) {
    if (!A) return;
    free_transpose(A);
    dfree(A->perm[0]);
    dfree(A->rp);
    dfree(A->ci);
    dfree(A->val);
    dfree(A->tile_row);
    dfree(A->tile_nz);
    dfree(A->carry_row);
    dfree(A->carry_val);
    dfree(A->head_row);
    dfree(A->head_val);
    delete A;
}

// Host-side validation + int32 conversion. Every index the kernels will use
// is checked here, so no launch can read out of bounds.
// ---- SpMV path choice ----

// Bins of the vector kernel for a target of t nonzeros per lane: a row of
// length L gets the smallest group G = 2^lg (lg <= 5) with G * t >= L.
void make_bins(const std::vector<int32_t>& rp, int t, std::vector<int32_t>& perm, SpmvBins& b) {
    const int64_t rows = static_cast<int64_t>(rp.size()) - 1;
    std::vector<int8_t> lg(rows);
    int64_t cnt[kSpmvMaxBins] = {};
    for (int64_t i = 0; i < rows; ++i) {
        const int64_t L = rp[i + 1] - rp[i], q = (L + t - 1) / t;
        int g = 0;
        while ((int64_t(1) << g) < q && g < kSpmvMaxBins - 1) ++g;
        lg[i] = static_cast<int8_t>(g);
        ++cnt[g];
    }
    perm.clear();
    perm.reserve(rows);
    b = SpmvBins{};
    int64_t uo = 0, ro = 0;
    int nb = 0;
    for (int g = 0; g < kSpmvMaxBins; ++g) {
        if (!cnt[g]) continue;
        b.lg[nb] = g;
        b.unit_off[nb] = static_cast<int>(uo);
        b.row_off[nb] = static_cast<int>(ro);
        for (int64_t i = 0; i < rows; ++i)
            if (lg[i] == g) perm.push_back(static_cast<int32_t>(i));
        const int64_t rpw = 32 >> g;
        uo += (cnt[g] + rpw - 1) / rpw;
        ro += cnt[g];
        ++nb;
    }
    if (uo * 32 >= INT32_MAX) fail(HN_ERR_UNSUPPORTED, "too many rows for the vector SpMV");
    b.nbins = nb;
    b.unit_off[nb] = static_cast<int>(uo);
    b.row_off[nb] = static_cast<int>(ro);
}

std::vector<int32_t> host_rows(const hn_csr* A, int d) {
    const int64_t rows = d ? A->n : A->m;
    std::vector<int32_t> rp(rows + 1);
    check_cuda(cudaMemcpy(rp.data(), d ? A->rpT : A->rp, sizeof(int32_t) * (rows + 1), cudaMemcpyDeviceToHost),
               "D2H rp");
    return rp;
}

void set_spmv_path(hn_csr* A, int d, int kind, int t) {
    dfree(A->perm[d]);
    A->perm[d] = nullptr;
    A->spmv_kind[d] = HN_SPMV_MERGE;
    A->spmv_t[d] = 0;
    if (kind != HN_SPMV_BINNED) return;
    std::vector<int32_t> perm;
    SpmvBins b;
    make_bins(host_rows(A, d), t, perm, b);
    A->perm[d] = dmalloc<int32_t>(perm.size());
    if (!perm.empty())
        check_cuda(cudaMemcpy(A->perm[d], perm.data(), sizeof(int32_t) * perm.size(), cudaMemcpyHostToDevice),
                   "H2D perm");
    A->bins[d] = b;
    A->spmv_kind[d] = HN_SPMV_BINNED;
    A->spmv_t[d] = t;
}

// The autotuner: for each direction, times the merge-path kernel and the
// binned vector kernel at t = 4, 8, 16 nonzeros per lane (three launches
// each after one warm-up, best of three, CUDA events) and keeps the binned
// kernel only when it is at least 5 % faster, so close calls stay on the
// merge path. Small matrices (< 2^20 nonzeros) keep the merge path untimed.
constexpr int64_t kAutotuneMinNnz = int64_t(1) << 20;
void autotune(hn_csr* A, cudaStream_t s) {
    for (int d = 0; d < (A->has_t ? 2 : 1); ++d) {
        const int64_t rows = d ? A->n : A->m, cols = d ? A->m : A->n;
        if ((d ? A->nnz_t : A->nnz) < kAutotuneMinNnz) continue;
        double* x = dmalloc<double>(cols);
        double* y = dmalloc<double>(rows);
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        try {
            check_cuda(cudaMemsetAsync(x, 0, sizeof(double) * cols, s), "memset");
            check_cuda(cudaEventCreate(&e0), "event");
            check_cuda(cudaEventCreate(&e1), "event");
            auto time_path = [&]() {
                const SpmvMat M = spmv_mat(A, d);
                spmv_launch(M, x, EpiAxpby{1.0, 0.0, y}, s);
                float best = 1e30f;
                for (int rep = 0; rep < 3; ++rep) {
                    check_cuda(cudaEventRecord(e0, s), "event");
                    spmv_launch(M, x, EpiAxpby{1.0, 0.0, y}, s);
                    check_cuda(cudaEventRecord(e1, s), "event");
                    check_cuda(cudaEventSynchronize(e1), "event sync");
                    float ms = 0.f;
                    check_cuda(cudaEventElapsedTime(&ms, e0, e1), "event time");
                    best = std::min(best, ms);
                }
                return best;
            };
            float best = time_path();
            int best_t = 0;
            for (int t : {4, 8, 16}) {
                set_spmv_path(A, d, HN_SPMV_BINNED, t);
                const float ms = time_path();
                if (ms < 0.95f * best) {
                    best = ms;
                    best_t = t;
                }
            }
            set_spmv_path(A, d, best_t ? HN_SPMV_BINNED : HN_SPMV_MERGE, best_t);
        } catch (...) {
            if (e0) cudaEventDestroy(e0);
            if (e1) cudaEventDestroy(e1);
            dfree(x);
            dfree(y);
            throw;
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        dfree(x);
        dfree(y);
    }
}

void convert_csr(int64_t m, int64_t n, const uint64_t* rp, const uint64_t* ci,
                 std::vector<int32_t>& rp32, std::vector<int32_t>& ci32) {
    if (m < 0 || n < 0) fail(HN_ERR_INVALID_ARG, "negative dimension");
    if (m >= INT32_MAX || n >= INT32_MAX) fail(HN_ERR_UNSUPPORTED, "dimension exceeds int32 range");
    if (!rp) fail(HN_ERR_INVALID_ARG, "null row_ptr");
    if (rp[0] != 0) fail(HN_ERR_INVALID_ARG, "row_ptr[0] must be 0");
    const uint64_t nnz = rp[m];
    if (nnz >= static_cast<uint64_t>(INT32_MAX) || static_cast<uint64_t>(m) + nnz >= (uint64_t)INT32_MAX)
        fail(HN_ERR_UNSUPPORTED, "nnz (+m) exceeds int32 range");
    if (nnz > 0 && !ci) fail(HN_ERR_INVALID_ARG, "null col_idx");
    rp32.resize(static_cast<size_t>(m) + 1);
    for (int64_t i = 0; i <= m; ++i) {
        if (i > 0 && rp[i] < rp[i - 1]) fail(HN_ERR_INVALID_ARG, "row_ptr is not non-decreasing");
        rp32[i] = static_cast<int32_t>(rp[i]);
    }
    ci32.resize(static_cast<size_t>(nnz));
    for (uint64_t k = 0; k < nnz; ++k) {
        if (ci[k] >= static_cast<uint64_t>(n))
            fail(HN_ERR_INVALID_ARG, "col_idx[" + std::to_string(k) + "] = " + std::to_string(ci[k]) +
                                         " out of range for " + std::to_string(n) + " columns");
        ci32[k] = static_cast<int32_t>(ci[k]);
    }
}

// CSR (device rp, ci, val) of m x n from nnz triplets already on the device
// (rows r, columns c, values v), with SparseMatrix::from_triplets semantics:
// entries ordered by (row, column), equal (row, column) entries summed in
// input order, exact-zero sums dropped. Two stable radix passes (columns,
// then rows) carry each entry's input position.
void coo_to_csr(int64_t m, int64_t n, int64_t nnz, const int32_t* r, const int32_t* c, const double* v,
                int32_t** rp_out, int32_t** ci_out, double** val_out, int64_t* nnz_out, cudaStream_t s) {
    int32_t* kA = dmalloc<int32_t>(nnz);
    int32_t* kB = dmalloc<int32_t>(nnz);
    int32_t* vA = dmalloc<int32_t>(nnz);
    int32_t* vB = dmalloc<int32_t>(nnz);
    if (nnz > 0) {
        check_cuda(cudaMemcpyAsync(kA, c, sizeof(int32_t) * nnz, cudaMemcpyDeviceToDevice, s), "copy keys");
        iota_kernel<<<blocks(nnz), 256, 0, s>>>(vA, nnz);
        launched("iota_kernel");
    }
    radix_sort_pairs(kA, vA, kB, vB, nnz, n, s);  // by column
    if (nnz > 0) {
        gather_i32_kernel<<<blocks(nnz), 256, 0, s>>>(nnz, vA, r, kA);
        launched("gather_i32_kernel");
    }
    radix_sort_pairs(kA, vA, kB, vB, nnz, m, s);  // then by row (stable)
    // kA: rows in (row, column) order, vA: input position of each entry
    int32_t* ci_raw = kB;  // reuse
    int32_t* keep = vB;    // reuse
    double* val_raw = dmalloc<double>(nnz);
    double* run_sum = dmalloc<double>(nnz);
    unsigned long long* kept_d = dmalloc<unsigned long long>(1);
    unsigned long long kept = 0;
    if (nnz > 0) {
        gather_t_kernel<<<blocks(nnz), 256, 0, s>>>(nnz, vA, c, v, ci_raw, val_raw);
        launched("gather_t_kernel");
        runs_kernel<<<blocks(nnz), 256, 0, s>>>(nnz, kA, ci_raw, val_raw, run_sum, keep);
        launched("runs_kernel");
        check_cuda(cudaMemsetAsync(kept_d, 0, sizeof(unsigned long long), s), "memset");
        sum_i32_kernel<<<grid_for(nnz, 256, 1024), 256, 0, s>>>(nnz, keep, kept_d);
        launched("sum_i32_kernel");
        check_cuda(cudaMemcpyAsync(&kept, kept_d, sizeof(kept), cudaMemcpyDeviceToHost, s), "D2H kept");
        check_cuda(cudaStreamSynchronize(s), "coo sync");
    }
    const int64_t nk = static_cast<int64_t>(kept);
    int32_t* pos = dmalloc<int32_t>(nnz);
    int32_t* ci = dmalloc<int32_t>(nk);
    double* val = dmalloc<double>(nk);
    int32_t* key = dmalloc<int32_t>(nk);
    int32_t* cnt = dmalloc<int32_t>(m + 1);
    check_cuda(cudaMemsetAsync(cnt, 0, sizeof(int32_t) * (m + 1), s), "memset cnt");
    if (nnz > 0) {
        scan_exclusive_i32(keep, pos, nnz, s);
        compact_kernel<<<blocks(nnz), 256, 0, s>>>(nnz, keep, pos, kA, ci_raw, run_sum, ci, val, key);
        launched("compact_kernel");
    }
    if (nk > 0) {
        histogram_kernel<<<blocks(nk), 256, 0, s>>>(nk, key, cnt);
        launched("histogram_kernel");
    }
    int32_t* rp = dmalloc<int32_t>(m + 1);
    scan_exclusive_i32(cnt, rp, m + 1, s);
    check_cuda(cudaStreamSynchronize(s), "coo sync");
    for (void* p : {(void*)kA, (void*)kB, (void*)vA, (void*)vB, (void*)val_raw, (void*)run_sum, (void*)kept_d,
                    (void*)pos, (void*)key, (void*)cnt})
        dfree(p);
    *rp_out = rp;
    *ci_out = ci;
    *val_out = val;
    *nnz_out = nk;
}

}  // namespace

void make_tile_table(const int32_t* rp, int64_t m, int64_t nnz, int64_t* ntiles, int32_t** trow, int32_t** tnz,
                     int32_t** crow, double** cval, int32_t** hrow, double** hval, cudaStream_t s) {
    build_tiles(rp, m, nnz, *ntiles, *trow, *tnz, *crow, *cval, *hrow, *hval, s);
}

}  // namespace hn

using namespace hn;

extern "C" {

int hn_csr_create(int64_t m, int64_t n, const uint64_t* rp, const uint64_t* ci, const double* val,
                  unsigned flags, hn_csr** out) {
    return guard("hn_csr_create", [&] {
        require_init();
        if (!out) fail(HN_ERR_INVALID_ARG, "null output handle");
        *out = nullptr;
        std::vector<int32_t> rp32, ci32;
        convert_csr(m, n, rp, ci, rp32, ci32);
        const int64_t nnz = static_cast<int64_t>(ci32.size());
        if (nnz > 0 && !val) fail(HN_ERR_INVALID_ARG, "null values");
        cudaStream_t s = nullptr;
        hn_csr* A = new hn_csr();
        try {
            A->m = m;
            A->n = n;
            A->nnz = nnz;
            A->rp = dmalloc<int32_t>(m + 1);
            A->ci = dmalloc<int32_t>(nnz);
            A->val = dmalloc<double>(nnz);
            check_cuda(cudaMemcpy(A->rp, rp32.data(), sizeof(int32_t) * (m + 1), cudaMemcpyHostToDevice),
                       "H2D row_ptr");
            if (nnz > 0) {
                check_cuda(cudaMemcpy(A->ci, ci32.data(), sizeof(int32_t) * nnz, cudaMemcpyHostToDevice),
                           "H2D col_idx");
                check_cuda(cudaMemcpy(A->val, val, sizeof(double) * nnz, cudaMemcpyHostToDevice),
                           "H2D values");
            }
            build_tiles(A->rp, m, nnz, A->ntiles, A->tile_row, A->tile_nz, A->carry_row, A->carry_val,
                        A->head_row, A->head_val, s);
            if (!(flags & HN_CSR_NO_TRANSPOSE)) build_transpose(A, s);
            check_cuda(cudaStreamSynchronize(s), "hn_csr_create sync");
            if (!(flags & HN_CSR_NO_AUTOTUNE)) autotune(A, s);
        } catch (...) {
            free_csr(A);
            throw;
        }
        *out = A;
    });
}

int hn_csr_create_coo(int64_t m, int64_t n, int64_t count, const int64_t* rows, const int64_t* cols,
                      const double* val, unsigned flags, hn_csr** out) {
    return guard("hn_csr_create_coo", [&] {
        require_init();
        if (!out) fail(HN_ERR_INVALID_ARG, "null output handle");
        *out = nullptr;
        if (m < 0 || n < 0 || count < 0) fail(HN_ERR_INVALID_ARG, "negative dimension or count");
        if (m >= INT32_MAX || n >= INT32_MAX || count >= INT32_MAX || m + count >= INT32_MAX)
            fail(HN_ERR_UNSUPPORTED, "dimension or count exceeds int32 range");
        if (count > 0 && (!rows || !cols || !val)) fail(HN_ERR_INVALID_ARG, "null triplet arrays");
        std::vector<int32_t> r32(static_cast<size_t>(count)), c32(static_cast<size_t>(count));
        for (int64_t k = 0; k < count; ++k) {
            if (rows[k] < 0 || rows[k] >= m || cols[k] < 0 || cols[k] >= n)
                fail(HN_ERR_INVALID_ARG, "triplet " + std::to_string(k) + " (" + std::to_string(rows[k]) + ", " +
                                             std::to_string(cols[k]) + ") outside " + std::to_string(m) + " x " +
                                             std::to_string(n));
            r32[k] = static_cast<int32_t>(rows[k]);
            c32[k] = static_cast<int32_t>(cols[k]);
        }
        cudaStream_t s = nullptr;
        int32_t* dr = nullptr;
        int32_t* dc = nullptr;
        double* dv = nullptr;
        hn_csr* A = new hn_csr();
        try {
            dr = dmalloc<int32_t>(count);
            dc = dmalloc<int32_t>(count);
            dv = dmalloc<double>(count);
            if (count > 0) {
                check_cuda(cudaMemcpy(dr, r32.data(), sizeof(int32_t) * count, cudaMemcpyHostToDevice), "H2D rows");
                check_cuda(cudaMemcpy(dc, c32.data(), sizeof(int32_t) * count, cudaMemcpyHostToDevice), "H2D cols");
                check_cuda(cudaMemcpy(dv, val, sizeof(double) * count, cudaMemcpyHostToDevice), "H2D values");
            }
            A->m = m;
            A->n = n;
            coo_to_csr(m, n, count, dr, dc, dv, &A->rp, &A->ci, &A->val, &A->nnz, s);
            dfree(dr);
            dfree(dc);
            dfree(dv);
            dr = dc = nullptr;
            dv = nullptr;
            build_tiles(A->rp, m, A->nnz, A->ntiles, A->tile_row, A->tile_nz, A->carry_row, A->carry_val,
                        A->head_row, A->head_val, s);
            if (!(flags & HN_CSR_NO_TRANSPOSE)) build_transpose(A, s);
            check_cuda(cudaStreamSynchronize(s), "hn_csr_create_coo sync");
            if (!(flags & HN_CSR_NO_AUTOTUNE)) autotune(A, s);
        } catch (...) {
            dfree(dr);
            dfree(dc);
            dfree(dv);
            free_csr(A);
            throw;
        }
        *out = A;
    });
}

int hn_csr_set_values(hn_csr* A, const double* val) {
    return guard("hn_csr_set_values", [&] {
        require_init();
        if (!A || (A->nnz > 0 && !val)) fail(HN_ERR_INVALID_ARG, "bad arguments");
        check_cuda(cudaDeviceSynchronize(), "sync before value update");
        if (A->nnz > 0)
            check_cuda(cudaMemcpy(A->val, val, sizeof(double) * A->nnz, cudaMemcpyHostToDevice),
                       "H2D values");
        if (A->has_t) {
            // exact-zero dropping depends on the values: rebuild A^T (and its bins)
            const int kind = A->spmv_kind[1], t = A->spmv_t[1];
            free_transpose(A);
            build_transpose(A, nullptr);
            set_spmv_path(A, 1, kind, t);
        }
    });
}

int hn_csr_destroy(hn_csr* A) {
    return guard("hn_csr_destroy", [&] {
        if (!A) return;
        require_init();
        cudaDeviceSynchronize();
        free_csr(A);
    });
}

int hn_csr_shape(const hn_csr* A, int64_t* m, int64_t* n, int64_t* nnz, int64_t* nnz_t) {
    return guard("hn_csr_shape", [&] {
        if (!A) fail(HN_ERR_INVALID_ARG, "null handle");
        if (m) *m = A->m;
        if (n) *n = A->n;
        if (nnz) *nnz = A->nnz;
        if (nnz_t) *nnz_t = A->has_t ? A->nnz_t : -1;
    });
}

int hn_csr_export(const hn_csr* A, int trans, uint64_t* rp, uint64_t* ci, double* val) {
    return guard("hn_csr_export", [&] {
        require_init();
        if (!A) fail(HN_ERR_INVALID_ARG, "null handle");
        if (trans && !A->has_t) fail(HN_ERR_INVALID_ARG, "handle was created without A^T");
        const int64_t rows = trans ? A->n : A->m;
        const int64_t nnz = trans ? A->nnz_t : A->nnz;
        std::vector<int32_t> r(rows + 1), c(nnz);
        check_cuda(cudaMemcpy(r.data(), trans ? A->rpT : A->rp, sizeof(int32_t) * (rows + 1),
                              cudaMemcpyDeviceToHost),
                   "D2H rp");
        if (nnz > 0) {
            check_cuda(cudaMemcpy(c.data(), trans ? A->ciT : A->ci, sizeof(int32_t) * nnz,
                                  cudaMemcpyDeviceToHost),
                       "D2H ci");
            if (val)
                check_cuda(cudaMemcpy(val, trans ? A->valT : A->val, sizeof(double) * nnz,
                                      cudaMemcpyDeviceToHost),
                           "D2H val");
        }
        if (rp)
            for (int64_t i = 0; i <= rows; ++i) rp[i] = static_cast<uint64_t>(r[i]);
        if (ci)
            for (int64_t k = 0; k < nnz; ++k) ci[k] = static_cast<uint64_t>(c[k]);
    });
}

int hn_csr_spmv_kind(const hn_csr* A, int trans, int* kind, int* t) {
    return guard("hn_csr_spmv_kind", [&] {
        if (!A) fail(HN_ERR_INVALID_ARG, "null handle");
        if (trans && !A->has_t) fail(HN_ERR_INVALID_ARG, "handle was created without A^T");
        const int d = trans ? 1 : 0;
        if (kind) *kind = A->spmv_kind[d];
        if (t) *t = A->spmv_t[d];
    });
}

int hn_csr_set_spmv_kind(hn_csr* A, int trans, int kind, int t) {
    return guard("hn_csr_set_spmv_kind", [&] {
        require_init();
        if (!A) fail(HN_ERR_INVALID_ARG, "null handle");
        if (trans && !A->has_t) fail(HN_ERR_INVALID_ARG, "handle was created without A^T");
        if (kind != HN_SPMV_MERGE && kind != HN_SPMV_BINNED) fail(HN_ERR_INVALID_ARG, "unknown SpMV kind");
        if (kind == HN_SPMV_BINNED && (t < 1 || t > 64)) fail(HN_ERR_INVALID_ARG, "t must be in [1, 64]");
        check_cuda(cudaDeviceSynchronize(), "sync before changing the SpMV path");
        set_spmv_path(A, trans ? 1 : 0, kind, t);
    });
}

int hn_csr_tiles(const hn_csr* A, int trans, int64_t* ntiles, int64_t* items) {
    return guard("hn_csr_tiles", [&] {
        if (!A) fail(HN_ERR_INVALID_ARG, "null handle");
        if (trans && !A->has_t) fail(HN_ERR_INVALID_ARG, "handle was created without A^T");
        if (ntiles) *ntiles = trans ? A->ntiles_t : A->ntiles;
        if (items) *items = kSpmvTile;
    });
}

int hn_csr_export_tiles(const hn_csr* A, int trans, int32_t* trow, int32_t* tnz) {
    return guard("hn_csr_export_tiles", [&] {
        require_init();
        if (!A || !trow || !tnz) fail(HN_ERR_INVALID_ARG, "bad arguments");
        if (trans && !A->has_t) fail(HN_ERR_INVALID_ARG, "handle was created without A^T");
        const int64_t nt = trans ? A->ntiles_t : A->ntiles;
        check_cuda(cudaMemcpy(trow, trans ? A->tile_row_t : A->tile_row, sizeof(int32_t) * (nt + 1),
                              cudaMemcpyDeviceToHost),
                   "D2H tiles");
        check_cuda(cudaMemcpy(tnz, trans ? A->tile_nz_t : A->tile_nz, sizeof(int32_t) * (nt + 1),
                              cudaMemcpyDeviceToHost),
                   "D2H tiles");
    });
}

}  // extern "C"
