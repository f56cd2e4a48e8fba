// Shared internals of the hn_sm100 library: error plumbing for the C ABI,
// the per-device context, per-stream reduction workspaces and small device
// helpers. Host code here never throws across the C boundary: every exported
// function runs its body through hn::guard(), which maps exceptions to a
// status code plus a thread-local message.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <climits>
#include <cstdio>
#include <mutex>
#include <stdexcept>
#include <string>
#include <unordered_map>

#include "hn_sm100.h"

namespace hn {

// ---------------------------------------------------------------- errors
struct Error : std::runtime_error {
    int status;
    Error(int s, const std::string& m) : std::runtime_error(m), status(s) {}
};

void set_last_error(const std::string& msg);
[[noreturn]] void fail(int status, const std::string& msg);
void check_cuda(cudaError_t e, const char* what);
// Checks the launch that just happened (non-blocking) and counts it.
void launched(const char* what);

// Runs `body`, translating exceptions into status codes. Also implements the
// host-side fault injector (hn_fault_inject) and the API-call counter.
template <class F>
int guard(const char* name, F&& body);

// ---------------------------------------------------------------- context
struct Workspace {
    double* partials = nullptr;    // per-block partial results of reductions
    unsigned* counter = nullptr;   // last-block-done ticket
    double* staging_h = nullptr;   // pinned host staging for *_host calls
    size_t staging_bytes = 0;
    double* staging_d = nullptr;   // device staging for *_host calls
    size_t staging_d_bytes = 0;
    unsigned long long* select = nullptr;  // pricing selection state, kSelectWords words
};
constexpr int kSelectWords = 8;

constexpr int kMaxReduceBlocks = 1184;  // 148 SMs x 8

struct Context {
    int device = -1;
    int sm_count = 0;
    std::mutex mu;
    std::unordered_map<cudaStream_t, Workspace> ws;
    std::atomic<uint64_t> launches{0};
    std::atomic<uint64_t> calls{0};
    std::atomic<int64_t> inject_after{-1};
    std::atomic<int> inject_status{0};
};
Context& ctx();
void require_init();
Workspace& workspace(cudaStream_t s);
// Grows the pinned host + device staging buffers of the stream's workspace.
void ensure_staging(Workspace& w, size_t bytes, cudaStream_t s);

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

template <class T>
T* dmalloc(size_t count) {
    if (count == 0) count = 1;
    void* p = nullptr;
    cudaError_t e = cudaMalloc(&p, count * sizeof(T));
    if (e != cudaSuccess) {
        cudaGetLastError();
        fail(e == cudaErrorMemoryAllocation ? HN_ERR_OUT_OF_MEMORY : HN_ERR_CUDA,
             std::string("cudaMalloc of ") + std::to_string(count * sizeof(T)) +
                 " bytes failed: " + cudaGetErrorString(e));
    }
    return static_cast<T*>(p);
}
inline void dfree(void* p) {
    if (p) cudaFree(p);
}

inline int grid_for(int64_t n, int threads, int cap) {
    int64_t g = (n + threads - 1) / threads;
    if (g < 1) g = 1;
    if (g > cap) g = cap;
    return static_cast<int>(g);
}

// ---------------------------------------------------------------- scans
// Exclusive prefix sums of `n` elements on `s` (in may equal out). Returns
// nothing; the total is out[n-1] + in[n-1] (callers size arrays n+1 and scan
// n+1 entries with a trailing zero to get it in place).
void scan_exclusive_i64(const int64_t* in, int64_t* out, int64_t n, cudaStream_t s);
void scan_exclusive_i32(const int32_t* in, int32_t* out, int64_t n, cudaStream_t s);

// ---------------------------------------------------------------- reductions
// Deterministic reductions into a device double (hn_core.cu).
void reduce_dot(int64_t n, const double* a, const double* b, double* out, cudaStream_t s);
void reduce_nrm2(int64_t n, const double* a, double* out, cudaStream_t s);
void reduce_maxabs(int64_t n, const double* a, double* out, cudaStream_t s);

// Merge-path tile table + carry buffers for a CSR with int32 row pointer rp
// (m rows, nnz nonzeros); allocates the six arrays (hn_csr.cu).
void make_tile_table(const int32_t* rp, int64_t m, int64_t nnz, int64_t* ntiles, int32_t** trow, int32_t** tnz,
                     int32_t** crow, double** cval, int32_t** hrow, double** hval, cudaStream_t s);

// A D A^T numeric without the regularisation step (hn_ada.cu): N's values
// with every diagonal still un-regularised. Used by the batched IPM, which
// regularises each instance's block with its own dyn_reg.
void ada_numeric_unregularised(const hn_pattern* P, const double* d, double* nval, cudaStream_t s);

// ---------------------------------------------------------------- device helpers
__device__ __forceinline__ double ld_stream(const double* p) {
    double v;
    asm volatile("ld.global.nc.L1::no_allocate.f64 %0, [%1];" : "=d"(v) : "l"(p));
    return v;
}
__device__ __forceinline__ int ld_stream(const int* p) {
    int v;
    asm volatile("ld.global.nc.L1::no_allocate.s32 %0, [%1];" : "=r"(v) : "l"(p));
    return v;
}

// Deterministic block sum: fixed shuffle tree inside each warp, then warp 0
// reduces the per-warp values in warp order. `sh` holds >= 32 doubles.
template <int THREADS>
__device__ __forceinline__ double block_sum(double v, double* sh) {
    static_assert(THREADS % 32 == 0 && THREADS <= 1024, "block size");
    constexpr int W = THREADS / 32;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    __syncthreads();
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    double r = 0.0;
    if (wid == 0) {
        r = lane < W ? sh[lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) r += __shfl_down_sync(0xffffffffu, r, o);
    }
    return r;  // valid in thread 0
}

template <int THREADS>
__device__ __forceinline__ double block_max(double v, double* sh) {
    constexpr int W = THREADS / 32;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
    __syncthreads();
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    double r = 0.0;
    if (wid == 0) {
        r = lane < W ? sh[lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) r = fmax(r, __shfl_down_sync(0xffffffffu, r, o));
    }
    return r;
}

template <int THREADS>
__device__ __forceinline__ double block_min(double v, double* sh) {
    constexpr int W = THREADS / 32;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_down_sync(0xffffffffu, v, o));
    __syncthreads();
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    double r = INFINITY;
    if (wid == 0) {
        r = lane < W ? sh[lane] : INFINITY;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) r = fmin(r, __shfl_down_sync(0xffffffffu, r, o));
    }
    return r;
}

template <int THREADS>
__device__ __forceinline__ int64_t block_sum_i64(int64_t v, int64_t* sh) {
    constexpr int W = THREADS / 32;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    __syncthreads();
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    int64_t r = 0;
    if (wid == 0) {
        r = lane < W ? sh[lane] : 0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) r += __shfl_down_sync(0xffffffffu, r, o);
    }
    return r;
}

// Exclusive block scan of one int64 per thread; returns the prefix and
// writes the block total to *total (all threads).
template <int THREADS>
__device__ __forceinline__ int64_t block_exclusive_scan_i64(int64_t v, int64_t* sh,
                                                            int64_t* total) {
    constexpr int W = THREADS / 32;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int64_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int64_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    __syncthreads();
    if (lane == 31) sh[wid] = x;
    __syncthreads();
    if (wid == 0) {
        int64_t w = lane < W ? sh[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int64_t y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < W) sh[lane] = w;  // inclusive warp totals
    }
    __syncthreads();
    const int64_t warp_prefix = wid > 0 ? sh[wid - 1] : 0;
    *total = sh[W - 1];
    return warp_prefix + x - v;
}

// ---------------------------------------------------------------- guard impl
template <class F>
int guard(const char* name, F&& body) {
    Context& c = ctx();
    c.calls.fetch_add(1, std::memory_order_relaxed);
    const int64_t left = c.inject_after.load();
    if (left >= 0) {
        if (left == 0) {
            c.inject_after.store(-1);
            set_last_error(std::string(name) + ": injected failure");
            return c.inject_status.load();
        }
        c.inject_after.store(left - 1);
    }
    try {
        body();
        return HN_OK;
    } catch (const Error& e) {
        set_last_error(std::string(name) + ": " + e.what());
        return e.status;
    } catch (const std::bad_alloc&) {
        set_last_error(std::string(name) + ": host allocation failed");
        return HN_ERR_OUT_OF_MEMORY;
    } catch (const std::exception& e) {
        set_last_error(std::string(name) + ": " + e.what());
        return HN_ERR_INVALID_ARG;
    } catch (...) {
        set_last_error(std::string(name) + ": unknown failure");
        return HN_ERR_INVALID_ARG;
    }
}

}  // namespace hn

// ---------------------------------------------------------------- objects
// Row-length bins of the vector SpMV: bin b holds rows whose group of
// 2^lg[b] lanes takes about `t` nonzeros per lane; perm lists the rows bin by
// bin (ascending within a bin); a warp handles 32 / 2^lg rows of one bin.
constexpr int kSpmvMaxBins = 6;
struct SpmvBins {
    int nbins = 0;
    int unit_off[kSpmvMaxBins + 1] = {};  // first warp of each bin
    int row_off[kSpmvMaxBins + 1] = {};   // first perm entry of each bin
    int lg[kSpmvMaxBins] = {};
};

struct hn_csr {
    int64_t m = 0, n = 0, nnz = 0;
    // A (int32 indices, padded by one slot so empty matrices have storage)
    int32_t* rp = nullptr;
    int32_t* ci = nullptr;
    double* val = nullptr;
    // merge-path tile table and carry buffers for A
    int64_t ntiles = 0;
    int32_t* tile_row = nullptr;
    int32_t* tile_nz = nullptr;
    int32_t* carry_row = nullptr;
    double* carry_val = nullptr;
    int32_t* head_row = nullptr;
    double* head_val = nullptr;
    // A^T
    bool has_t = false;
    int64_t nnz_t = 0;
    int32_t* rpT = nullptr;
    int32_t* ciT = nullptr;
    double* valT = nullptr;
    int32_t* permT = nullptr;  // valT[p] = val[permT[p]] when no entry was merged/dropped
    bool t_compacted = false;  // duplicates merged or zeros dropped
    int64_t ntiles_t = 0;
    int32_t* tile_row_t = nullptr;
    int32_t* tile_nz_t = nullptr;
    int32_t* carry_row_t = nullptr;
    double* carry_val_t = nullptr;
    int32_t* head_row_t = nullptr;
    double* head_val_t = nullptr;
    // SpMV path per direction (0: A, 1: A^T): HN_SPMV_MERGE or HN_SPMV_BINNED
    // (with its target nonzeros per lane, row permutation and bins)
    int spmv_kind[2] = {0, 0};
    int spmv_t[2] = {0, 0};
    int32_t* perm[2] = {nullptr, nullptr};
    SpmvBins bins[2];
};

struct hn_pattern {
    int64_t m = 0, nnz = 0;
    const hn_csr* A = nullptr;
    int64_t* rp = nullptr;       // m+1
    int32_t* ci = nullptr;       // nnz
    int64_t* diag_pos = nullptr; // m
    unsigned long long* maxdiag = nullptr;  // scratch: max diagonal as ordered bits
    // gather map of the numeric phase: for slot t of N, gmap[t] = (p, e) --
    // its single term (A_ij A_kj) d_j comes from A^T entry p and A entry e --
    // or (kMulti | ms, 0) for a slot with several terms, whose (p, e) pairs
    // are mlist[mbeg[ms] .. mbeg[ms+1]) in column order
    int64_t nq = 0;                  // terms in total (sum over columns of count^2)
    uint2* gmap = nullptr;           // nnz
    int64_t nms = 0;                 // slots with several terms (+ every diagonal)
    int64_t* mpos = nullptr;         // nms: N position (bit 62 set for a diagonal)
    int32_t* mbeg = nullptr;         // nms+1
    int64_t nmq = 0;                 // terms into those slots
    uint2* mlist = nullptr;          // nmq
    double2* vd = nullptr;           // nnz(A): (A value, d of its column), per numeric call
    double* mval = nullptr;          // nms: sums of the multi slots, per numeric call
    // row mode (every row of N fits in shared memory): instead of gmap, the
    // terms of row i in enumeration order (A entries e of row i with a
    // nonzero value, then the entries p of A^T row ci[e]) carry their slot
    // offset within the row, or kSlotMulti for a term of a multi slot
    bool row_mode = false;
    int32_t max_row = 0;             // longest row of N (slots)
    int64_t* tq = nullptr;           // m+1: term offsets per row
    uint16_t* smap = nullptr;        // nq
    int64_t* msrow = nullptr;        // m+1: multi-slot offsets per row (row mode and relative map)
    // relative map (rows of N long enough to keep a warp busy): instead of
    // gmap, 4 bytes per slot -- ((e - rp_A[i]) << qbits) | (p - rp_AT[j]) for
    // the single term of A entry e (column j) and A^T entry p, or kMulti |
    // (index of the slot among row i's multi slots); ecs[e] = rp_AT[ci[e]].
    // Rows are handed out longest first (order) from a counter (row_next).
    uint32_t* rmap = nullptr;        // nnz
    int32_t* ecs = nullptr;          // nnz(A)
    int32_t* order = nullptr;        // m
    unsigned* row_next = nullptr;    // 1
    int qbits = 0;
};
