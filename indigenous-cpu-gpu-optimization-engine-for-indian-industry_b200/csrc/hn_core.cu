// Context, error plumbing, device-memory helpers, scans and BLAS-1 kernels.
#include "hn_internal.cuh"

#include <cstring>
#include <vector>

namespace hn {

namespace {
thread_local std::string g_last_error;
Context g_ctx;
}  // namespace

void set_last_error(const std::string& msg) { g_last_error = msg; }

void fail(int status, const std::string& msg) { throw Error(status, msg); }

void check_cuda(cudaError_t e, const char* what) {
    if (e != cudaSuccess) {
        cudaGetLastError();
        fail(e == cudaErrorMemoryAllocation ? HN_ERR_OUT_OF_MEMORY : HN_ERR_CUDA,
             std::string(what) + ": " + cudaGetErrorString(e));
    }
}

void launched(const char* what) {
    g_ctx.launches.fetch_add(1, std::memory_order_relaxed);
    check_cuda(cudaGetLastError(), what);
}

Context& ctx() { return g_ctx; }

void require_init() {
    if (g_ctx.device < 0) fail(HN_ERR_NOT_INITIALIZED, "hn_init has not been called");
    int cur = -1;
    check_cuda(cudaGetDevice(&cur), "cudaGetDevice");
    if (cur != g_ctx.device) check_cuda(cudaSetDevice(g_ctx.device), "cudaSetDevice");
}

Workspace& workspace(cudaStream_t s) {
    std::lock_guard<std::mutex> lk(g_ctx.mu);
    auto it = g_ctx.ws.find(s);
    if (it != g_ctx.ws.end()) return it->second;
    Workspace w;
    w.partials = dmalloc<double>(4 * kMaxReduceBlocks + 8);
    w.counter = dmalloc<unsigned>(4);
    w.select = dmalloc<unsigned long long>(kSelectWords);
    check_cuda(cudaMemsetAsync(w.counter, 0, 4 * sizeof(unsigned), s), "workspace init");
    check_cuda(cudaMemsetAsync(w.select, 0, kSelectWords * sizeof(unsigned long long), s), "workspace init");
    check_cuda(cudaStreamSynchronize(s), "workspace init sync");
    return g_ctx.ws.emplace(s, w).first->second;
}

void ensure_staging(Workspace& w, size_t bytes, cudaStream_t s) {
    if (w.staging_bytes < bytes) {
        check_cuda(cudaStreamSynchronize(s), "staging sync");
        if (w.staging_h) cudaFreeHost(w.staging_h);
        w.staging_h = nullptr;
        w.staging_bytes = 0;
        check_cuda(cudaMallocHost(reinterpret_cast<void**>(&w.staging_h), bytes),
                   "cudaMallocHost staging");
        w.staging_bytes = bytes;
    }
    if (w.staging_d_bytes < bytes) {
        check_cuda(cudaStreamSynchronize(s), "staging sync");
        dfree(w.staging_d);
        w.staging_d = nullptr;
        w.staging_d_bytes = 0;
        w.staging_d = dmalloc<double>((bytes + 7) / 8);
        w.staging_d_bytes = bytes;
    }
}

// ---------------------------------------------------------------- scans
namespace {
constexpr int kScanThreads = 512;
constexpr int kScanItems = 8;
constexpr int64_t kScanTile = kScanThreads * kScanItems;

template <class T>
__global__ void __launch_bounds__(kScanThreads) scan_tile_kernel(const T* in, T* out, int64_t n,
                                                                  int64_t* tile_sums) {
    __shared__ int64_t sh[32];
    const int64_t base = blockIdx.x * kScanTile + threadIdx.x * kScanItems;
    int64_t v[kScanItems];
    int64_t s = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        v[i] = (base + i < n) ? static_cast<int64_t>(in[base + i]) : 0;
        s += v[i];
    }
    int64_t total;
    int64_t pre = block_exclusive_scan_i64<kScanThreads>(s, sh, &total);
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        if (base + i < n) out[base + i] = static_cast<T>(pre);
        pre += v[i];
    }
    if (threadIdx.x == 0 && tile_sums) tile_sums[blockIdx.x] = total;
}

template <class T>
__global__ void scan_add_kernel(T* out, int64_t n, const int64_t* tile_offsets) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) out[i] += static_cast<T>(tile_offsets[i / kScanTile]);
}

template <class T>
void scan_exclusive_impl(const T* in, T* out, int64_t n, cudaStream_t s) {
    if (n <= 0) return;
    const int64_t tiles = (n + kScanTile - 1) / kScanTile;
    if (tiles == 1) {
        scan_tile_kernel<T><<<1, kScanThreads, 0, s>>>(in, out, n, nullptr);
        launched("scan_tile_kernel");
        return;
    }
    int64_t* sums = dmalloc<int64_t>(tiles);
    scan_tile_kernel<T><<<(unsigned)tiles, kScanThreads, 0, s>>>(in, out, n, sums);
    launched("scan_tile_kernel");
    scan_exclusive_impl<int64_t>(sums, sums, tiles, s);
    scan_add_kernel<T><<<(unsigned)((n + 255) / 256), 256, 0, s>>>(out, n, sums);
    launched("scan_add_kernel");
    check_cuda(cudaStreamSynchronize(s), "scan sync");
    dfree(sums);
}
}  // namespace

void scan_exclusive_i64(const int64_t* in, int64_t* out, int64_t n, cudaStream_t s) {
    scan_exclusive_impl<int64_t>(in, out, n, s);
}
void scan_exclusive_i32(const int32_t* in, int32_t* out, int64_t n, cudaStream_t s) {
    scan_exclusive_impl<int32_t>(in, out, n, s);
}

// ---------------------------------------------------------------- BLAS-1
namespace {
constexpr int kRedThreads = 256;

enum RedOp { kDot = 0, kSumSq = 1, kMaxAbs = 2 };

// Deterministic grid reduction: each block folds a fixed, grid-strided slice
// in index order, reduces it with a fixed tree into partials[block]; the last
// block to finish folds the partials in block order. The grid size depends
// only on n, so the bits do not change from run to run.
template <int OP>
__global__ void __launch_bounds__(kRedThreads) reduce_kernel(int64_t n, const double* __restrict__ a,
                                                             const double* __restrict__ b,
                                                             double* partials, unsigned* counter,
                                                             double* out) {
    __shared__ double sh[32];
    __shared__ bool last;
    double acc = 0.0;
    const int64_t stride = (int64_t)gridDim.x * kRedThreads;
    for (int64_t i = blockIdx.x * (int64_t)kRedThreads + threadIdx.x; i < n; i += stride) {
        if (OP == kDot) acc += a[i] * b[i];
        else if (OP == kSumSq) acc += a[i] * a[i];
        else acc = fmax(acc, fabs(a[i]));
    }
    double r = (OP == kMaxAbs) ? block_max<kRedThreads>(acc, sh) : block_sum<kRedThreads>(acc, sh);
    if (threadIdx.x == 0) {
        partials[blockIdx.x] = r;
        __threadfence();
        const unsigned t = atomicAdd(counter, 1u);
        last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    double v = (OP == kMaxAbs) ? 0.0 : 0.0;
    for (int i = threadIdx.x; i < (int)gridDim.x; i += kRedThreads) {
        const double p = __ldcg(partials + i);
        v = (OP == kMaxAbs) ? fmax(v, p) : v + p;
    }
    r = (OP == kMaxAbs) ? block_max<kRedThreads>(v, sh) : block_sum<kRedThreads>(v, sh);
    if (threadIdx.x == 0) {
        *out = (OP == kSumSq) ? sqrt(r) : r;
        *counter = 0u;
    }
}

__global__ void axpy_kernel(int64_t n, double alpha, const double* __restrict__ x,
                            double* __restrict__ y) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += stride)
        y[i] += alpha * x[i];
}

template <int OP>
void run_reduce(int64_t n, const double* a, const double* b, double* out, cudaStream_t s) {
    Workspace& w = workspace(s);
    const int grid = grid_for(n, kRedThreads * 4, kMaxReduceBlocks);
    reduce_kernel<OP><<<grid, kRedThreads, 0, s>>>(n, a, b, w.partials, w.counter, out);
    launched("reduce_kernel");
}
}  // namespace

void reduce_dot(int64_t n, const double* a, const double* b, double* out, cudaStream_t s) {
    run_reduce<kDot>(n, a, b, out, s);
}
void reduce_nrm2(int64_t n, const double* a, double* out, cudaStream_t s) {
    run_reduce<kSumSq>(n, a, nullptr, out, s);
}
void reduce_maxabs(int64_t n, const double* a, double* out, cudaStream_t s) {
    run_reduce<kMaxAbs>(n, a, nullptr, out, s);
}

}  // namespace hn

using namespace hn;

// ================================================================ C ABI
extern "C" {

int hn_init(int device) {
    return guard("hn_init", [&] {
        int count = 0;
        check_cuda(cudaGetDeviceCount(&count), "cudaGetDeviceCount");
        if (device < 0 || device >= count)
            fail(HN_ERR_INVALID_ARG, "device " + std::to_string(device) + " out of range (" +
                                         std::to_string(count) + " devices)");
        cudaDeviceProp p;
        check_cuda(cudaGetDeviceProperties(&p, device), "cudaGetDeviceProperties");
        if (p.major != 10 || p.minor != 0)
            fail(HN_ERR_UNSUPPORTED, std::string("device is sm_") + std::to_string(p.major) +
                                         std::to_string(p.minor) +
                                         "; this library is built for sm_100a only");
        check_cuda(cudaSetDevice(device), "cudaSetDevice");
        check_cuda(cudaFree(nullptr), "context creation");
        ctx().device = device;
        ctx().sm_count = p.multiProcessorCount;
    });
}

int hn_shutdown(void) {
    return guard("hn_shutdown", [&] {
        Context& c = ctx();
        if (c.device < 0) return;
        cudaDeviceSynchronize();
        std::lock_guard<std::mutex> lk(c.mu);
        for (auto& kv : c.ws) {
            dfree(kv.second.partials);
            dfree(kv.second.counter);
            dfree(kv.second.select);
            dfree(kv.second.staging_d);
            if (kv.second.staging_h) cudaFreeHost(kv.second.staging_h);
        }
        c.ws.clear();
    });
}

const char* hn_last_error(void) { return g_last_error.c_str(); }

int hn_device_info(hn_device_info_t* out) {
    return guard("hn_device_info", [&] {
        require_init();
        if (!out) fail(HN_ERR_INVALID_ARG, "null output");
        cudaDeviceProp p;
        check_cuda(cudaGetDeviceProperties(&p, ctx().device), "cudaGetDeviceProperties");
        std::memset(out, 0, sizeof(*out));
        std::strncpy(out->name, p.name, sizeof(out->name) - 1);
        out->device = ctx().device;
        out->sm_count = p.multiProcessorCount;
        out->cc_major = p.major;
        out->cc_minor = p.minor;
        check_cuda(cudaMemGetInfo(&out->free_mem, &out->total_mem), "cudaMemGetInfo");
    });
}

int hn_stats(uint64_t* kernel_launches, uint64_t* api_calls) {
    if (kernel_launches) *kernel_launches = ctx().launches.load();
    if (api_calls) *api_calls = ctx().calls.load();
    return HN_OK;
}

int hn_reset_stats(void) {
    ctx().launches.store(0);
    ctx().calls.store(0);
    return HN_OK;
}

int hn_fault_inject(int64_t after_calls, int status) {
    ctx().inject_status.store(status);
    ctx().inject_after.store(after_calls < 0 ? -1 : after_calls);
    return HN_OK;
}

int hn_malloc(void** ptr_dev, size_t bytes) {
    return guard("hn_malloc", [&] {
        require_init();
        if (!ptr_dev) fail(HN_ERR_INVALID_ARG, "null output");
        *ptr_dev = dmalloc<char>(bytes);
    });
}

int hn_free(void* p) {
    return guard("hn_free", [&] {
        require_init();
        check_cuda(cudaFree(p), "cudaFree");
    });
}

int hn_memcpy_h2d(void* dst, const void* src, size_t bytes, void* stream) {
    return guard("hn_memcpy_h2d", [&] {
        require_init();
        check_cuda(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, as_stream(stream)),
                   "cudaMemcpyAsync H2D");
    });
}

int hn_memcpy_d2h(void* dst, const void* src, size_t bytes, void* stream) {
    return guard("hn_memcpy_d2h", [&] {
        require_init();
        check_cuda(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, as_stream(stream)),
                   "cudaMemcpyAsync D2H");
        check_cuda(cudaStreamSynchronize(as_stream(stream)), "D2H sync");
    });
}

int hn_memcpy_d2d(void* dst, const void* src, size_t bytes, void* stream) {
    return guard("hn_memcpy_d2d", [&] {
        require_init();
        check_cuda(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, as_stream(stream)),
                   "cudaMemcpyAsync D2D");
    });
}

int hn_memset(void* p, int byte, size_t bytes, void* stream) {
    return guard("hn_memset", [&] {
        require_init();
        check_cuda(cudaMemsetAsync(p, byte, bytes, as_stream(stream)), "cudaMemsetAsync");
    });
}

int hn_stream_sync(void* stream) {
    return guard("hn_stream_sync", [&] {
        require_init();
        check_cuda(cudaStreamSynchronize(as_stream(stream)), "cudaStreamSynchronize");
    });
}

int hn_dot(int64_t n, const double* a, const double* b, double* result, void* stream) {
    return guard("hn_dot", [&] {
        require_init();
        if (n < 0 || !result || (n > 0 && (!a || !b))) fail(HN_ERR_INVALID_ARG, "bad arguments");
        reduce_dot(n, a, b, result, as_stream(stream));
    });
}

int hn_axpy(int64_t n, double alpha, const double* x, double* y, void* stream) {
    return guard("hn_axpy", [&] {
        require_init();
        if (n < 0 || (n > 0 && (!x || !y))) fail(HN_ERR_INVALID_ARG, "bad arguments");
        if (n == 0) return;
        axpy_kernel<<<grid_for(n, 256, ctx().sm_count * 16), 256, 0, as_stream(stream)>>>(n, alpha,
                                                                                       x, y);
        launched("axpy_kernel");
    });
}

int hn_nrm_inf(int64_t n, const double* v, double* result, void* stream) {
    return guard("hn_nrm_inf", [&] {
        require_init();
        if (n < 0 || !result || (n > 0 && !v)) fail(HN_ERR_INVALID_ARG, "bad arguments");
        reduce_maxabs(n, v, result, as_stream(stream));
    });
}

int hn_nrm2(int64_t n, const double* v, double* result, void* stream) {
    return guard("hn_nrm2", [&] {
        require_init();
        if (n < 0 || !result || (n > 0 && !v)) fail(HN_ERR_INVALID_ARG, "bad arguments");
        reduce_nrm2(n, v, result, as_stream(stream));
    });
}

}  // extern "C"
