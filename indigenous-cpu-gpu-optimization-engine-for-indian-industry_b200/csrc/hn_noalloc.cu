// y = A x for callers that cannot allocate device memory.
//
// hn_spmv (hn_spmv.cu) needs a matrix handle, and creating one calls
// cudaMalloc for the int32 copy, the merge-path tile table and the carry
// buffers. Some callers cannot do that: a solver embedded in a framework whose
// memory pool owns the whole device, or an IPM or branch-and-bound loop that
// must not allocate mid-solve (cudaMalloc synchronises the device and can fail
// with the pool already holding the memory). hn_spmv_noalloc takes the CSR
// arrays already on the device and keeps the merge-path scratch -- the tile
// table and the per-tile carries -- in one file-scope __device__ array of
// fixed size instead of allocated buffers. It runs the same tile and fix-up
// kernels as hn_spmv, so its results are the same.
//
// Scratch: kNoAllocTiles tiles of kSpmvTile merge items, i.e. m + nnz <=
// 65,536 * 1,792 = 117,440,512; 2 MB of device memory that every GPU loading
// this library holds until the process exits. Every launch rewrites all the
// scratch it reads (tile table, carries, head flags), so nothing needs
// clearing between calls; but all calls share the one array, so two calls
// that overlap on the GPU (different streams, or different host threads)
// race and corrupt each other's results -- serialise them.
#include "hn_spmv.cuh"

namespace hn {
namespace {

constexpr int64_t kNoAllocTiles = 65536;

struct NoAllocScratch {
    int32_t tile_row[kNoAllocTiles + 1];
    int32_t tile_nz[kNoAllocTiles + 1];
    int32_t carry_row[kNoAllocTiles];
    int32_t head_row[kNoAllocTiles];
    double carry_val[kNoAllocTiles];
    double head_val[kNoAllocTiles];
};

static __device__ __align__(256) NoAllocScratch g_noalloc_scratch;

// Merge-path coordinates of diagonals t * kSpmvTile (same search as the tile
// table hn_csr_create builds).
__global__ void noalloc_tiles_kernel(const int32_t* __restrict__ rp, int64_t m, int64_t nnz, int64_t ntiles,
                                     NoAllocScratch* sc) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t > ntiles) return;
    int64_t diag = t * kSpmvTile;
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
    sc->tile_row[t] = static_cast<int32_t>(lo);
    sc->tile_nz[t] = static_cast<int32_t>(diag - lo);
}

// Device address of the scratch array, looked up once per device (host code
// cannot use the symbol's name as a device pointer).
constexpr int kMaxDevices = 64;
NoAllocScratch* g_scratch_addr[kMaxDevices] = {};
std::mutex g_scratch_mu;

NoAllocScratch* scratch_for_current_device() {
    int dev = -1;
    check_cuda(cudaGetDevice(&dev), "cudaGetDevice");
    if (dev < 0 || dev >= kMaxDevices) fail(HN_ERR_UNSUPPORTED, "device index beyond the scratch table");
    std::lock_guard<std::mutex> lk(g_scratch_mu);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        check_cuda(cudaGetSymbolAddress(&p, g_noalloc_scratch), "cudaGetSymbolAddress(scratch)");
        g_scratch_addr[dev] = static_cast<NoAllocScratch*>(p);
    }
    return g_scratch_addr[dev];
}

}  // namespace
}  // namespace hn

using namespace hn;

extern "C" {

int hn_spmv_noalloc(int64_t m, int64_t n, int64_t nnz, const int32_t* rp, const int32_t* ci, const double* val,
                    const double* x, double* y, void* stream) {
    return guard("hn_spmv_noalloc", [&] {
        require_init();
        if (m < 0 || n < 0 || nnz < 0) fail(HN_ERR_INVALID_ARG, "negative size");
        if (m + nnz > kNoAllocTiles * kSpmvTile)
            fail(HN_ERR_INVALID_ARG, "m + nnz = " + std::to_string(m + nnz) + " exceeds the scratch limit of " +
                                         std::to_string(kNoAllocTiles * kSpmvTile) + " merge items");
        if (m > 0 && (!rp || !y)) fail(HN_ERR_INVALID_ARG, "null row_ptr or y");
        if (nnz > 0 && (!ci || !val || !x)) fail(HN_ERR_INVALID_ARG, "null col_idx, values or x");
        NoAllocScratch* sc = scratch_for_current_device();
        const int64_t ntiles = (m + nnz + kSpmvTile - 1) / kSpmvTile;
        if (ntiles == 0) return;
        cudaStream_t s = as_stream(stream);
        noalloc_tiles_kernel<<<(unsigned)((ntiles + 1 + 255) / 256), 256, 0, s>>>(rp, m, nnz, ntiles, sc);
        launched("noalloc_tiles_kernel");
        SpmvMat M{(int)m, (int)nnz, rp, ci, val, sc->tile_row, sc->tile_nz, sc->carry_row, sc->carry_val,
                  sc->head_row, sc->head_val, ntiles};
        spmv_launch(M, x, EpiAxpby{1.0, 0.0, y}, s);
    });
}

}  // extern "C"
