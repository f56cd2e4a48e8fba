// C ABI of the products: SpMV (A and A^T) and SpMM.
#include <cstring>

#include "hn_spmv.cuh"

namespace hn {
namespace {

// C = op(A) B, B row-major (ncols x k). One warp per row; lanes own output
// columns, kSpmmCols register accumulators each, nonzeros in CSR order so each
// C entry is summed in the reference's order (gpu_backend.cpp:112-121).
constexpr int kSpmmCols = 4;  // 32 lanes x 4 = 128 columns per pass

__global__ void __launch_bounds__(256) spmm_kernel(int m, const int32_t* __restrict__ rp,
                                                   const int32_t* __restrict__ ci,
                                                   const double* __restrict__ val,
                                                   const double* __restrict__ B, int64_t k,
                                                   double* __restrict__ C) {
    const int64_t row = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (row >= m) return;
    const int32_t p0 = rp[row], p1 = rp[row + 1];
    for (int64_t c0 = 0; c0 < k; c0 += 32 * kSpmmCols) {
        double acc[kSpmmCols];
#pragma unroll
        for (int u = 0; u < kSpmmCols; ++u) acc[u] = 0.0;
        for (int32_t p = p0; p < p1; ++p) {
            const double a = __ldg(val + p);
            const double* Bj = B + (int64_t)__ldg(ci + p) * k;
#pragma unroll
            for (int u = 0; u < kSpmmCols; ++u) {
                const int64_t c = c0 + u * 32 + lane;
                if (c < k) acc[u] += a * __ldg(Bj + c);
            }
        }
#pragma unroll
        for (int u = 0; u < kSpmmCols; ++u) {
            const int64_t c = c0 + u * 32 + lane;
            if (c < k) C[row * k + c] = acc[u];
        }
    }
}

void check_handle(const hn_csr* A, int trans) {
    if (!A) fail(HN_ERR_INVALID_ARG, "null matrix handle");
    if (trans && !A->has_t) fail(HN_ERR_INVALID_ARG, "handle was created without A^T");
}

void spmm_run(const hn_csr* A, int trans, const double* B, int64_t k, double* C, cudaStream_t s) {
    const SpmvMat M = spmv_mat(A, trans);
    if (M.m == 0 || k == 0) return;
    const int64_t threads = (int64_t)M.m * 32;
    spmm_kernel<<<(unsigned)((threads + 255) / 256), 256, 0, s>>>(M.m, M.rp, M.ci, M.val, B, k, C);
    launched("spmm_kernel");
}

}  // namespace
}  // namespace hn

using namespace hn;

extern "C" {

int hn_spmv(const hn_csr* A, int trans, double alpha, const double* x, double beta, double* y,
            void* stream) {
    return guard("hn_spmv", [&] {
        require_init();
        check_handle(A, trans);
        const SpmvMat M = spmv_mat(A, trans);
        const int64_t cols = trans ? A->m : A->n;
        if (M.m > 0 && !y) fail(HN_ERR_INVALID_ARG, "null y");
        if (cols > 0 && M.nnz > 0 && !x) fail(HN_ERR_INVALID_ARG, "null x");
        spmv_launch(M, x, EpiAxpby{alpha, beta, y}, as_stream(stream));
    });
}

int hn_spmv_residual(const hn_csr* A, int trans, const double* x, const double* b, double* y, void* stream) {
    return guard("hn_spmv_residual", [&] {
        require_init();
        check_handle(A, trans);
        const SpmvMat M = spmv_mat(A, trans);
        const int64_t cols = trans ? A->m : A->n;
        if (M.m > 0 && (!y || !b)) fail(HN_ERR_INVALID_ARG, "null b or y");
        if (cols > 0 && M.nnz > 0 && !x) fail(HN_ERR_INVALID_ARG, "null x");
        spmv_launch(M, x, EpiSub{b, y}, as_stream(stream));
    });
}

int hn_spmv_host(const hn_csr* A, int trans, const double* x, double* y) {
    return guard("hn_spmv_host", [&] {
        require_init();
        check_handle(A, trans);
        const SpmvMat M = spmv_mat(A, trans);
        const int64_t cols = trans ? A->m : A->n;
        const int64_t rows = M.m;
        if ((rows > 0 && !y) || (cols > 0 && !x)) fail(HN_ERR_INVALID_ARG, "null vector");
        cudaStream_t s = nullptr;
        Workspace& w = workspace(s);
        ensure_staging(w, sizeof(double) * (cols + rows + 2), s);
        double* xh = w.staging_h;
        double* yh = w.staging_h + cols;
        double* xd = w.staging_d;
        double* yd = w.staging_d + cols;
        std::memcpy(xh, x, sizeof(double) * cols);
        check_cuda(cudaMemcpyAsync(xd, xh, sizeof(double) * cols, cudaMemcpyHostToDevice, s), "H2D x");
        spmv_launch(M, xd, EpiAxpby{1.0, 0.0, yd}, s);
        check_cuda(cudaMemcpyAsync(yh, yd, sizeof(double) * rows, cudaMemcpyDeviceToHost, s), "D2H y");
        check_cuda(cudaStreamSynchronize(s), "hn_spmv_host sync");
        std::memcpy(y, yh, sizeof(double) * rows);
    });
}

int hn_spmm(const hn_csr* A, int trans, const double* B, int64_t k, double* C, void* stream) {
    return guard("hn_spmm", [&] {
        require_init();
        check_handle(A, trans);
        if (k < 0) fail(HN_ERR_INVALID_ARG, "negative k");
        spmm_run(A, trans, B, k, C, as_stream(stream));
    });
}

int hn_spmm_host(const hn_csr* A, int trans, const double* B, int64_t k, double* C) {
    return guard("hn_spmm_host", [&] {
        require_init();
        check_handle(A, trans);
        if (k < 0) fail(HN_ERR_INVALID_ARG, "negative k");
        const int64_t cols = trans ? A->m : A->n;
        const int64_t rows = trans ? A->n : A->m;
        cudaStream_t s = nullptr;
        Workspace& w = workspace(s);
        const size_t nb = sizeof(double) * (size_t)(cols * k), nc = sizeof(double) * (size_t)(rows * k);
        ensure_staging(w, nb + nc + 16, s);
        double* Bd = w.staging_d;
        double* Cd = w.staging_d + cols * k;
        std::memcpy(w.staging_h, B, nb);
        check_cuda(cudaMemcpyAsync(Bd, w.staging_h, nb, cudaMemcpyHostToDevice, s), "H2D B");
        spmm_run(A, trans, Bd, k, Cd, s);
        check_cuda(cudaMemcpyAsync(w.staging_h + cols * k, Cd, nc, cudaMemcpyDeviceToHost, s), "D2H C");
        check_cuda(cudaStreamSynchronize(s), "hn_spmm_host sync");
        std::memcpy(C, w.staging_h + cols * k, nc);
    });
}

}  // extern "C"
