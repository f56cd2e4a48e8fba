// hn::execution -- the compute-backend interface HyperNova's solvers call,
// with the B200 implementation behind it.
//
// IComputeBackend restates hypernova::execution::IComputeBackend
// (core/execution/gpu_backend.hpp:18-51) member for member -- same names,
// arguments and calling conventions (callee-resized outputs, C overwritten) --
// and adds the products the IPM needs beyond it (A^T x, A D A^T). B200Backend
// runs every call on the GPU through libhn_sm100.so; there is no CPU path.
// A failure throws std::runtime_error with the library's message, as
// CudaDriverBackend does (gpu_backend.cpp:212-214).
#pragma once

#include <cstddef>
#include <cstdint>
#include <memory>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

struct hn_csr;

namespace hn::execution {

enum class ComputeBackendType { CPU, CUDA, HIP, SYCL, AUTO };

class IComputeBackend {
public:
    virtual ~IComputeBackend() = default;
    virtual ComputeBackendType type() const = 0;
    virtual std::string name() const = 0;
    virtual bool is_available() const = 0;
    virtual void initialize() = 0;
    virtual void finalize() = 0;
    virtual void spmv(const std::vector<double>& values, const std::vector<std::size_t>& col_indices,
                      const std::vector<std::size_t>& row_ptr, const std::vector<double>& x,
                      std::vector<double>& y) = 0;
    virtual void spmm(const std::vector<double>& values, const std::vector<std::size_t>& col_indices,
                      const std::vector<std::size_t>& row_ptr, const std::vector<double>& B,
                      std::vector<double>& C, std::size_t ncols_B) = 0;
    virtual double dot(const std::vector<double>& a, const std::vector<double>& b) = 0;
    virtual void axpy(double alpha, const std::vector<double>& x, std::vector<double>& y) = 0;
    virtual double norm_inf(const std::vector<double>& v) = 0;
    virtual std::size_t device_memory() const = 0;
    virtual std::size_t free_memory() const = 0;
    virtual bool was_gpu_kernel_executed() const { return false; }
    virtual std::size_t gpu_kernel_executions() const { return 0; }
    virtual void reset_execution_stats() {}
    // Extensions (no reference counterpart): y = A^T x for the same CSR
    // arrays, ncols columns (the IPM's matvec_t, interior_point.cpp:61-69).
    virtual void spmv_t(const std::vector<double>& values, const std::vector<std::size_t>& col_indices,
                        const std::vector<std::size_t>& row_ptr, std::size_t ncols, const std::vector<double>& x,
                        std::vector<double>& y) = 0;
};

class B200Backend : public IComputeBackend {
public:
    explicit B200Backend(int device = 0) : device_(device) {}
    ~B200Backend() override;
    ComputeBackendType type() const override { return ComputeBackendType::CUDA; }
    std::string name() const override;
    bool is_available() const override { return available_; }
    void initialize() override;
    void finalize() override;
    void spmv(const std::vector<double>& values, const std::vector<std::size_t>& col_indices,
              const std::vector<std::size_t>& row_ptr, const std::vector<double>& x,
              std::vector<double>& y) override;
    void spmm(const std::vector<double>& values, const std::vector<std::size_t>& col_indices,
              const std::vector<std::size_t>& row_ptr, const std::vector<double>& B, std::vector<double>& C,
              std::size_t ncols_B) override;
    double dot(const std::vector<double>& a, const std::vector<double>& b) override;
    void axpy(double alpha, const std::vector<double>& x, std::vector<double>& y) override;
    double norm_inf(const std::vector<double>& v) override;
    std::size_t device_memory() const override;
    std::size_t free_memory() const override;
    bool was_gpu_kernel_executed() const override;
    std::size_t gpu_kernel_executions() const override;
    void reset_execution_stats() override;
    void spmv_t(const std::vector<double>& values, const std::vector<std::size_t>& col_indices,
                const std::vector<std::size_t>& row_ptr, std::size_t ncols, const std::vector<double>& x,
                std::vector<double>& y) override;
    const std::string& last_error() const { return last_error_; }

private:
    struct Resident {
        hn_csr* h = nullptr;
        std::size_t nnz = 0, nrows = 0, ncols = 0;
        uint64_t fingerprint = 0;
    };
    // Device copy of a matrix, keyed by the host values pointer like the
    // reference's cache (gpu_backend.cpp:289-306) but also checked against
    // sizes and a hash of every entry of the three arrays, so a reused buffer
    // with new contents is uploaded again instead of returning stale data.
    Resident& resident(const std::vector<double>& values, const std::vector<std::size_t>& col_indices,
                       const std::vector<std::size_t>& row_ptr, std::size_t ncols);
    void require(const char* op) const;
    double* staging(std::size_t doubles);
    void release();

    int device_;
    bool initialized_ = false;
    bool available_ = false;
    std::string last_error_;
    std::string device_name_;
    std::unordered_map<const void*, Resident> cache_;
    double* dev_buf_ = nullptr;
    std::size_t dev_buf_len_ = 0;
    uint64_t launches_at_reset_ = 0;
    mutable std::mutex mutex_;
};

class ComputeBackendFactory {
public:
    // CUDA and AUTO give a B200Backend; other types are not provided by this
    // library (the reference's CPU backend stays in the reference).
    static std::unique_ptr<IComputeBackend> create_backend(ComputeBackendType type);
};

}  // namespace hn::execution
