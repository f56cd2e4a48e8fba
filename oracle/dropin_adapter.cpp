// The HyperNova-side adapter a maintainer adds (hn::execution::B200Backend
// behind the reference's IComputeBackend), compiled against the
// reference's own headers -- TEST INFRASTRUCTURE ONLY (built into
// oracle/_ref/libhnref_dropin.so with the reference objects). It lets a GPU
// test run the reference's unchanged InteriorPointSolver::solve
// (core/lp/interior_point.cpp:402-886) with InteriorPointOptions::compute_backend
// set to the B200 backend, i.e. the drop-in exactly as a maintainer wires it.
#include "gpu_backend.hpp"
#include "hn_backend.hpp"
#include "interior_point.hpp"
#include "problem.hpp"

#include <cstdint>
#include <memory>
#include <stdexcept>

namespace hypernova::execution {
class B200ComputeBackend final : public IComputeBackend {
public:
    ComputeBackendType type() const override { return ComputeBackendType::CUDA; }
    std::string name() const override { return impl_.name(); }
    bool is_available() const override { return impl_.is_available(); }
    void initialize() override { impl_.initialize(); }
    void finalize() override { impl_.finalize(); }
    void spmv(const std::vector<double>& v, const std::vector<std::size_t>& c, const std::vector<std::size_t>& r,
              const std::vector<double>& x, std::vector<double>& y) override {
        impl_.spmv(v, c, r, x, y);
    }
    void spmm(const std::vector<double>& v, const std::vector<std::size_t>& c, const std::vector<std::size_t>& r,
              const std::vector<double>& B, std::vector<double>& C, std::size_t k) override {
        impl_.spmm(v, c, r, B, C, k);
    }
    double dot(const std::vector<double>& a, const std::vector<double>& b) override { return impl_.dot(a, b); }
    void axpy(double al, const std::vector<double>& x, std::vector<double>& y) override { impl_.axpy(al, x, y); }
    double norm_inf(const std::vector<double>& v) override { return impl_.norm_inf(v); }
    std::size_t device_memory() const override { return impl_.device_memory(); }
    std::size_t free_memory() const override { return impl_.free_memory(); }
    bool was_gpu_kernel_executed() const override { return impl_.was_gpu_kernel_executed(); }
    std::size_t gpu_kernel_executions() const override { return impl_.gpu_kernel_executions(); }
    void reset_execution_stats() override { impl_.reset_execution_stats(); }

private:
    hn::execution::B200Backend impl_;
};
}  // namespace hypernova::execution

extern "C" {

// The reference IPM (crossover off) on an all-EQ, x >= 0 LP with the B200
// backend plugged in. Returns the ProblemStatus; *kernels receives the number
// of GPU kernels the backend launched.
int hnref_ipm_solve_b200(int64_t m, int64_t n, const uint64_t* rp, const uint64_t* ci, const double* val,
                         const double* c, const double* b, double* obj, int64_t* iters, uint64_t* kernels) {
    using namespace hypernova::model;
    ProblemBuilder builder("dropin");
    for (int64_t j = 0; j < n; ++j) builder.add_variable(0.0);
    for (int64_t i = 0; i < m; ++i) {
        std::vector<std::pair<std::size_t, double>> coeffs;
        for (uint64_t k = rp[i]; k < rp[i + 1]; ++k) coeffs.emplace_back(ci[k], val[k]);
        builder.add_constraint(coeffs, ConstraintSense::EQ, b[i]);
    }
    std::vector<std::pair<std::size_t, double>> objc;
    for (int64_t j = 0; j < n; ++j) objc.emplace_back(j, c[j]);
    builder.set_objective(objc, ObjectiveSense::MINIMIZE);
    Problem prob = builder.build();
    auto backend = std::make_shared<hypernova::execution::B200ComputeBackend>();
    backend->initialize();
    if (!backend->is_available()) return -1;
    hypernova::lp::InteriorPointOptions opts;
    opts.crossover = false;
    opts.compute_backend = backend;
    hypernova::lp::InteriorPointSolver solver(hypernova::numerical::ToleranceConfig::industrial_defaults(), opts);
    auto r = solver.solve(prob);
    *obj = r.objective_value;
    *iters = static_cast<int64_t>(r.iterations);
    *kernels = backend->gpu_kernel_executions();
    return static_cast<int>(r.status);
}

}  // extern "C"
