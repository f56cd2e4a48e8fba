// Second shim over the reference (TEST INFRASTRUCTURE ONLY): reaches the IPM
// helpers that core/lp/interior_point.cpp keeps in an anonymous namespace --
// build_normal_equations (:144-200), matvec (:52-59), matvec_t (:61-69),
// max_step (:134-142) and remove_duplicate_rows (the crossover's problem) --
// by compiling that file into this translation unit.
// oracle/Makefile links this object in place of interior_point.o, so the
// library still holds exactly one InteriorPointSolver.
#include "interior_point.cpp"

#include <chrono>
#include <cstring>
#include <thread>

namespace {
hypernova::numerical::SparseMatrix shim_csr(int64_t m, int64_t n, const uint64_t* rp, const uint64_t* ci,
                                            const double* val) {
    hypernova::numerical::SparseMatrix A(static_cast<std::size_t>(m), static_cast<std::size_t>(n));
    const std::size_t nnz = static_cast<std::size_t>(rp[m]);
    A.mutable_row_ptr().assign(rp, rp + m + 1);
    A.mutable_col_indices().assign(ci, ci + nnz);
    A.mutable_values().assign(val, val + nnz);
    return A;
}
}  // namespace

extern "C" {

// N = build_normal_equations(A, D, reg). Returns nnz(N) and fills rp (m+1)
// and ci/val when they are non-null and hold `cap` entries.
int64_t hnref_normal_equations(int64_t m, int64_t n, const uint64_t* rp, const uint64_t* ci,
                               const double* val, const double* D, double reg, int64_t cap,
                               uint64_t* rpN, uint64_t* ciN, double* valN) {
    auto A = shim_csr(m, n, rp, ci, val);
    std::vector<double> d(D, D + n);
    auto N = hypernova::lp::build_normal_equations(A, d, reg);
    if (rpN)
        for (std::size_t i = 0; i < N.row_ptr().size(); ++i) rpN[i] = N.row_ptr()[i];
    if (ciN && valN && static_cast<int64_t>(N.nnz()) <= cap)
        for (std::size_t k = 0; k < N.nnz(); ++k) {
            ciN[k] = N.col_indices()[k];
            valN[k] = N.values()[k];
        }
    return static_cast<int64_t>(N.nnz());
}

void hnref_matvec_t(int64_t m, int64_t n, const uint64_t* rp, const uint64_t* ci, const double* val,
                    const double* x, double* y) {
    auto A = shim_csr(m, n, rp, ci, val);
    std::vector<double> xx(x, x + m);
    auto r = hypernova::lp::matvec_t(A, xx);
    std::memcpy(y, r.data(), sizeof(double) * r.size());
}

double hnref_max_step(int64_t n, const double* v, const double* d) {
    std::vector<double> vv(v, v + n), dd(d, d + n);
    return hypernova::lp::max_step(vv, dd);
}

// CPU baseline of one pass of the per-iteration sparse path: every host
// thread runs, with the reference's own code, y = A x (CPUBackend::spmv),
// t = A^T lam (the IPM's matvec_t) and build_normal_equations on its own
// column slice of A (columns [t*ns/T, (t+1)*ns/T) of the first ns columns).
// Returns the wall seconds of `reps` passes; *trip_out receives the number of
// triplets the slices emit per pass and *nnzn_out the summed nnz(N) of the slices.
double hnref_step_sample(int64_t m, int64_t n, const uint64_t* rp, const uint64_t* ci, const double* val,
                         const double* x, const double* lam, const double* D, int64_t ns, int threads,
                         int reps, int64_t* trip_out, int64_t* nnzn_out) {
    if (threads < 1) threads = 1;
    auto A = shim_csr(m, n, rp, ci, val);
    const std::vector<double> xx(x, x + n), ll(lam, lam + m);
    std::vector<hypernova::numerical::SparseMatrix> slices(threads);
    std::vector<std::vector<double>> dsl(threads);
    int64_t trip = 0;
    for (int t = 0; t < threads; ++t) {
        const int64_t c0 = ns * t / threads, c1 = ns * (t + 1) / threads;
        std::vector<hypernova::numerical::Triplet> tr;
        std::vector<int64_t> cnt(c1 - c0, 0);
        for (int64_t i = 0; i < m; ++i)
            for (uint64_t k = rp[i]; k < rp[i + 1]; ++k)
                if (static_cast<int64_t>(ci[k]) >= c0 && static_cast<int64_t>(ci[k]) < c1) {
                    tr.emplace_back(i, ci[k] - c0, val[k]);
                    ++cnt[ci[k] - c0];
                }
        slices[t] = hypernova::numerical::SparseMatrix::from_triplets(m, c1 - c0, tr);
        dsl[t].assign(D + c0, D + c1);
        for (auto c : cnt) trip += c * c;
    }
    std::vector<int64_t> nnzn(threads, 0);
    auto run = [&](int t) {
        auto backend = hypernova::execution::ComputeBackendFactory::create_backend(
            hypernova::execution::ComputeBackendType::CPU);
        std::vector<double> y;
        for (int r = 0; r < reps; ++r) {
            backend->spmv(A.values(), A.col_indices(), A.row_ptr(), xx, y);
            auto tv = hypernova::lp::matvec_t(A, ll);
            auto N = hypernova::lp::build_normal_equations(slices[t], dsl[t], 1e-8);
            nnzn[t] = static_cast<int64_t>(N.nnz());
        }
    };
    auto t0 = std::chrono::steady_clock::now();
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; ++t) pool.emplace_back(run, t);
    for (auto& th : pool) th.join();
    auto t1 = std::chrono::steady_clock::now();
    if (trip_out) *trip_out = trip + m * threads;
    if (nnzn_out) {
        int64_t s = 0;
        for (auto v : nnzn) s += v;
        *nnzn_out = s;
    }
    return std::chrono::duration<double>(t1 - t0).count();
}

// The reference's crossover polish (interior_point.cpp:792-876) from a given
// barrier endpoint: SimplexSolver::solve_with_basis on the problem with
// duplicate rows removed, from `var_status` (the caller's warm basis), with
// crossover_max_iter iterations; if that gives no definitive verdict, a
// cold SimplexSolver::solve. `barrier_status` is the barrier's verdict
// (OPTIMAL = converged). Returns the final status; objective, iterations.
int hnref_crossover_polish(int64_t m, int64_t n, const uint64_t* rp, const uint64_t* ci, const double* val,
                           const double* c, const double* b, const int* sense, const double* lb,
                           const double* ub, int maximize, int barrier_status, const int* var_status,
                           double* obj, int64_t* iters) {
    using namespace hypernova::model;
    ProblemBuilder builder("hnref");
    for (int64_t j = 0; j < n; ++j) builder.add_variable(lb[j], ub[j]);
    for (int64_t i = 0; i < m; ++i) {
        std::vector<std::pair<std::size_t, double>> coeffs;
        for (uint64_t k = rp[i]; k < rp[i + 1]; ++k) coeffs.emplace_back(ci[k], val[k]);
        const ConstraintSense s =
            sense[i] == 0 ? ConstraintSense::LE : (sense[i] == 1 ? ConstraintSense::GE : ConstraintSense::EQ);
        builder.add_constraint(coeffs, s, b[i]);
    }
    std::vector<std::pair<std::size_t, double>> objc;
    for (int64_t j = 0; j < n; ++j) objc.emplace_back(j, c[j]);
    builder.set_objective(objc, maximize ? ObjectiveSense::MAXIMIZE : ObjectiveSense::MINIMIZE);
    Problem cleaned = hypernova::lp::remove_duplicate_rows(builder.build());
    const bool done = barrier_status == static_cast<int>(ProblemStatus::OPTIMAL);
    int status = barrier_status;
    *obj = 0.0;
    *iters = 0;
    auto adopt = [&](const hypernova::lp::SimplexResult& sim) {
        if (sim.status == ProblemStatus::OPTIMAL) {
            status = static_cast<int>(ProblemStatus::OPTIMAL);
            *obj = sim.objective_value;
            *iters = static_cast<int64_t>(sim.iterations);
        } else if (!done && sim.status == ProblemStatus::INFEASIBLE) {
            status = static_cast<int>(ProblemStatus::INFEASIBLE);
        } else if (sim.status == ProblemStatus::UNBOUNDED) {
            status = static_cast<int>(ProblemStatus::UNBOUNDED);
        }
    };
    const auto tol = hypernova::numerical::ToleranceConfig::industrial_defaults();
    bool resolved = false;
    try {
        hypernova::lp::SimplexOptions warm;
        warm.max_iterations = hypernova::lp::InteriorPointOptions{}.crossover_max_iter;
        hypernova::lp::SimplexSolver polisher(tol, warm);
        auto sim = polisher.solve_with_basis(cleaned, std::vector<int>(var_status, var_status + n));
        adopt(sim);
        resolved = sim.status == ProblemStatus::OPTIMAL || sim.status == ProblemStatus::UNBOUNDED ||
                   (sim.status == ProblemStatus::INFEASIBLE && !done);
    } catch (...) {
    }
    if (!resolved) {
        try {
            hypernova::lp::SimplexSolver polisher(tol, hypernova::lp::SimplexOptions{});
            adopt(polisher.solve(cleaned));
        } catch (...) {
        }
    }
    return status;
}

}  // extern "C"
