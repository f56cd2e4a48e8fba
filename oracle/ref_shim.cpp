// extern "C" shim over the HyperNova reference LP stack, compiled from the
// reference's own sources into oracle/_ref/libhnref.so by oracle/Makefile.
//
// TEST INFRASTRUCTURE ONLY: this library is the checker used by tests/, by
// __graft_entry__.smoke() and by bench.py's CPU-baseline leg. Nothing in the
// product (the sm_100a library and its host code) links or calls it.
//
// Every entry point calls the reference's public API unchanged:
//   hnref_backend_*     -> execution::ComputeBackendFactory::create_backend(CPU)
//                          (CPUBackend, core/execution/gpu_backend.cpp:81-139)
//   hnref_multiply      -> numerical::SparseMatrix::multiply (sparse_matrix.cpp:136-159)
//   hnref_tmultiply     -> numerical::SparseMatrix::transpose_multiply (:161-184)
//   hnref_transposed    -> numerical::SparseMatrix::transposed (:84-96)
//   hnref_from_triplets -> numerical::SparseMatrix::from_triplets (:8-53)
//   hnref_cholesky_*    -> numerical::SparseCholesky (factorization.hpp:162-208)
//                          (solve; stats: nnz(L), singular, phase times)
//   hnref_ipm_solve     -> lp::InteriorPointSolver::solve (interior_point.cpp:402-886)
#include "sparse_matrix.hpp"
#include "factorization.hpp"
#include "gpu_backend.hpp"
#include "problem.hpp"
#include "interior_point.hpp"

#include <atomic>
#include <chrono>
#include <cstdint>
#include <cstring>
#include <limits>
#include <memory>
#include <thread>
#include <vector>

using hypernova::numerical::SparseMatrix;
using hypernova::numerical::StorageOrder;
using hypernova::numerical::Triplet;

namespace {

SparseMatrix make_csr(int64_t m, int64_t n, const uint64_t* rp, const uint64_t* ci,
                      const double* val) {
    SparseMatrix A(static_cast<std::size_t>(m), static_cast<std::size_t>(n), StorageOrder::CSR);
    const std::size_t nnz = static_cast<std::size_t>(rp[m]);
    A.mutable_row_ptr().assign(rp, rp + m + 1);
    A.mutable_col_indices().assign(ci, ci + nnz);
    A.mutable_values().assign(val, val + nnz);
    return A;
}

template <class V, class T>
std::vector<V> to_vec(const T* p, std::size_t n) {
    return std::vector<V>(p, p + n);
}

hypernova::execution::IComputeBackend& cpu_backend() {
    static std::unique_ptr<hypernova::execution::IComputeBackend> b =
        hypernova::execution::ComputeBackendFactory::create_backend(
            hypernova::execution::ComputeBackendType::CPU);
    return *b;
}

}  // namespace

extern "C" {

int hnref_backend_spmv(int64_t m, int64_t n, const uint64_t* rp, const uint64_t* ci,
                       const double* val, const double* x, double* y) {
    const std::size_t nnz = static_cast<std::size_t>(rp[m]);
    std::vector<double> v(val, val + nnz), xx(x, x + n), yy;
    std::vector<std::size_t> c(ci, ci + nnz), r(rp, rp + m + 1);
    cpu_backend().spmv(v, c, r, xx, yy);
    std::memcpy(y, yy.data(), sizeof(double) * yy.size());
    return static_cast<int>(yy.size() == static_cast<std::size_t>(m) ? 0 : 1);
}

int hnref_backend_spmm(int64_t m, int64_t n, const uint64_t* rp, const uint64_t* ci,
                       const double* val, const double* B, int64_t k, double* C) {
    const std::size_t nnz = static_cast<std::size_t>(rp[m]);
    std::vector<double> v(val, val + nnz), bb(B, B + n * k), cc;
    std::vector<std::size_t> c(ci, ci + nnz), r(rp, rp + m + 1);
    cpu_backend().spmm(v, c, r, bb, cc, static_cast<std::size_t>(k));
    std::memcpy(C, cc.data(), sizeof(double) * cc.size());
    return 0;
}

double hnref_backend_dot(int64_t n, const double* a, const double* b) {
    return cpu_backend().dot(to_vec<double>(a, n), to_vec<double>(b, n));
}

void hnref_backend_axpy(int64_t n, double alpha, const double* x, double* y) {
    std::vector<double> yy(y, y + n);
    cpu_backend().axpy(alpha, to_vec<double>(x, n), yy);
    std::memcpy(y, yy.data(), sizeof(double) * n);
}

double hnref_backend_norm_inf(int64_t n, const double* v) {
    return cpu_backend().norm_inf(to_vec<double>(v, n));
}

int hnref_multiply(int64_t m, int64_t n, const uint64_t* rp, const uint64_t* ci,
                   const double* val, const double* x, double* y) {
    SparseMatrix A = make_csr(m, n, rp, ci, val);
    std::vector<double> r = A.multiply(to_vec<double>(x, n));
    std::memcpy(y, r.data(), sizeof(double) * r.size());
    return 0;
}

int hnref_tmultiply(int64_t m, int64_t n, const uint64_t* rp, const uint64_t* ci,
                    const double* val, const double* x, double* y) {
    SparseMatrix A = make_csr(m, n, rp, ci, val);
    std::vector<double> r = A.transpose_multiply(to_vec<double>(x, m));
    std::memcpy(y, r.data(), sizeof(double) * r.size());
    return 0;
}

// Returns nnz of A^T; rpT has n+1 entries, ciT/valT have room for nnz(A).
int64_t hnref_transposed(int64_t m, int64_t n, const uint64_t* rp, const uint64_t* ci,
                         const double* val, uint64_t* rpT, uint64_t* ciT, double* valT) {
    SparseMatrix A = make_csr(m, n, rp, ci, val);
    SparseMatrix T = A.transposed();
    for (std::size_t i = 0; i < T.row_ptr().size(); ++i) rpT[i] = T.row_ptr()[i];
    for (std::size_t k = 0; k < T.nnz(); ++k) {
        ciT[k] = T.col_indices()[k];
        valT[k] = T.values()[k];
    }
    return static_cast<int64_t>(T.nnz());
}

// CSR from triplets; returns nnz. rp has rows+1 entries, ci/val room for nt.
int64_t hnref_from_triplets(int64_t rows, int64_t cols, int64_t nt, const uint64_t* ti,
                            const uint64_t* tj, const double* tv, uint64_t* rp, uint64_t* ci,
                            double* val) {
    std::vector<Triplet> t;
    t.reserve(static_cast<std::size_t>(nt));
    for (int64_t k = 0; k < nt; ++k) t.emplace_back(ti[k], tj[k], tv[k]);
    SparseMatrix A = SparseMatrix::from_triplets(rows, cols, t, StorageOrder::CSR);
    for (std::size_t i = 0; i < A.row_ptr().size(); ++i) rp[i] = A.row_ptr()[i];
    for (std::size_t k = 0; k < A.nnz(); ++k) {
        ci[k] = A.col_indices()[k];
        val[k] = A.values()[k];
    }
    return static_cast<int64_t>(A.nnz());
}

// SparseCholesky analyze+factorize then solve N x = b in place (x holds b).
int hnref_cholesky_solve(int64_t m, const uint64_t* rp, const uint64_t* ci, const double* val,
                         double* x) {
    SparseMatrix N = make_csr(m, m, rp, ci, val);
    hypernova::numerical::SparseCholesky ch;
    ch.analyze(N);
    ch.factorize(N);
    std::vector<double> b(x, x + m);
    ch.solve(b);
    std::memcpy(x, b.data(), sizeof(double) * m);
    return ch.stats().singular ? 1 : 0;
}

// SparseCholesky::analyze + factorize on N (CSR, both triangles): nnz(L),
// the singular flag and the two phase times (ms); x (m, may be null) is a
// right-hand side replaced by the solution.
int hnref_cholesky_stats(int64_t m, const uint64_t* rp, const uint64_t* ci, const double* val, int64_t* nnz_L,
                         double* analyze_ms, double* factor_ms, double* x) {
    SparseMatrix N = make_csr(m, m, rp, ci, val);
    hypernova::numerical::SparseCholesky ch;
    const auto t0 = std::chrono::steady_clock::now();
    ch.analyze(N);
    const auto t1 = std::chrono::steady_clock::now();
    ch.factorize(N);
    const auto t2 = std::chrono::steady_clock::now();
    *nnz_L = static_cast<int64_t>(ch.stats().nnz_L);
    *analyze_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
    *factor_ms = std::chrono::duration<double, std::milli>(t2 - t1).count();
    if (x) {
        std::vector<double> b(x, x + m);
        ch.solve(b);
        std::memcpy(x, b.data(), sizeof(double) * m);
    }
    return ch.stats().singular ? 1 : 0;
}

// LP: optimise c^T x subject to rows (sense 0 LE, 1 GE, 2 EQ) with rhs b and
// lb <= x <= ub, through InteriorPointSolver::solve with the given options.
// Returns the ProblemStatus as int; fills obj, iters, time_ms and x (n).
int hnref_ipm_solve(int64_t m, int64_t n, const uint64_t* rp, const uint64_t* ci,
                    const double* val, const double* c, const double* b, const int* sense,
                    const double* lb, const double* ub, int maximize, int max_iter,
                    int crossover, double* obj, int64_t* iters, double* time_ms, double* x) {
    using namespace hypernova::model;
    ProblemBuilder builder("hnref");
    for (int64_t j = 0; j < n; ++j) builder.add_variable(lb[j], ub[j]);
    for (int64_t i = 0; i < m; ++i) {
        std::vector<std::pair<std::size_t, double>> coeffs;
        for (uint64_t k = rp[i]; k < rp[i + 1]; ++k) coeffs.emplace_back(ci[k], val[k]);
        const ConstraintSense s =
            sense[i] == 0 ? ConstraintSense::LE : (sense[i] == 1 ? ConstraintSense::GE
                                                                  : ConstraintSense::EQ);
        builder.add_constraint(coeffs, s, b[i]);
    }
    std::vector<std::pair<std::size_t, double>> objc;
    for (int64_t j = 0; j < n; ++j) objc.emplace_back(j, c[j]);
    builder.set_objective(objc, maximize ? ObjectiveSense::MAXIMIZE : ObjectiveSense::MINIMIZE);
    Problem prob = builder.build();

    hypernova::lp::InteriorPointOptions opts;
    opts.crossover = crossover != 0;
    if (max_iter > 0) opts.max_iterations = max_iter;
    hypernova::lp::InteriorPointSolver solver(
        hypernova::numerical::ToleranceConfig::industrial_defaults(), opts);
    auto r = solver.solve(prob);
    *obj = r.objective_value;
    *iters = static_cast<int64_t>(r.iterations);
    *time_ms = r.solve_time_ms;
    if (x) {
        for (std::size_t j = 0; j < r.primal.size() && j < static_cast<std::size_t>(n); ++j)
            x[j] = r.primal[j];
    }
    return static_cast<int>(r.status);
}

// CPU baseline for one pass of the per-iteration sparse path, farmed over
// `threads` host threads: each thread runs the reference's CPUBackend::spmv and
// SparseMatrix::transpose_multiply on its own row slice of A (slices are
// independent CSR matrices). Returns the wall time in seconds of `reps` passes.
double hnref_bench_spmv_pair(int64_t m, int64_t n, const uint64_t* rp, const uint64_t* ci,
                             const double* val, const double* x, const double* xt, int threads,
                             int reps) {
    if (threads < 1) threads = 1;
    struct Slice {
        std::vector<double> v;
        std::vector<std::size_t> c, r;
        SparseMatrix A;
        std::vector<double> xt_part, y, yt;
    };
    std::vector<Slice> slices(static_cast<std::size_t>(threads));
    const uint64_t nnz = rp[m];
    int64_t row = 0;
    for (int t = 0; t < threads; ++t) {
        const uint64_t target = nnz * static_cast<uint64_t>(t + 1) / static_cast<uint64_t>(threads);
        int64_t end = row;
        while (end < m && rp[end] < target) ++end;
        if (t == threads - 1) end = m;
        Slice& s = slices[t];
        const int64_t rows = end - row;
        s.r.resize(rows + 1);
        for (int64_t i = 0; i <= rows; ++i) s.r[i] = rp[row + i] - rp[row];
        s.c.assign(ci + rp[row], ci + rp[end]);
        s.v.assign(val + rp[row], val + rp[end]);
        s.A = SparseMatrix(static_cast<std::size_t>(rows), static_cast<std::size_t>(n));
        s.A.mutable_row_ptr() = s.r;
        s.A.mutable_col_indices() = s.c;
        s.A.mutable_values() = s.v;
        s.xt_part.assign(xt + row, xt + end);
        row = end;
    }
    std::vector<double> xx(x, x + n);
    auto run = [&](int t) {
        Slice& s = slices[t];
        std::unique_ptr<hypernova::execution::IComputeBackend> b =
            hypernova::execution::ComputeBackendFactory::create_backend(
                hypernova::execution::ComputeBackendType::CPU);
        for (int r = 0; r < reps; ++r) {
            b->spmv(s.v, s.c, s.r, xx, s.y);
            s.yt = s.A.transpose_multiply(s.xt_part);
        }
    };
    auto t0 = std::chrono::steady_clock::now();
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; ++t) pool.emplace_back(run, t);
    for (auto& th : pool) th.join();
    auto t1 = std::chrono::steady_clock::now();
    return std::chrono::duration<double>(t1 - t0).count();
}

}  // extern "C"
