// extern "C" shim over the pricing steps of HyperNova's revised simplex,
// compiled against the reference's own simplex.cpp into oracle/_ref/libhnref.so.
//
// TEST INFRASTRUCTURE ONLY (the checker for tests/): nothing in the product
// links or calls it.
//
// The pricing steps are private members of lp::SimplexSolver
// (core/lp/simplex.hpp:107-120), so this translation unit opens the class's
// access to drive them directly on a solver whose state it sets:
//   hnref_price_reduced_costs  -> SimplexSolver::compute_reduced_costs   (simplex.cpp:1225-1233)
//   hnref_price_devex_update   -> SimplexSolver::update_devex_weights    (simplex.cpp:1235-1271)
//   hnref_price_ranked         -> SimplexSolver::ranked_candidates       (simplex.cpp:1283-1308)
//   hnref_price_select         -> SimplexSolver::select_entering_variable (simplex.cpp:1321-1361,
//                                 Bland and Devex/Dantzig branches)
//   hnref_price_edge_weight    -> SimplexSolver::exact_edge_weight       (simplex.cpp:1312-1319) on a
//                                 unit basis: 1 + ||a_j||^2 of the column that the file-local
//                                 extract_column (simplex.cpp:25-35) gathers
// update_devex_weights obtains its row multiplier u = e_leaving^T B^-1 from the
// basis factorisation; a factorisation whose solve_transpose returns a given u
// lets the test drive the step with any u.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <functional>
#include <limits>
#include <memory>
#include <string>
#include <vector>

#include "factorization.hpp"
#include "problem.hpp"
#include "sparse_matrix.hpp"
#include "tolerance.hpp"
#define private public
#include "simplex.hpp"
#undef private

using hypernova::numerical::SparseMatrix;
using hypernova::numerical::StorageOrder;

namespace {

SparseMatrix csr(int64_t m, int64_t n, const uint64_t* rp, const uint64_t* ci, const double* val) {
    SparseMatrix A(static_cast<std::size_t>(m), static_cast<std::size_t>(n), StorageOrder::CSR);
    const std::size_t nnz = static_cast<std::size_t>(rp[m]);
    A.mutable_row_ptr().assign(rp, rp + m + 1);
    A.mutable_col_indices().assign(ci, ci + nnz);
    A.mutable_values().assign(val, val + nnz);
    return A;
}

// A basis factorisation whose transposed solve returns a fixed vector u and
// whose solve is the identity (unit basis).
class FixedRowFactorization : public hypernova::numerical::SparseFactorization {
public:
    explicit FixedRowFactorization(std::vector<double> u) : u_(std::move(u)) {}
    void solve(std::vector<double>&) const override {}
    void solve_transpose(std::vector<double>& x) const override { x = u_; }
    void solve_multiple(std::vector<std::vector<double>>&) const override {}
    hypernova::numerical::FactorizationStats stats() const override { return {}; }
    hypernova::numerical::FactorizationType type() const override {
        return hypernova::numerical::FactorizationType::LU;
    }
    std::unique_ptr<hypernova::numerical::SparseFactorization> clone() const override {
        return std::make_unique<FixedRowFactorization>(u_);
    }

private:
    std::vector<double> u_;
};

}  // namespace

extern "C" {

void hnref_price_reduced_costs(int64_t m, int64_t n, const uint64_t* rp, const uint64_t* ci, const double* val,
                               const double* y, const double* cost, double* rc) {
    hypernova::model::Problem p;
    p.constraint_matrix = csr(m, n, rp, ci, val);
    hypernova::lp::SimplexSolver s;
    s.problem_ = &p;
    s.dual_solution_.assign(y, y + m);
    s.phase_cost_.assign(cost, cost + n);
    s.nonbasis_.assign(static_cast<std::size_t>(n), 0);
    s.reduced_costs_.assign(static_cast<std::size_t>(n), 0.0);
    s.compute_reduced_costs();
    std::copy(s.reduced_costs_.begin(), s.reduced_costs_.end(), rc);
}

void hnref_price_devex_update(int64_t m, int64_t n, const uint64_t* rp, const uint64_t* ci, const double* val,
                              const double* u, const int32_t* nonbasis, double* weights) {
    hypernova::model::Problem p;
    p.constraint_matrix = csr(m, n, rp, ci, val);
    hypernova::lp::SimplexOptions o;
    o.pricing = hypernova::lp::PricingStrategy::DEVEX;
    hypernova::lp::SimplexSolver s(hypernova::numerical::ToleranceConfig::industrial_defaults(), o);
    s.problem_ = &p;
    s.basis_.assign(static_cast<std::size_t>(m), 0);
    s.nonbasis_.assign(nonbasis, nonbasis + n);
    s.reduced_costs_.assign(static_cast<std::size_t>(n), 0.0);
    s.pricing_weights_.assign(weights, weights + n);
    s.basis_factorization_ = std::make_unique<FixedRowFactorization>(std::vector<double>(u, u + m));
    s.update_devex_weights(0);
    std::copy(s.pricing_weights_.begin(), s.pricing_weights_.end(), weights);
}

// ranked_candidates: writes up to `cap` indices, returns the full count.
int64_t hnref_price_ranked(int64_t n, const double* rc, const double* w, const int32_t* nonbasis,
                           const uint8_t* artificial, int phase1, int maximize, int64_t cap, int64_t* out) {
    hypernova::lp::SimplexSolver s;
    s.reduced_costs_.assign(rc, rc + n);
    s.pricing_weights_.assign(w, w + n);
    s.nonbasis_.assign(nonbasis, nonbasis + n);
    s.artificial_cols_.assign(artificial, artificial + n);
    s.phase1_active_ = phase1 != 0;
    const std::vector<std::size_t> c = s.ranked_candidates(maximize != 0);
    for (std::size_t k = 0; k < c.size() && static_cast<int64_t>(k) < cap; ++k) out[k] = static_cast<int64_t>(c[k]);
    return static_cast<int64_t>(c.size());
}

// select_entering_variable with bland_rule on (rule 0) or Devex pricing (rule 1).
int64_t hnref_price_select(int64_t n, const double* rc, const double* w, const int32_t* nonbasis,
                           const uint8_t* artificial, int phase1, int maximize, int rule) {
    hypernova::lp::SimplexOptions o;
    o.bland_rule = rule == 0;
    o.pricing = hypernova::lp::PricingStrategy::DEVEX;
    hypernova::lp::SimplexSolver s(hypernova::numerical::ToleranceConfig::industrial_defaults(), o);
    s.reduced_costs_.assign(rc, rc + n);
    s.pricing_weights_.assign(w, w + n);
    s.nonbasis_.assign(nonbasis, nonbasis + n);
    s.artificial_cols_.assign(artificial, artificial + n);
    s.phase1_active_ = phase1 != 0;
    s.maximize_ = maximize != 0;
    return s.select_entering_variable();
}

double hnref_price_edge_weight(int64_t m, int64_t n, const uint64_t* rp, const uint64_t* ci, const double* val,
                               int64_t var) {
    hypernova::model::Problem p;
    p.constraint_matrix = csr(m, n, rp, ci, val);
    hypernova::lp::SimplexSolver s;
    s.problem_ = &p;
    s.basis_factorization_ = std::make_unique<FixedRowFactorization>(std::vector<double>());
    return s.exact_edge_weight(static_cast<std::size_t>(var));
}

}  // extern "C"
