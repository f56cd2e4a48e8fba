// Host-side LP types and the GPU interior-point solver.
//
// The solver mirrors HyperNova's lp::InteriorPointSolver
// (core/lp/interior_point.hpp:16-54, interior_point.cpp:402-886): the same
// options, statuses, standard form, starting point, Mehrotra predictor-
// corrector steps and exit logic, with every vector resident on the B200 and
// the iteration's sparse and elementwise work in the sm_100a library
// (include/hn_sm100.h). The normal-equation factorisation stays on the host
// (dense LDL^T with the reference's pivot clamp, hn_ldlt.cpp).
#pragma once

#include <cstddef>
#include <cstdint>
#include <functional>
#include <limits>
#include <memory>
#include <string>
#include <vector>

namespace hn::model {

// Same enumerators, same order as hypernova::model (core/model/problem.hpp:24-45).
enum class ConstraintSense { LE, GE, EQ };
enum class ObjectiveSense { MINIMIZE, MAXIMIZE };
enum class ProblemStatus {
    UNKNOWN,
    OPTIMAL,
    INFEASIBLE,
    UNBOUNDED,
    SUBOPTIMAL,
    TIME_LIMIT,
    ITER_LIMIT,
    NUMERICAL_ERROR,
    INTERRUPTED
};

// The parts of model::Problem the IPM reads (problem.hpp:79-93): constraint
// matrix as CSR, per-variable bounds and costs, per-row sense and rhs.
struct LpProblem {
    std::size_t num_rows = 0;
    std::size_t num_cols = 0;
    std::vector<std::size_t> row_ptr{0};
    std::vector<std::size_t> col_indices;
    std::vector<double> values;
    std::vector<double> objective;
    std::vector<double> lower;
    std::vector<double> upper;
    std::vector<ConstraintSense> sense;
    std::vector<double> rhs;
    ObjectiveSense obj_sense = ObjectiveSense::MINIMIZE;
    double obj_offset = 0.0;
};

}  // namespace hn::model

namespace hn::lp {

// A starting point in the original space of the minimisation form (the
// objective negated for a maximisation): x (num_cols), y (num_rows) and s
// (num_cols) with A^T y + s = c at a dual-feasible point. y or s may be empty
// (y = 0; s = c - A^T y). No counterpart in the reference, whose IPM always
// starts from Mehrotra's default point (interior_point.cpp:443-453).
struct WarmStart {
    std::vector<double> x, y, s;
    bool empty() const { return x.empty(); }
};

struct InteriorPointOptions {
    int max_iterations = 100;
    double time_limit_seconds = 0.0;
    double convergence_tol = 1e-8;
    double complementarity_tol = 1e-8;
    double regularization = 1e-8;
    // Tolerances the reference takes from ToleranceConfig::industrial_defaults
    // (core/numerical/tolerance.hpp:60-75).
    double feasibility_tol = 1e-9;
    double singular_tol = 1e-10;
    std::function<bool()> interrupt_callback;
    int device = 0;
    bool verbose = false;
    // Warm start: mapped to the scaled standard form, shifted to strict
    // interiority (Mehrotra's heuristic, with the final shift at least
    // warm_start_floor times the default start's entries) and used only when
    // its KKT residual is below the default start's.
    WarmStart initial_point;
    double warm_start_floor = 1e-2;
    // Normal-matrix factorisation on the host: 0 auto (dense LDL^T up to
    // 12,000 rows, sparse LDL^T above), 1 dense, 2 sparse (SparseLDLT).
    int factorization = 0;
    // Tightening past the reference's stop (no counterpart in the reference,
    // whose absolute tests on the scaled form can leave a relative duality
    // gap above 1e-8): once those tests hold, the solve keeps iterating until
    // the relative KKT residual of the unscaled LP (hn_ipm_kkt) is <= kkt_tol
    // or kkt_extra_iterations more iterations have run, and returns the
    // better of that iterate and the one the reference's rule accepted. The
    // status is the reference rule's. kkt_tol <= 0: the reference's rule alone.
    double kkt_tol = 1e-8;
    int kkt_extra_iterations = 10;
};

struct InteriorPointResult {
    model::ProblemStatus status = model::ProblemStatus::UNKNOWN;
    double objective_value = 0.0;
    std::vector<double> primal;
    std::vector<double> dual;
    std::size_t iterations = 0;
    double solve_time_ms = 0.0;
    // phase times (ms) of the whole solve
    double device_ms = 0.0;
    double factor_ms = 0.0;
    double solve_ms = 0.0;
    std::size_t nnz_normal = 0;
    // start point: relative KKT residual of the default start and of the
    // warm start (0 when none was given), and which one was used
    bool warm_start_used = false;
    double kkt_default = 0.0, kkt_warm = 0.0;
    // the barrier's dual estimate in the original space of the minimisation
    // form (A^T y + s = c): the reference's barrier leaves `dual` zero and
    // fills it only through crossover, so `dual` stays zero here and the
    // estimate is reported beside it (a WarmStart for a related LP)
    std::vector<double> dual_estimate, reduced_cost_estimate;
    // relative KKT residual of the returned iterate on the unscaled LP:
    // max of the primal, dual and gap parts (hn_ipm_kkt), NaN if unmeasured;
    // reference_iterations: the iteration at which the reference's stopping
    // rule first held (-1: never; iterations - reference_iterations extra
    // iterations tightened the result)
    double kkt = std::numeric_limits<double>::quiet_NaN();
    double kkt_primal = kkt, kkt_dual = kkt, kkt_gap = kkt;
    long reference_iterations = -1;
    std::string error;
};

class InteriorPointSolver {
public:
    explicit InteriorPointSolver(const InteriorPointOptions& options = InteriorPointOptions())
        : options_(options) {}
    InteriorPointResult solve(const model::LpProblem& problem);
    const InteriorPointOptions& options() const { return options_; }
    void set_options(const InteriorPointOptions& o) { options_ = o; }

private:
    InteriorPointOptions options_;
};

// ---- batched solver ----
namespace detail {
struct StandardForm;
}

// Standard forms of a batch packed block-diagonally (instance i: rows
// row_off[i]..row_off[i+1], columns col_off[i]..col_off[i+1]) with their start
// points; the matrix in the reference's CSR layout.
struct PackedForm {
    std::vector<int64_t> row_off{0}, col_off{0};
    std::vector<uint64_t> rp{0}, ci;
    std::vector<double> val, rhs, c, x0, z0, lam0;
    std::vector<std::shared_ptr<detail::StandardForm>> forms;
    std::vector<char> warm_used;
    std::vector<double> kkt_default, kkt_warm;
    // unscale factors of the packed rows / columns and each instance's
    // objective constant, for the relative KKT residual (hn_ipm_kkt)
    std::vector<double> ru, cu, offset;
};
// warm: empty, or one (possibly empty) WarmStart per problem
void build_forms(const std::vector<model::LpProblem>& problems, double feas_tol, PackedForm& out,
                 const std::vector<WarmStart>* warm = nullptr, double warm_floor = 1e-2);
std::vector<double> to_original_primal_packed(const PackedForm& pf, std::size_t i, const std::vector<double>& y);
// y = the standard form's multipliers of the original rows mapped back, s = c - A^T y
// (minimisation form); empty when the standard form dropped duplicate rows.
void original_duals_packed(const PackedForm& pf, std::size_t i, const model::LpProblem& p, const double* lam,
                           std::vector<double>& y, std::vector<double>& s);

struct BatchStats {
    std::size_t rows = 0, cols = 0, nnz = 0, nnz_normal = 0;
    int iterations = 0;
    double total_ms = 0.0, factor_ms = 0.0, solve_ms = 0.0;
    double forms_ms = 0.0, setup_ms = 0.0;  // host standard forms and start points; device matrix, pattern, batch
    std::vector<std::size_t> running_per_iter;
    std::string error;
};

// Many LPs advanced in lockstep on the GPU (csrc/hn_batch.cu); each result
// has the meaning of InteriorPointSolver::solve's for its instance.
class BatchInteriorPointSolver {
public:
    explicit BatchInteriorPointSolver(const InteriorPointOptions& options = InteriorPointOptions())
        : options_(options) {}
    std::vector<InteriorPointResult> solve(const std::vector<model::LpProblem>& problems,
                                           const std::vector<WarmStart>* warm = nullptr);
    const BatchStats& stats() const { return stats_; }

private:
    InteriorPointOptions options_;
    BatchStats stats_;
};

// Dense LDL^T of a symmetric m x m matrix (lower triangle, row-major) with the
// pivot rule of SparseCholesky::numeric_factorization
// (core/numerical/factorization.cpp:1299-1305): a pivot <= singular_tol is
// replaced by singular_tol. Multithreaded (OpenMP), blocked right-looking.
class DenseLDLT {
public:
    // a: m*m row-major; only the lower triangle is read; overwritten by L.
    bool factorize(std::vector<double>& a, std::size_t m, double singular_tol);
    void solve(std::vector<double>& x) const;  // in place
    std::size_t size() const { return m_; }
    bool singular() const { return singular_; }

private:
    std::vector<double> L_;
    std::vector<double> D_;
    std::size_t m_ = 0;
    bool singular_ = false;
};

// Sparse LDL^T (hn_sparse_ldlt.cpp): approximate-minimum-degree ordering,
// supernodes, multifrontal numerics with the reference's pivot clamp.
// analyze() takes the symmetric pattern with both triangles (the layout of
// the IPM's normal matrix); factorize() the values in that pattern.
class SparseLDLT {
public:
    void analyze(std::size_t m, const uint64_t* rp, const uint64_t* ci);
    bool factorize(const double* val, double singular_tol);  // false when a pivot was clamped
    void solve(std::vector<double>& x) const;                // in place
    std::size_t size() const { return m_; }
    std::size_t nnz_L() const { return nnz_L_; }              // strictly lower entries of L
    std::size_t supernodes() const { return snode_start_.empty() ? 0 : snode_start_.size() - 1; }
    bool singular() const { return singular_; }
    const std::vector<int>& perm() const { return perm_; }   // new -> old

private:
    std::size_t m_ = 0, nnz_L_ = 0;
    std::vector<int> perm_, iperm_, parent_, snode_start_, snode_of_, snode_parent_, srows_;
    std::vector<std::size_t> srows_off_, panel_off_, amap_off_;
    std::vector<std::pair<uint64_t, std::size_t>> amap_;  // (input entry, front position)
    std::vector<double> L_, D_;
    bool analyzed_ = false, factored_ = false, singular_ = false;
};
// ordering alone: pattern of a symmetric matrix (both triangles), new -> old
std::vector<int> amd_order(int n, const std::vector<int>& rp, const std::vector<int>& ci);

}  // namespace hn::lp
