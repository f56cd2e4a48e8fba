// C ABI of the host layer (include/hn_host.h).
#include <algorithm>
#include <climits>
#include <chrono>
#include <cmath>
#include <cstring>
#include <stdexcept>
#include <string>

#include "hn_backend.hpp"
#include "hn_host.h"
#include "hn_lp.hpp"
#include "hn_read.hpp"
#include "hn_sm100.h"

namespace {
thread_local std::string g_err;

template <class F>
int wrap(F&& f) {
    try {
        f();
        return HN_OK;
    } catch (const std::invalid_argument& e) {
        g_err = e.what();
        return HN_ERR_INVALID_ARG;
    } catch (const std::exception& e) {
        g_err = e.what();
        return HN_ERR_CUDA;
    }
}

template <class T>
std::vector<T> vec(const T* p, int64_t n) {
    return n > 0 ? std::vector<T>(p, p + n) : std::vector<T>();
}
}  // namespace

struct hn_backend {
    hn::execution::B200Backend be;
    explicit hn_backend(int d) : be(d) {}
};

extern "C" {

void hn_ipm_default_options(hn_ipm_options* o) {
    o->max_iterations = 100;
    o->time_limit_seconds = 0.0;
    o->convergence_tol = 1e-8;
    o->complementarity_tol = 1e-8;
    o->regularization = 1e-8;
    o->device = 0;
    o->verbose = 0;
    o->interrupt_cb = nullptr;
    o->interrupt_user = nullptr;
    o->initial_x = nullptr;
    o->initial_y = nullptr;
    o->initial_s = nullptr;
    o->warm_start_floor = 1e-2;
    o->factorization = 0;
    o->kkt_tol = 1e-8;
    o->kkt_extra_iterations = 10;
}

const char* hn_host_last_error(void) { return g_err.c_str(); }

int hn_amd_order(int64_t m, const uint64_t* rp, const uint64_t* ci, int64_t* perm) {
    return wrap([&] {
        if (m < 0 || m >= INT32_MAX || !rp || (m > 0 && !perm)) throw std::invalid_argument("hn_amd_order: bad arguments");
        std::vector<int> r(m + 1), c(rp[m]);
        for (int64_t i = 0; i <= m; ++i) r[i] = static_cast<int>(rp[i]);
        for (uint64_t k = 0; k < rp[m]; ++k) {
            if (ci[k] >= static_cast<uint64_t>(m)) throw std::invalid_argument("hn_amd_order: column out of range");
            c[k] = static_cast<int>(ci[k]);
        }
        const auto ord = hn::lp::amd_order(static_cast<int>(m), r, c);
        for (int64_t k = 0; k < m; ++k) perm[k] = ord[k];
    });
}

int hn_sparse_ldlt_solve(int64_t m, const uint64_t* rp, const uint64_t* ci, const double* val, double singular_tol,
                         int64_t nrhs, double* x, hn_sparse_ldlt_stats* stats) {
    return wrap([&] {
        if (m < 0 || m >= INT32_MAX || !rp || (m > 0 && (!val || !ci)) || nrhs < 0 || (nrhs > 0 && !x))
            throw std::invalid_argument("hn_sparse_ldlt_solve: bad arguments");
        for (uint64_t k = 0; k < rp[m]; ++k)
            if (ci[k] >= static_cast<uint64_t>(m)) throw std::invalid_argument("hn_sparse_ldlt_solve: column out of range");
        hn::lp::SparseLDLT f;
        const auto t0 = std::chrono::steady_clock::now();
        f.analyze(static_cast<std::size_t>(m), rp, ci);
        const auto t1 = std::chrono::steady_clock::now();
        f.factorize(val, singular_tol);
        const auto t2 = std::chrono::steady_clock::now();
        std::vector<double> b(static_cast<std::size_t>(m));
        for (int64_t r = 0; r < nrhs; ++r) {
            std::memcpy(b.data(), x + r * m, sizeof(double) * m);
            f.solve(b);
            std::memcpy(x + r * m, b.data(), sizeof(double) * m);
        }
        if (stats) {
            stats->nnz_L = static_cast<int64_t>(f.nnz_L());
            stats->supernodes = static_cast<int64_t>(f.supernodes());
            stats->singular = f.singular() ? 1 : 0;
            stats->analyze_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
            stats->factor_ms = std::chrono::duration<double, std::milli>(t2 - t1).count();
        }
    });
}

// The starting basis HyperNova's crossover offers its simplex polisher
// (interior_point.cpp:825-842), from a barrier endpoint x: a variable within
// 1e-6 (1 + max(|lb|, |ub|)) of a bound is nonbasic there (-1 lower, +1
// upper, lower tested first), every other one a basic candidate (0). With an
// infinite bound the tolerance is infinite, as in the reference: a variable
// with a finite lower and no upper bound is always offered at its lower
// bound. IEEE arithmetic as the reference's (no contraction).
int hn_crossover_basis(int64_t n, const double* x, const double* lb, const double* ub, int* var_status) {
    if (n < 0 || (n > 0 && (!x || !lb || !ub || !var_status))) {
        g_err = "hn_crossover_basis: bad arguments";
        return HN_ERR_INVALID_ARG;
    }
    for (int64_t j = 0; j < n; ++j) {
        const double at_tol = 1e-6 * (1.0 + std::max(std::abs(lb[j]), std::abs(ub[j])));
        var_status[j] = x[j] <= lb[j] + at_tol ? -1 : (x[j] >= ub[j] - at_tol ? 1 : 0);
    }
    return HN_OK;
}
}  // extern "C"

namespace hn {
void set_host_error(const std::string& msg) { g_err = msg; }
}  // namespace hn

extern "C" {

int hn_lp_solve(int64_t m, int64_t n, const uint64_t* rp, const uint64_t* ci, const double* val, const double* c,
                const double* b, const int* sense, const double* lb, const double* ub, int maximize,
                double obj_offset, const hn_ipm_options* opt, hn_ipm_result* res, double* x_out, double* y_out,
                double* s_out) {
    return wrap([&] {
        if (m < 0 || n < 0 || !rp || !res) throw std::invalid_argument("bad arguments");
        hn::model::LpProblem p;
        p.num_rows = (std::size_t)m;
        p.num_cols = (std::size_t)n;
        p.row_ptr.assign(rp, rp + m + 1);
        p.col_indices.assign(ci, ci + rp[m]);
        p.values.assign(val, val + rp[m]);
        p.objective = vec(c, n);
        p.lower = vec(lb, n);
        p.upper = vec(ub, n);
        p.rhs = vec(b, m);
        for (int64_t i = 0; i < m; ++i)
            p.sense.push_back(sense[i] == 0 ? hn::model::ConstraintSense::LE
                                            : sense[i] == 1 ? hn::model::ConstraintSense::GE
                                                            : hn::model::ConstraintSense::EQ);
        p.obj_sense = maximize ? hn::model::ObjectiveSense::MAXIMIZE : hn::model::ObjectiveSense::MINIMIZE;
        p.obj_offset = obj_offset;
        hn::lp::InteriorPointOptions o;
        if (opt) {
            o.max_iterations = opt->max_iterations;
            o.time_limit_seconds = opt->time_limit_seconds;
            o.convergence_tol = opt->convergence_tol;
            o.complementarity_tol = opt->complementarity_tol;
            o.regularization = opt->regularization;
            o.device = opt->device;
            o.verbose = opt->verbose != 0;
            if (opt->interrupt_cb) {
                auto cb = opt->interrupt_cb;
                void* user = opt->interrupt_user;
                o.interrupt_callback = [cb, user]() { return cb(user) != 0; };
            }
            o.warm_start_floor = opt->warm_start_floor;
            o.factorization = opt->factorization;
            o.kkt_tol = opt->kkt_tol;
            o.kkt_extra_iterations = opt->kkt_extra_iterations;
            if (opt->initial_x) {
                o.initial_point.x = vec(opt->initial_x, n);
                if (opt->initial_y) o.initial_point.y = vec(opt->initial_y, m);
                if (opt->initial_s) o.initial_point.s = vec(opt->initial_s, n);
            }
        }
        hn::lp::InteriorPointSolver solver(o);
        auto r = solver.solve(p);
        res->status = static_cast<int>(r.status);
        res->iterations = (int64_t)r.iterations;
        res->objective = r.objective_value;
        res->solve_time_ms = r.solve_time_ms;
        res->device_ms = r.device_ms;
        res->factor_ms = r.factor_ms;
        res->solve_ms = r.solve_ms;
        res->nnz_normal = (int64_t)r.nnz_normal;
        res->warm_start_used = r.warm_start_used ? 1 : 0;
        res->kkt_default = r.kkt_default;
        res->kkt_warm = r.kkt_warm;
        res->kkt = r.kkt;
        res->kkt_primal = r.kkt_primal;
        res->kkt_dual = r.kkt_dual;
        res->kkt_gap = r.kkt_gap;
        res->reference_iterations = (int64_t)r.reference_iterations;
        if (x_out && r.primal.size() == (std::size_t)n) std::memcpy(x_out, r.primal.data(), 8 * n);
        if (y_out && r.dual_estimate.size() == (std::size_t)m) std::memcpy(y_out, r.dual_estimate.data(), 8 * m);
        if (s_out && r.reduced_cost_estimate.size() == (std::size_t)n)
            std::memcpy(s_out, r.reduced_cost_estimate.data(), 8 * n);
        g_err = r.error;
    });
}

int hn_lp_solve_batch(int64_t K, const int64_t* row_off, const int64_t* col_off, const int64_t* nnz_off,
                      const uint64_t* rp, const uint64_t* ci, const double* val, const double* c, const double* b,
                      const int* sense, const double* lb, const double* ub, const int* maximize,
                      const double* obj_offset, const hn_ipm_options* opt, int* status, double* objective,
                      int64_t* iterations, double* x_out, hn_batch_stats* stats, int* warm_used, double* y_out,
                      double* s_out, double* kkt_out, int64_t* reference_iterations) {
    return wrap([&] {
        if (K < 0 || !row_off || !col_off || !nnz_off || !status || !objective || !iterations)
            throw std::invalid_argument("bad arguments");
        std::vector<hn::model::LpProblem> probs((std::size_t)K);
        for (int64_t i = 0; i < K; ++i) {
            hn::model::LpProblem& p = probs[(std::size_t)i];
            const int64_t m = row_off[i + 1] - row_off[i], n = col_off[i + 1] - col_off[i];
            const uint64_t* r = rp + row_off[i] + i;
            const int64_t e0 = nnz_off[i];
            p.num_rows = (std::size_t)m;
            p.num_cols = (std::size_t)n;
            p.row_ptr.assign(r, r + m + 1);
            p.col_indices.assign(ci + e0, ci + e0 + (int64_t)r[m]);
            p.values.assign(val + e0, val + e0 + (int64_t)r[m]);
            p.objective.assign(c + col_off[i], c + col_off[i + 1]);
            p.lower.assign(lb + col_off[i], lb + col_off[i + 1]);
            p.upper.assign(ub + col_off[i], ub + col_off[i + 1]);
            p.rhs.assign(b + row_off[i], b + row_off[i + 1]);
            for (int64_t k = row_off[i]; k < row_off[i + 1]; ++k)
                p.sense.push_back(sense[k] == 0 ? hn::model::ConstraintSense::LE
                                                : sense[k] == 1 ? hn::model::ConstraintSense::GE
                                                                : hn::model::ConstraintSense::EQ);
            p.obj_sense = (maximize && maximize[i]) ? hn::model::ObjectiveSense::MAXIMIZE
                                                    : hn::model::ObjectiveSense::MINIMIZE;
            p.obj_offset = obj_offset ? obj_offset[i] : 0.0;
        }
        hn::lp::InteriorPointOptions o;
        if (opt) {
            o.max_iterations = opt->max_iterations;
            o.time_limit_seconds = opt->time_limit_seconds;
            o.convergence_tol = opt->convergence_tol;
            o.complementarity_tol = opt->complementarity_tol;
            o.regularization = opt->regularization;
            o.device = opt->device;
            o.warm_start_floor = opt->warm_start_floor;
            o.factorization = opt->factorization;
            o.kkt_tol = opt->kkt_tol;
            o.kkt_extra_iterations = opt->kkt_extra_iterations;
        }
        std::vector<hn::lp::WarmStart> warm;
        if (opt && opt->initial_x) {
            warm.resize((std::size_t)K);
            for (int64_t i = 0; i < K; ++i) {
                auto& w = warm[(std::size_t)i];
                w.x = vec(opt->initial_x + col_off[i], col_off[i + 1] - col_off[i]);
                if (opt->initial_y) w.y = vec(opt->initial_y + row_off[i], row_off[i + 1] - row_off[i]);
                if (opt->initial_s) w.s = vec(opt->initial_s + col_off[i], col_off[i + 1] - col_off[i]);
            }
        }
        hn::lp::BatchInteriorPointSolver solver(o);
        auto res = solver.solve(probs, warm.empty() ? nullptr : &warm);
        for (int64_t i = 0; i < K; ++i) {
            const auto& r = res[(std::size_t)i];
            status[i] = static_cast<int>(r.status);
            objective[i] = r.objective_value;
            iterations[i] = (int64_t)r.iterations;
            if (warm_used) warm_used[i] = r.warm_start_used ? 1 : 0;
            if (kkt_out) {
                kkt_out[4 * i] = r.kkt;
                kkt_out[4 * i + 1] = r.kkt_primal;
                kkt_out[4 * i + 2] = r.kkt_dual;
                kkt_out[4 * i + 3] = r.kkt_gap;
            }
            if (reference_iterations) reference_iterations[i] = (int64_t)r.reference_iterations;
            const auto& pi = probs[(std::size_t)i];
            if (y_out && r.dual_estimate.size() == pi.num_rows)
                std::memcpy(y_out + row_off[i], r.dual_estimate.data(), 8 * pi.num_rows);
            if (s_out && r.reduced_cost_estimate.size() == pi.num_cols)
                std::memcpy(s_out + col_off[i], r.reduced_cost_estimate.data(), 8 * pi.num_cols);
            if (x_out && r.primal.size() == probs[(std::size_t)i].num_cols)
                std::memcpy(x_out + col_off[i], r.primal.data(), 8 * r.primal.size());
        }
        const auto& S = solver.stats();
        if (stats) {
            stats->rows = (int64_t)S.rows;
            stats->cols = (int64_t)S.cols;
            stats->nnz = (int64_t)S.nnz;
            stats->nnz_normal = (int64_t)S.nnz_normal;
            stats->iterations = S.iterations;
            stats->total_ms = S.total_ms;
            stats->factor_ms = S.factor_ms;
            stats->solve_ms = S.solve_ms;
            stats->forms_ms = S.forms_ms;
            stats->setup_ms = S.setup_ms;
        }
        if (!S.error.empty()) throw std::runtime_error(S.error);
    });
}

int hn_be_create(int device, hn_backend** out) {
    return wrap([&] {
        auto* b = new hn_backend(device);
        b->be.initialize();
        if (!b->be.is_available()) {
            std::string e = b->be.last_error();
            delete b;
            throw std::runtime_error("B200 backend unavailable: " + e);
        }
        *out = b;
    });
}

int hn_be_destroy(hn_backend* be) {
    return wrap([&] { delete be; });
}

int hn_be_spmv(hn_backend* be, int64_t m, int64_t nnz, const uint64_t* rp, const uint64_t* ci, const double* val,
               int64_t nx, const double* x, double* y) {
    return wrap([&] {
        std::vector<double> v = vec(val, nnz), xx = vec(x, nx), yy;
        std::vector<std::size_t> c(ci, ci + nnz), r(rp, rp + m + 1);
        be->be.spmv(v, c, r, xx, yy);
        std::memcpy(y, yy.data(), 8 * yy.size());
    });
}

int hn_be_spmv_t(hn_backend* be, int64_t m, int64_t n, int64_t nnz, const uint64_t* rp, const uint64_t* ci,
                 const double* val, const double* x, double* y) {
    return wrap([&] {
        std::vector<double> v = vec(val, nnz), xx = vec(x, m), yy;
        std::vector<std::size_t> c(ci, ci + nnz), r(rp, rp + m + 1);
        be->be.spmv_t(v, c, r, (std::size_t)n, xx, yy);
        std::memcpy(y, yy.data(), 8 * yy.size());
    });
}

int hn_be_spmm(hn_backend* be, int64_t m, int64_t nnz, const uint64_t* rp, const uint64_t* ci, const double* val,
               int64_t nb, const double* B, int64_t k, double* C) {
    return wrap([&] {
        std::vector<double> v = vec(val, nnz), bb = vec(B, nb * k), cc;
        std::vector<std::size_t> c(ci, ci + nnz), r(rp, rp + m + 1);
        be->be.spmm(v, c, r, bb, cc, (std::size_t)k);
        std::memcpy(C, cc.data(), 8 * cc.size());
    });
}

int hn_be_dot(hn_backend* be, int64_t n, const double* a, const double* b, double* out) {
    return wrap([&] { *out = be->be.dot(vec(a, n), vec(b, n)); });
}

int hn_be_axpy(hn_backend* be, int64_t n, double alpha, const double* x, double* y) {
    return wrap([&] {
        std::vector<double> yy = vec(y, n);
        be->be.axpy(alpha, vec(x, n), yy);
        std::memcpy(y, yy.data(), 8 * n);
    });
}

int hn_be_norm_inf(hn_backend* be, int64_t n, const double* v, double* out) {
    return wrap([&] { *out = be->be.norm_inf(vec(v, n)); });
}

int hn_be_kernel_executions(hn_backend* be, uint64_t* out) {
    return wrap([&] { *out = be->be.gpu_kernel_executions(); });
}

}  // extern "C"
