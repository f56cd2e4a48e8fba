// Batched GPU IPM: many LPs of uneven sizes advanced in lockstep.
//
// Each instance gets HyperNova's standard form and start point exactly as the
// single-LP solver builds them (hn_ipm.cpp, restating interior_point.cpp:202-453);
// the standard forms are packed as one block-diagonal matrix, so every
// sparse product of an iteration is one launch for the whole batch, and the
// per-instance work (reductions, dyn_reg, dense LDL^T, solves, masks) runs in
// the batch kernels of csrc/hn_batch.cu. The host only checks, once per
// iteration, how many instances are still iterating.
#include <omp.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>

#include "hn_lp.hpp"
#include "hn_sm100.h"

namespace hn::lp {

namespace {
void ck(int st, const char* what) {
    if (st != HN_OK) throw std::runtime_error(std::string(what) + ": " + hn_last_error());
}

struct DevBuf {
    void* p = nullptr;
    explicit DevBuf(std::size_t bytes) { ck(hn_malloc(&p, bytes ? bytes : 8), "hn_malloc"); }
    ~DevBuf() {
        if (p) hn_free(p);
    }
    double* d() const { return static_cast<double*>(p); }
    int32_t* i() const { return static_cast<int32_t*>(p); }
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
};

using Clock = std::chrono::steady_clock;
double ms_since(Clock::time_point t) { return std::chrono::duration<double, std::milli>(Clock::now() - t).count(); }
}  // namespace

std::vector<InteriorPointResult> BatchInteriorPointSolver::solve(const std::vector<model::LpProblem>& problems,
                                                                 const std::vector<WarmStart>* warm) {
    const auto start = Clock::now();
    const auto& O = options_;
    const std::size_t K = problems.size();
    std::vector<InteriorPointResult> results(K);
    if (K == 0) return results;
    stats_ = BatchStats{};
    try {
        PackedForm pf;
        build_forms(problems, O.feasibility_tol, pf, warm, O.warm_start_floor);
        stats_.forms_ms = ms_since(start);
        const std::size_t m = pf.row_off.back(), n = pf.col_off.back();
        stats_.rows = m;
        stats_.cols = n;
        stats_.nnz = pf.val.size();
        ck(hn_init(O.device), "hn_init");
        hn_csr* M = nullptr;
        ck(hn_csr_create((int64_t)m, (int64_t)n, pf.rp.data(), pf.ci.data(), pf.val.data(), 0, &M), "hn_csr_create");
        std::unique_ptr<hn_csr, int (*)(hn_csr*)> Mh(M, hn_csr_destroy);
        hn_pattern* P = nullptr;
        ck(hn_ada_symbolic(M, &P), "hn_ada_symbolic");
        std::unique_ptr<hn_pattern, int (*)(hn_pattern*)> Ph(P, hn_pattern_destroy);
        int64_t pm = 0, pnnz = 0;
        ck(hn_pattern_info(P, &pm, &pnnz), "hn_pattern_info");
        stats_.nnz_normal = (std::size_t)pnnz;
        hn_batch* B = nullptr;
        ck(hn_batch_create((int64_t)K, pf.row_off.data(), pf.col_off.data(), P, &B), "hn_batch_create");
        std::unique_ptr<hn_batch, int (*)(hn_batch*)> Bh(B, hn_batch_destroy);

        DevBuf x(8 * n), z(8 * n), lam(8 * m), b(8 * m), c(8 * n), mx(8 * m), rp(8 * m), rd(8 * n), D(8 * n),
            Drd(8 * n), rhs_pred(8 * m), rhs(8 * m), dlam(8 * m), dx(8 * n), dz(8 * n), zs(8 * n),
            nval(8 * (std::size_t)pnnz), scal(8 * HN_IPM_NSCAL * K), status(4 * K), iters(4 * K);
        void* st = nullptr;
        ck(hn_memcpy_h2d(x.p, pf.x0.data(), 8 * n, st), "H2D");
        ck(hn_memcpy_h2d(z.p, pf.z0.data(), 8 * n, st), "H2D");
        ck(hn_memcpy_h2d(lam.p, pf.lam0.data(), 8 * m, st), "H2D");
        ck(hn_memcpy_h2d(b.p, pf.rhs.data(), 8 * m, st), "H2D");
        ck(hn_memcpy_h2d(c.p, pf.c.data(), 8 * n, st), "H2D");
        ck(hn_memset(status.p, 0, 4 * K, st), "memset");
        ck(hn_memset(iters.p, 0, 4 * K, st), "memset");
        ck(hn_memset(scal.p, 0, 8 * HN_IPM_NSCAL * K, st), "memset");
        // relative KKT residual per instance and tightening past the reference's rule
        DevBuf ru(8 * m), cu(8 * n), koff(8 * K);
        ck(hn_memcpy_h2d(ru.p, pf.ru.data(), 8 * m, st), "H2D");
        ck(hn_memcpy_h2d(cu.p, pf.cu.data(), 8 * n, st), "H2D");
        ck(hn_memcpy_h2d(koff.p, pf.offset.data(), 8 * K, st), "H2D");
        ck(hn_batch_set_kkt(B, ru.d(), cu.d(), koff.d(), O.kkt_tol, O.kkt_extra_iterations), "hn_batch_set_kkt");
        std::vector<int32_t> hstatus(K), hiters(K);
        auto read_status = [&]() {
            ck(hn_memcpy_d2h(hstatus.data(), status.p, 4 * K, st), "D2H status");
            std::size_t running = 0;
            for (int32_t v : hstatus) running += (v == 0);
            return running;
        };
        stats_.setup_ms = ms_since(start) - stats_.forms_ms;
        const int max_it = O.max_iterations;
        int iter = 0;
        bool time_up = false;
        for (iter = 0; iter < max_it; ++iter) {
            if (O.time_limit_seconds > 0.0 && ms_since(start) >= O.time_limit_seconds * 1e3) {
                time_up = true;
                break;
            }
            ck(hn_batch_residuals(B, M, x.d(), lam.d(), z.d(), b.d(), c.d(), mx.d(), rp.d(), rd.d(), D.d(), Drd.d(),
                                  scal.d(), status.i(), iters.i(), iter, O.convergence_tol, O.complementarity_tol, st),
               "hn_batch_residuals");
            const std::size_t running = read_status();
            stats_.running_per_iter.push_back(running);
            if (running == 0) break;
            auto tf = Clock::now();
            ck(hn_batch_factor(B, D.d(), O.regularization, O.singular_tol, nval.d(), status.i(), st),
               "hn_batch_factor");
            ck(hn_stream_sync(st), "sync");
            stats_.factor_ms += ms_since(tf);
            ck(hn_ipm_rhs(M, Drd.d(), rp.d(), mx.d(), rhs_pred.d(), st), "hn_ipm_rhs");
            auto ts = Clock::now();
            ck(hn_batch_solve(B, nval.d(), rhs_pred.d(), dlam.d(), status.i(), st), "hn_batch_solve");
            stats_.solve_ms += ms_since(ts);
            ck(hn_ipm_direction(M, dlam.d(), D.d(), rd.d(), x.d(), nullptr, dx.d(), dz.d(), st), "direction");
            ck(hn_batch_steps(B, x.d(), dx.d(), z.d(), dz.d(), dlam.d(), scal.d(), status.i(), st), "steps");
            ck(hn_batch_corrector(B, M, x.d(), dx.d(), z.d(), dz.d(), rhs_pred.d(), zs.d(), rhs.d(), scal.d(),
                                  status.i(), st),
               "corrector");
            ts = Clock::now();
            ck(hn_batch_solve(B, nval.d(), rhs.d(), dlam.d(), status.i(), st), "hn_batch_solve");
            stats_.solve_ms += ms_since(ts);
            ck(hn_ipm_direction(M, dlam.d(), D.d(), rd.d(), x.d(), zs.d(), dx.d(), dz.d(), st), "direction");
            ck(hn_batch_steps(B, x.d(), dx.d(), z.d(), dz.d(), dlam.d(), scal.d(), status.i(), st), "steps");
            ck(hn_batch_update(B, x.d(), dx.d(), z.d(), dz.d(), lam.d(), dlam.d(), scal.d(), status.i(), iters.i(),
                               iter, st),
               "update");
        }
        stats_.iterations = iter;
        // final residuals of the instances still iterating (relaxed acceptance, :727-753)
        DevBuf st_copy(4 * K);
        ck(hn_memcpy_d2d(st_copy.p, status.p, 4 * K, st), "copy status");
        ck(hn_batch_residuals(B, M, x.d(), lam.d(), z.d(), b.d(), c.d(), mx.d(), rp.d(), rd.d(), D.d(), Drd.d(),
                              scal.d(), st_copy.i(), iters.i(), iter, O.convergence_tol, O.complementarity_tol, st),
           "hn_batch_residuals");
        ck(hn_batch_finish(B, x.d(), z.d(), lam.d(), status.i(), iters.i(), st), "hn_batch_finish");
        std::vector<double> hscal(HN_IPM_NSCAL * K), hx(n), hl(m), hkkt(4 * K);
        std::vector<int32_t> href(K);
        ck(hn_batch_kkt(B, hkkt.data(), href.data()), "hn_batch_kkt");
        ck(hn_memcpy_d2h(hl.data(), lam.p, 8 * m, st), "D2H lam");
        ck(hn_memcpy_d2h(hscal.data(), scal.p, 8 * HN_IPM_NSCAL * K, st), "D2H scal");
        ck(hn_memcpy_d2h(hstatus.data(), status.p, 4 * K, st), "D2H status");
        ck(hn_memcpy_d2h(hiters.data(), iters.p, 4 * K, st), "D2H iters");
        ck(hn_memcpy_d2h(hx.data(), x.p, 8 * n, st), "D2H x");
        const double total_ms = ms_since(start);
#pragma omp parallel for schedule(dynamic, 16)
        for (std::size_t i = 0; i < K; ++i) {
            InteriorPointResult& r = results[i];
            const double* s = &hscal[HN_IPM_NSCAL * i];
            bool done = hstatus[i] == 1, numerical_error = hstatus[i] == 7;
            if (hstatus[i] == 0 && s[HN_IPM_NRP] < 1e-4 && s[HN_IPM_NRD] < 1e-4 && s[HN_IPM_MU] < 1e-4) done = true;
            std::vector<double> xi(hx.begin() + pf.col_off[i], hx.begin() + pf.col_off[i + 1]);
            r.primal = to_original_primal_packed(pf, i, xi);
            const model::LpProblem& p = problems[i];
            double obj = 0.0;
            bool obj_ok = std::isfinite(p.obj_offset);
            for (std::size_t j = 0; j < p.num_cols && obj_ok; ++j) {
                const double t = p.objective[j] * r.primal[j];
                if (!std::isfinite(t)) obj_ok = false;
                obj += t;
            }
            if (obj_ok) obj += p.obj_offset;
            if (!obj_ok) numerical_error = true;
            r.objective_value = obj_ok ? obj : 0.0;
            r.dual.assign(p.num_rows, 0.0);
            r.iterations = (std::size_t)hiters[i];
            r.nnz_normal = 0;
            original_duals_packed(pf, i, p, hl.data() + pf.row_off[i], r.dual_estimate, r.reduced_cost_estimate);
            r.warm_start_used = pf.warm_used[i] != 0;
            r.kkt_default = pf.kkt_default[i];
            r.kkt_warm = pf.kkt_warm[i];
            r.kkt = hkkt[4 * i];
            r.kkt_primal = hkkt[4 * i + 1];
            r.kkt_dual = hkkt[4 * i + 2];
            r.kkt_gap = hkkt[4 * i + 3];
            r.reference_iterations = href[i];
            r.solve_time_ms = total_ms;
            const bool feasible_incumbent = s[HN_IPM_NRP] <= O.feasibility_tol;
            r.status = numerical_error ? model::ProblemStatus::NUMERICAL_ERROR
                       : done          ? model::ProblemStatus::OPTIMAL
                       : feasible_incumbent ? model::ProblemStatus::SUBOPTIMAL
                       : time_up            ? model::ProblemStatus::TIME_LIMIT
                                            : model::ProblemStatus::ITER_LIMIT;
        }
        stats_.total_ms = ms_since(start);
    } catch (const std::exception& e) {
        for (auto& r : results) {
            r.status = model::ProblemStatus::NUMERICAL_ERROR;
            r.error = e.what();
        }
        stats_.error = e.what();
    }
    return results;
}

}  // namespace hn::lp
