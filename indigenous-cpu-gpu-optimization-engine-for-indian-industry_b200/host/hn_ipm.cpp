// GPU Mehrotra predictor-corrector IPM: host control flow of
// lp::InteriorPointSolver::solve (core/lp/interior_point.cpp:402-886), with
// the iterate, residuals, directions, step lengths and A D A^T assembly on
// the B200 (include/hn_sm100.h) and the normal-equation factorisation on the
// host (DenseLDLT, or SparseLDLT above 12,000 rows / on request). Only scalars, N's values and the m-vectors of the two
// normal-equation solves cross PCIe each iteration.
#include <omp.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <unordered_set>

#include "hn_lp.hpp"
#include "hn_sm100.h"

namespace hn::lp {
namespace detail {
// ---- standard form (interior_point.cpp:29-49, 202-373) ----
struct VarInfo {
    std::vector<int> slots;
    std::vector<double> signs;
    std::vector<double> shifts;
    double fixed = 0.0;
    bool is_fixed = false;
};

struct StandardForm {
    std::size_t m = 0, n = 0;
    std::vector<std::size_t> rp, ci;
    std::vector<double> val, rhs, c, col_scale;
    double offset = 0.0;
    std::vector<VarInfo> var_info;
    std::size_t nslots = 0;         // structural columns; the rest are slacks (one entry each)
    std::vector<double> row_mult;   // original row i -> standard row i scaled by this (-gamma for GE)
};

}  // namespace detail
using detail::StandardForm;
using detail::VarInfo;

namespace {

using model::ConstraintSense;
using model::ProblemStatus;

void ck(int st, const char* what) {
    if (st != HN_OK) throw std::runtime_error(std::string(what) + ": " + hn_last_error());
}

struct Trip {
    std::size_t r, c;
    double v;
};

// CSR from triplets with SparseMatrix::from_triplets semantics
// (core/numerical/sparse_matrix.cpp:8-53, 230-262): sort by (row, col),
// sum equal keys, drop exact zero sums.
void csr_from_triplets(std::size_t rows, std::vector<Trip>& t, std::vector<std::size_t>& rp,
                       std::vector<std::size_t>& ci, std::vector<double>& val) {
    std::stable_sort(t.begin(), t.end(), [](const Trip& a, const Trip& b) {
        return a.r != b.r ? a.r < b.r : a.c < b.c;
    });
    rp.assign(rows + 1, 0);
    ci.clear();
    val.clear();
    std::size_t k = 0;
    for (std::size_t i = 0; i < rows; ++i) {
        while (k < t.size() && t[k].r == i) {
            const std::size_t c = t[k].c;
            double s = t[k].v;
            ++k;
            while (k < t.size() && t[k].r == i && t[k].c == c) s += t[k++].v;
            if (s != 0.0) {
                ci.push_back(c);
                val.push_back(s);
            }
        }
        rp[i + 1] = ci.size();
    }
}

// remove_duplicate_rows (interior_point.cpp:79-132): a row equal to an
// earlier one in entries (sorted by column, then value), sense and rhs bits
// is dropped. Rows are compared through a 64-bit hash of that key and then
// exactly (the reference compares decimal string keys of the same fields).
model::LpProblem remove_duplicate_rows(const model::LpProblem& p) {
    if (p.num_rows == 0) return p;
    using Entry = std::pair<std::size_t, double>;
    auto bits = [](double v) {
        std::uint64_t b;
        std::memcpy(&b, &v, 8);
        return b;
    };
    auto row_entries = [&](std::size_t i) {
        std::vector<Entry> ent;
        ent.reserve(p.row_ptr[i + 1] - p.row_ptr[i]);
        for (std::size_t k = p.row_ptr[i]; k < p.row_ptr[i + 1]; ++k) ent.emplace_back(p.col_indices[k], p.values[k]);
        std::sort(ent.begin(), ent.end());
        return ent;
    };
    auto same = [&](const std::vector<Entry>& a, std::size_t ia, const std::vector<Entry>& b, std::size_t ib) {
        if (p.sense[ia] != p.sense[ib] || bits(p.rhs[ia]) != bits(p.rhs[ib]) || a.size() != b.size()) return false;
        for (std::size_t k = 0; k < a.size(); ++k)
            if (a[k].first != b[k].first || bits(a[k].second) != bits(b[k].second)) return false;
        return true;
    };
    std::unordered_map<std::uint64_t, std::vector<std::size_t>> seen;  // hash -> kept rows
    std::vector<std::vector<Entry>> kept_ent;
    std::vector<std::size_t> keep;
    for (std::size_t i = 0; i < p.num_rows; ++i) {
        std::vector<Entry> ent = row_entries(i);
        std::uint64_t h = 0x9e3779b97f4a7c15ull ^ bits(p.rhs[i]) ^ (static_cast<std::uint64_t>(p.sense[i]) << 61);
        for (const Entry& e : ent) {
            h ^= e.first + 0x9e3779b97f4a7c15ull + (h << 6) + (h >> 2);
            h ^= bits(e.second) + 0x9e3779b97f4a7c15ull + (h << 6) + (h >> 2);
        }
        auto& bucket = seen[h];
        bool dup = false;
        for (std::size_t q : bucket)
            if (same(kept_ent[q], keep[q], ent, i)) {
                dup = true;
                break;
            }
        if (dup) continue;
        bucket.push_back(keep.size());
        keep.push_back(i);
        kept_ent.push_back(std::move(ent));
    }
    if (keep.size() == p.num_rows) return p;
    model::LpProblem q = p;
    q.num_rows = keep.size();
    q.row_ptr.assign(1, 0);
    q.col_indices.clear();
    q.values.clear();
    q.sense.clear();
    q.rhs.clear();
    for (std::size_t t = 0; t < keep.size(); ++t) {
        const std::size_t i = keep[t];
        for (const Entry& e : kept_ent[t]) {
            q.col_indices.push_back(e.first);
            q.values.push_back(e.second);
        }
        q.row_ptr.push_back(q.col_indices.size());
        q.sense.push_back(p.sense[i]);
        q.rhs.push_back(p.rhs[i]);
    }
    return q;
}

StandardForm build_standard_form(const model::LpProblem& p, double feas_tol) {
    StandardForm f;
    const std::size_t n = p.num_cols, norig = p.num_rows;
    const bool negate = p.obj_sense == model::ObjectiveSense::MAXIMIZE;
    std::vector<double> cbase(n);
    for (std::size_t j = 0; j < n; ++j) cbase[j] = negate ? -p.objective[j] : p.objective[j];
    f.var_info.resize(n);
    std::size_t nslots = 0, ntle = 0, m_ub = 0;
    for (std::size_t j = 0; j < n; ++j) {
        const double lb = p.lower[j], ub = p.upper[j];
        VarInfo& v = f.var_info[j];
        if (std::isfinite(lb) && std::isfinite(ub) && std::abs(ub - lb) <= feas_tol) {
            v.is_fixed = true;
            v.fixed = lb;
            f.offset += cbase[j] * lb;
        } else if (std::isfinite(lb)) {
            v.slots.push_back(static_cast<int>(nslots++));
            v.signs.push_back(1.0);
            v.shifts.push_back(lb);
            f.offset += cbase[j] * lb;
            if (std::isfinite(ub)) ++m_ub;
        } else if (std::isfinite(ub)) {
            v.slots.push_back(static_cast<int>(nslots++));
            v.signs.push_back(-1.0);
            v.shifts.push_back(ub);
            f.offset += cbase[j] * ub;
        } else {
            v.slots.push_back(static_cast<int>(nslots++));
            v.signs.push_back(1.0);
            v.shifts.push_back(0.0);
            v.slots.push_back(static_cast<int>(nslots++));
            v.signs.push_back(-1.0);
            v.shifts.push_back(0.0);
        }
    }
    for (std::size_t i = 0; i < norig; ++i)
        if (p.sense[i] == ConstraintSense::LE || p.sense[i] == ConstraintSense::GE) ++ntle;
    const std::size_t m_rows = norig + m_ub, ncols = nslots + ntle + m_ub;
    f.nslots = nslots;
    f.m = m_rows;
    f.n = ncols;
    f.rhs.assign(m_rows, 0.0);
    f.c.assign(ncols, 0.0);
    for (std::size_t j = 0; j < n; ++j)
        for (std::size_t s = 0; s < f.var_info[j].slots.size(); ++s)
            f.c[f.var_info[j].slots[s]] = f.var_info[j].signs[s] > 0 ? cbase[j] : -cbase[j];
    std::vector<double> gamma(norig, 1.0);
    for (std::size_t i = 0; i < norig; ++i) {
        double rowmax = 0.0;
        for (std::size_t k = p.row_ptr[i]; k < p.row_ptr[i + 1]; ++k) rowmax = std::max(rowmax, std::abs(p.values[k]));
        if (rowmax > 0.0) gamma[i] = 1.0 / rowmax;
    }
    f.row_mult.resize(norig);
    for (std::size_t i = 0; i < norig; ++i) f.row_mult[i] = p.sense[i] == ConstraintSense::GE ? -gamma[i] : gamma[i];
    std::vector<Trip> trips;
    std::size_t next_slack = nslots;
    for (std::size_t i = 0; i < norig; ++i) {
        double const_i = 0.0;
        const bool flip = p.sense[i] == ConstraintSense::GE;
        for (std::size_t k = p.row_ptr[i]; k < p.row_ptr[i + 1]; ++k) {
            const std::size_t j = p.col_indices[k];
            const double a = gamma[i] * p.values[k];
            const VarInfo& v = f.var_info[j];
            if (v.is_fixed) {
                const_i += a * v.fixed;
            } else {
                for (std::size_t s = 0; s < v.slots.size(); ++s) {
                    trips.push_back({i, static_cast<std::size_t>(v.slots[s]), flip ? -a * v.signs[s] : a * v.signs[s]});
                    const_i += a * v.shifts[s];
                }
            }
        }
        if (p.sense[i] == ConstraintSense::LE || p.sense[i] == ConstraintSense::GE)
            trips.push_back({i, next_slack++, gamma[i]});
        f.rhs[i] = flip ? (-gamma[i] * p.rhs[i] + const_i) : (gamma[i] * p.rhs[i] - const_i);
    }
    std::size_t next_ub_row = norig;
    for (std::size_t j = 0; j < n; ++j) {
        const double lb = p.lower[j], ub = p.upper[j];
        if (std::isfinite(lb) && std::isfinite(ub) && std::abs(ub - lb) > feas_tol) {
            const std::size_t gi = static_cast<std::size_t>(f.var_info[j].slots[0]);
            trips.push_back({next_ub_row, gi, 1.0});
            trips.push_back({next_ub_row, next_slack++, 1.0});
            f.rhs[next_ub_row] = ub - lb;
            ++next_ub_row;
        }
    }
    csr_from_triplets(m_rows, trips, f.rp, f.ci, f.val);
    // column scaling (:346-370)
    f.col_scale.assign(ncols, 1.0);
    std::vector<double> colmax(ncols, 0.0);
    for (std::size_t k = 0; k < f.val.size(); ++k) colmax[f.ci[k]] = std::max(colmax[f.ci[k]], std::abs(f.val[k]));
    for (std::size_t j = 0; j < ncols; ++j)
        if (colmax[j] > 0.0) f.col_scale[j] = 1.0 / colmax[j];
    // the scaled matrix: the reference rebuilds it from triplets; the
    // pattern is already sorted and duplicate-free, so that amounts to
    // scaling in place and dropping entries that became exactly zero
    {
        std::size_t w = 0, k = 0;
        for (std::size_t i = 0; i < m_rows; ++i) {
            const std::size_t e = f.rp[i + 1];
            for (; k < e; ++k) {
                const double v = f.val[k] * f.col_scale[f.ci[k]];
                if (v == 0.0) continue;
                f.ci[w] = f.ci[k];
                f.val[w] = v;
                ++w;
            }
            f.rp[i + 1] = w;
        }
        f.ci.resize(w);
        f.val.resize(w);
    }
    for (std::size_t j = 0; j < ncols; ++j) f.c[j] *= f.col_scale[j];
    return f;
}

// ---- start points ----

// Mehrotra's default start on the scaled standard form (interior_point.cpp:439-453).
void default_start(const StandardForm& f, std::vector<double>& x, std::vector<double>& z, std::vector<double>& lam) {
    double b_norm = 1.0, c_norm = 1.0;
    for (double v : f.rhs) b_norm = std::max(b_norm, std::abs(v));
    for (double v : f.c) c_norm = std::max(c_norm, std::abs(v));
    x.assign(f.n, b_norm + 1.0);
    z.resize(f.n);
    for (std::size_t j = 0; j < f.n; ++j) z[j] = std::max(c_norm + 1.0, std::abs(f.c[j]));
    lam.assign(f.m, 0.0);
}

// Relative KKT residual of (x, z, lam) on the scaled form:
// max(||Mx-b||inf/(1+||b||inf), ||M^T lam + z - c||inf/(1+||c||inf), |x^T z|/(1+|c^T x|)).
double start_kkt(const StandardForm& f, const std::vector<double>& x, const std::vector<double>& z,
                 const std::vector<double>& lam) {
    double bn = 0.0, cn = 0.0, rp = 0.0, rd = 0.0, xz = 0.0, cx = 0.0;
    std::vector<double> mtl(f.n, 0.0);
    for (std::size_t i = 0; i < f.m; ++i) {
        double s = 0.0;
        for (std::size_t k = f.rp[i]; k < f.rp[i + 1]; ++k) {
            s += f.val[k] * x[f.ci[k]];
            mtl[f.ci[k]] += f.val[k] * lam[i];
        }
        rp = std::max(rp, std::abs(s - f.rhs[i]));
        bn = std::max(bn, std::abs(f.rhs[i]));
    }
    for (std::size_t j = 0; j < f.n; ++j) {
        rd = std::max(rd, std::abs(mtl[j] + z[j] - f.c[j]));
        cn = std::max(cn, std::abs(f.c[j]));
        xz += x[j] * z[j];
        cx += f.c[j] * x[j];
    }
    return std::max({rp / (1.0 + bn), rd / (1.0 + cn), std::abs(xz) / (1.0 + std::abs(cx))});
}

// Maps an original-space (x, y, s) to the scaled standard form and shifts it
// to strict interiority with Mehrotra's heuristic (S. Mehrotra, "On the
// implementation of a primal-dual interior point method", SIAM J. Optim.
// 2(4), 1992, section 7): dx = max(-1.5 min x, 0), dz likewise, then
// x += 0.5 x'z / sum z, z += 0.5 x'z / sum x, the second shifts at least
// `floor` times the default start's x and z entries (a point on the boundary
// would otherwise start with almost no centrality). Returns false when the
// point cannot be made strictly interior.
bool warm_point(const StandardForm& f, const WarmStart& w, double floor, std::vector<double>& x,
                std::vector<double>& z, std::vector<double>& lam) {
    const std::size_t norig = f.row_mult.size();
    if (w.x.size() != f.var_info.size() || (!w.y.empty() && w.y.size() != norig) ||
        (!w.s.empty() && w.s.size() != f.var_info.size()))
        return false;
    x.assign(f.n, 0.0);
    for (std::size_t j = 0; j < f.var_info.size(); ++j) {
        const VarInfo& v = f.var_info[j];
        if (v.is_fixed) continue;
        if (v.slots.size() == 1) {
            const int g = v.slots[0];
            x[g] = (w.x[j] - v.shifts[0]) / (v.signs[0] * f.col_scale[g]);
        } else if (v.slots.size() == 2) {
            x[v.slots[0]] = std::max(w.x[j], 0.0) / f.col_scale[v.slots[0]];
            x[v.slots[1]] = std::max(-w.x[j], 0.0) / f.col_scale[v.slots[1]];
        }
    }
    // slack columns from the rows' residuals (each slack has one entry)
    std::vector<double> r(f.rhs);
    std::vector<std::size_t> slack_row(f.n - f.nslots);
    std::vector<double> slack_coef(f.n - f.nslots, 0.0);
    for (std::size_t i = 0; i < f.m; ++i)
        for (std::size_t k = f.rp[i]; k < f.rp[i + 1]; ++k) {
            if (f.ci[k] < f.nslots) {
                r[i] -= f.val[k] * x[f.ci[k]];
            } else {
                slack_row[f.ci[k] - f.nslots] = i;
                slack_coef[f.ci[k] - f.nslots] = f.val[k];
            }
        }
    for (std::size_t s = 0; s < slack_coef.size(); ++s)
        if (slack_coef[s] != 0.0) x[f.nslots + s] = r[slack_row[s]] / slack_coef[s];
    lam.assign(f.m, 0.0);
    if (!w.y.empty())
        for (std::size_t i = 0; i < norig; ++i) lam[i] = w.y[i] / f.row_mult[i];
    // z = c - M^T lam, then the given reduced costs on the structural slots
    z = f.c;
    for (std::size_t i = 0; i < f.m; ++i)
        if (lam[i] != 0.0)
            for (std::size_t k = f.rp[i]; k < f.rp[i + 1]; ++k) z[f.ci[k]] -= f.val[k] * lam[i];
    if (!w.s.empty())
        for (std::size_t j = 0; j < f.var_info.size(); ++j) {
            const VarInfo& v = f.var_info[j];
            for (std::size_t q = 0; q < v.slots.size(); ++q)
                z[v.slots[q]] = v.signs[q] * f.col_scale[v.slots[q]] * w.s[j];
        }
    for (std::size_t j = 0; j < f.n; ++j)
        if (!std::isfinite(x[j]) || !std::isfinite(z[j])) return false;
    double xmin = 0.0, zmin = 0.0;
    for (std::size_t j = 0; j < f.n; ++j) {
        xmin = std::min(xmin, x[j]);
        zmin = std::min(zmin, z[j]);
    }
    const double dx = std::max(-1.5 * xmin, 0.0), dz = std::max(-1.5 * zmin, 0.0);
    double xz = 0.0, sx = 0.0, sz = 0.0;
    for (std::size_t j = 0; j < f.n; ++j) {
        x[j] += dx;
        z[j] += dz;
        xz += x[j] * z[j];
        sx += x[j];
        sz += z[j];
    }
    if (!(xz > 0.0) || !(sx > 0.0) || !(sz > 0.0)) return false;
    double b_norm = 1.0, c_norm = 1.0;
    for (double v : f.rhs) b_norm = std::max(b_norm, std::abs(v));
    for (double v : f.c) c_norm = std::max(c_norm, std::abs(v));
    const double dx2 = std::max(0.5 * xz / sz, floor * (b_norm + 1.0));
    const double dz2 = std::max(0.5 * xz / sx, floor * (c_norm + 1.0));
    for (std::size_t j = 0; j < f.n; ++j) {
        x[j] += dx2;
        z[j] += dz2;
        if (!(x[j] > 0.0) || !(z[j] > 0.0) || !std::isfinite(x[j]) || !std::isfinite(z[j])) return false;
    }
    return true;
}

// The start the solve uses: the warm one when given, usable and better by
// the KKT residual, else the default. Returns whether the warm one is used.
bool choose_start(const StandardForm& f, const WarmStart* w, double floor, std::vector<double>& x,
                  std::vector<double>& z, std::vector<double>& lam, double* kkt_default, double* kkt_warm) {
    default_start(f, x, z, lam);
    *kkt_default = start_kkt(f, x, z, lam);
    *kkt_warm = 0.0;
    if (!w || w->empty()) return false;
    std::vector<double> wx, wz, wl;
    if (!warm_point(f, *w, floor, wx, wz, wl)) return false;
    *kkt_warm = start_kkt(f, wx, wz, wl);
    if (!(*kkt_warm < *kkt_default)) return false;
    x.swap(wx);
    z.swap(wz);
    lam.swap(wl);
    return true;
}

void original_duals(const StandardForm& f, const model::LpProblem& p, const double* lam, std::vector<double>& y,
                    std::vector<double>& s) {
    y.clear();
    s.clear();
    if (f.row_mult.size() != p.num_rows) return;
    y.resize(p.num_rows);
    for (std::size_t i = 0; i < p.num_rows; ++i) y[i] = f.row_mult[i] * lam[i];
    const bool negate = p.obj_sense == model::ObjectiveSense::MAXIMIZE;
    s.resize(p.num_cols);
    for (std::size_t j = 0; j < p.num_cols; ++j) s[j] = negate ? -p.objective[j] : p.objective[j];
    for (std::size_t i = 0; i < p.num_rows; ++i)
        for (std::size_t k = p.row_ptr[i]; k < p.row_ptr[i + 1]; ++k) s[p.col_indices[k]] -= p.values[k] * y[i];
}

std::vector<double> to_original_primal(const StandardForm& f, const std::vector<double>& y) {
    // :375-396
    const std::size_t n = f.var_info.size();
    std::vector<double> primal(n, 0.0);
    for (std::size_t j = 0; j < n; ++j) {
        const VarInfo& v = f.var_info[j];
        if (v.is_fixed) {
            primal[j] = v.fixed;
            continue;
        }
        double val = 0.0;
        for (std::size_t s = 0; s < v.slots.size(); ++s) {
            const int gi = v.slots[s];
            if (gi < 0 || static_cast<std::size_t>(gi) >= f.col_scale.size()) continue;
            val += v.signs[s] * f.col_scale[gi] * y[gi];
            if (s == 0) val += v.shifts[s];
        }
        primal[j] = val;
    }
    return primal;
}

// Unscale factors for the relative KKT residual (hn_ipm_kkt): row i of the
// standard form is the original row times row_mult[i] (+-gamma_i) -- the
// upper-bound rows are unscaled -- and column j carries col_scale[j]; offset
// is the minimisation form's objective constant (shifts plus obj_offset).
void unscale_factors(const StandardForm& f, const model::LpProblem& p, double* ru, double* cu, double* offset) {
    for (std::size_t i = 0; i < f.m; ++i)
        ru[i] = i < f.row_mult.size() && f.row_mult[i] != 0.0 ? 1.0 / std::abs(f.row_mult[i]) : 1.0;
    for (std::size_t j = 0; j < f.n; ++j) cu[j] = 1.0 / f.col_scale[j];
    const bool negate = p.obj_sense == model::ObjectiveSense::MAXIMIZE;
    *offset = f.offset + (negate ? -p.obj_offset : p.obj_offset);
}

// Device buffer owning helper.
struct DevBuf {
    void* p = nullptr;
    explicit DevBuf(std::size_t bytes) { ck(hn_malloc(&p, bytes ? bytes : 8), "hn_malloc"); }
    ~DevBuf() {
        if (p) hn_free(p);
    }
    double* d() const { return static_cast<double*>(p); }
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
};

using Clock = std::chrono::steady_clock;
double ms_since(Clock::time_point t) { return std::chrono::duration<double, std::milli>(Clock::now() - t).count(); }

// The normal matrix on the host: the device pattern (CSR, both triangles)
// plus its values, kept for the refinement products, and a dense lower
// triangle for the factorisation.
struct HostNormal {
    std::size_t m = 0;
    std::vector<uint64_t> rp, ci;
    std::vector<double> val;
    std::vector<double> dense;
    void to_dense() {
        dense.assign(m * m, 0.0);
        for (std::size_t i = 0; i < m; ++i)
            for (uint64_t k = rp[i]; k < rp[i + 1]; ++k)
                if (ci[k] <= i) dense[i * m + ci[k]] = val[k];
    }
    // y = N x with SparseMatrix::multiply's order (sparse_matrix.cpp:142-149)
    void multiply(const std::vector<double>& x, std::vector<double>& y) const {
        y.assign(m, 0.0);
        for (std::size_t i = 0; i < m; ++i) {
            double s = 0.0;
            for (uint64_t k = rp[i]; k < rp[i + 1]; ++k) s += val[k] * x[ci[k]];
            y[i] = s;
        }
    }
};

// iterative_refinement(fac, N, x, rhs) with its defaults 1e-10 / 5 sweeps
// (core/numerical/refinement.cpp:7-37).
template <class Fac>
void refine(const Fac& fac, const HostNormal& N, std::vector<double>& x, const std::vector<double>& rhs) {
    const std::size_t n = x.size();
    double norm_rhs = 0.0;
    for (double v : rhs) norm_rhs = std::max(norm_rhs, std::abs(v));
    if (norm_rhs == 0.0 || norm_rhs != norm_rhs) return;
    std::vector<double> ax, r(n);
    for (int it = 0; it < 5; ++it) {
        N.multiply(x, ax);
        double rel = 0.0;
        for (std::size_t i = 0; i < n; ++i) rel = std::max(rel, std::abs(rhs[i] - ax[i]));
        rel /= norm_rhs;
        if (rel <= 1e-10) break;
        for (std::size_t i = 0; i < n; ++i) r[i] = rhs[i] - ax[i];
        fac.solve(r);
        for (std::size_t i = 0; i < n; ++i) x[i] += r[i];
    }
}

constexpr std::size_t kMaxDenseRows = 12000;

}  // namespace

void build_forms(const std::vector<model::LpProblem>& problems, double feas_tol, PackedForm& out,
                 const std::vector<WarmStart>* warm, double warm_floor) {
    const std::size_t K = problems.size();
    std::vector<std::shared_ptr<StandardForm>> forms(K);
    std::string err;
#pragma omp parallel for schedule(dynamic, 8)
    for (std::size_t i = 0; i < K; ++i) {
        try {
            auto f = std::make_shared<StandardForm>(build_standard_form(remove_duplicate_rows(problems[i]), feas_tol));
            forms[i] = f;
        } catch (const std::exception& e) {
#pragma omp critical
            err = e.what();
        }
    }
    if (!err.empty()) throw std::runtime_error(err);
    out = PackedForm{};
    std::size_t nnz = 0;
    for (std::size_t i = 0; i < K; ++i) {
        const StandardForm& f = *forms[i];
        if (f.m == 0 || f.n == 0)
            throw std::invalid_argument("batch instance " + std::to_string(i) + " has an empty standard form");
        out.row_off.push_back(out.row_off.back() + (int64_t)f.m);
        out.col_off.push_back(out.col_off.back() + (int64_t)f.n);
        nnz += f.val.size();
    }
    out.rp.reserve(out.row_off.back() + 1);
    out.ci.reserve(nnz);
    out.val.reserve(nnz);
    for (std::size_t i = 0; i < K; ++i) {
        const StandardForm& f = *forms[i];
        const uint64_t cb = (uint64_t)out.col_off[i];
        for (std::size_t r = 0; r < f.m; ++r) {
            for (std::size_t k = f.rp[r]; k < f.rp[r + 1]; ++k) {
                out.ci.push_back(cb + f.ci[k]);
                out.val.push_back(f.val[k]);
            }
            out.rp.push_back(out.ci.size());
        }
        out.rhs.insert(out.rhs.end(), f.rhs.begin(), f.rhs.end());
        out.c.insert(out.c.end(), f.c.begin(), f.c.end());
    }
    // start points per instance (default :439-453, or the warm start)
    out.x0.resize(out.col_off.back());
    out.z0.resize(out.col_off.back());
    out.lam0.resize(out.row_off.back());
    out.warm_used.assign(K, 0);
    out.kkt_default.assign(K, 0.0);
    out.kkt_warm.assign(K, 0.0);
#pragma omp parallel for schedule(dynamic, 8)
    for (std::size_t i = 0; i < K; ++i) {
        const StandardForm& f = *forms[i];
        std::vector<double> x, z, lam;
        const WarmStart* w = (warm && i < warm->size()) ? &(*warm)[i] : nullptr;
        out.warm_used[i] = choose_start(f, w, warm_floor, x, z, lam, &out.kkt_default[i], &out.kkt_warm[i]);
        std::copy(x.begin(), x.end(), out.x0.begin() + out.col_off[i]);
        std::copy(z.begin(), z.end(), out.z0.begin() + out.col_off[i]);
        std::copy(lam.begin(), lam.end(), out.lam0.begin() + out.row_off[i]);
    }
    out.ru.resize(out.row_off.back());
    out.cu.resize(out.col_off.back());
    out.offset.resize(K);
#pragma omp parallel for schedule(dynamic, 8)
    for (std::size_t i = 0; i < K; ++i)
        unscale_factors(*forms[i], problems[i], out.ru.data() + out.row_off[i], out.cu.data() + out.col_off[i],
                        &out.offset[i]);
    out.forms = std::move(forms);
}

std::vector<double> to_original_primal_packed(const PackedForm& pf, std::size_t i, const std::vector<double>& y) {
    return to_original_primal(*pf.forms[i], y);
}

void original_duals_packed(const PackedForm& pf, std::size_t i, const model::LpProblem& p, const double* lam,
                           std::vector<double>& y, std::vector<double>& s) {
    original_duals(*pf.forms[i], p, lam, y, s);
}

InteriorPointResult InteriorPointSolver::solve(const model::LpProblem& problem) {
    const auto start = Clock::now();
    InteriorPointResult result;
    const auto& O = options_;
    if (problem.num_cols == 0) {
        result.status = ProblemStatus::OPTIMAL;
        result.objective_value = problem.obj_offset;
        return result;
    }
    try {
        const model::LpProblem cleaned = remove_duplicate_rows(problem);
        const StandardForm f = build_standard_form(cleaned, O.feasibility_tol);
        if (f.n == 0) {
            result.status = ProblemStatus::OPTIMAL;
            result.objective_value = f.offset;
            result.primal = to_original_primal(f, {});
            return result;
        }
        if (f.m == 0) {
            bool unbounded = false;
            for (double cj : f.c)
                if (cj < -1e-9) unbounded = true;  // optimality_tol of industrial_defaults
            result.status = unbounded ? ProblemStatus::UNBOUNDED : ProblemStatus::OPTIMAL;
            result.primal = to_original_primal(f, std::vector<double>(f.n, 0.0));
            double obj = problem.obj_offset;
            for (std::size_t j = 0; j < problem.num_cols; ++j) obj += problem.objective[j] * result.primal[j];
            result.objective_value = obj;
            return result;
        }
        const bool sparse_fac = O.factorization == 2 || (O.factorization == 0 && f.m > kMaxDenseRows);
        if (!sparse_fac && f.m > kMaxDenseRows)
            throw std::runtime_error("standard form has " + std::to_string(f.m) +
                                     " rows; the host dense factorisation supports up to 12000");
        const std::size_t m = f.m, n = f.n;
        ck(hn_init(O.device), "hn_init");
        hn_csr* M = nullptr;
        ck(hn_csr_create((int64_t)m, (int64_t)n, reinterpret_cast<const uint64_t*>(f.rp.data()),
                         reinterpret_cast<const uint64_t*>(f.ci.data()), f.val.data(), 0, &M),
           "hn_csr_create");
        std::unique_ptr<hn_csr, int (*)(hn_csr*)> Mh(M, hn_csr_destroy);
        hn_pattern* P = nullptr;
        ck(hn_ada_symbolic(M, &P), "hn_ada_symbolic");
        std::unique_ptr<hn_pattern, int (*)(hn_pattern*)> Ph(P, hn_pattern_destroy);
        HostNormal N;
        N.m = m;
        int64_t pm = 0, pnnz = 0;
        ck(hn_pattern_info(P, &pm, &pnnz), "hn_pattern_info");
        N.rp.resize(m + 1);
        N.ci.resize((std::size_t)pnnz);
        N.val.resize((std::size_t)pnnz);
        ck(hn_pattern_export(P, N.rp.data(), N.ci.data()), "hn_pattern_export");
        result.nnz_normal = (std::size_t)pnnz;

        // start point (:439-453, or the warm start)
        std::vector<double> hx, hz, hlam;
        result.warm_start_used =
            choose_start(f, &O.initial_point, O.warm_start_floor, hx, hz, hlam, &result.kkt_default,
                         &result.kkt_warm);

        DevBuf x(8 * n), z(8 * n), lam(8 * m), b(8 * m), c(8 * n), mx(8 * m), rp(8 * m), rd(8 * n), D(8 * n),
            Drd(8 * n), rhs_pred(8 * m), rhs(8 * m), dlam(8 * m), dx(8 * n), dz(8 * n), zs(8 * n),
            nval(8 * (std::size_t)pnnz), scal(8 * HN_IPM_NSCAL), dyn(8);
        void* st = nullptr;  // legacy default stream
        ck(hn_memcpy_h2d(x.p, hx.data(), 8 * n, st), "H2D");
        ck(hn_memcpy_h2d(z.p, hz.data(), 8 * n, st), "H2D");
        ck(hn_memcpy_h2d(lam.p, hlam.data(), 8 * m, st), "H2D");
        ck(hn_memcpy_h2d(b.p, f.rhs.data(), 8 * m, st), "H2D");
        ck(hn_memcpy_h2d(c.p, f.c.data(), 8 * n, st), "H2D");
        ck(hn_memset(scal.p, 0, 8 * HN_IPM_NSCAL, st), "memset");
        double sc[HN_IPM_NSCAL];
        auto read_scal = [&]() { ck(hn_memcpy_d2h(sc, scal.p, sizeof(sc), st), "D2H scal"); };
        // relative KKT residual of the unscaled LP, and the iterate the
        // reference's rule accepted (kept while the solve tightens past it)
        const bool tighten = O.kkt_tol > 0.0;
        std::vector<double> hru(m), hcu(n);
        double koff = 0.0;
        unscale_factors(f, cleaned, hru.data(), hcu.data(), &koff);
        DevBuf ru(8 * m), cu(8 * n), kkt(8 * 4), xb(tighten ? 8 * n : 8), zb(tighten ? 8 * n : 8),
            lb(tighten ? 8 * m : 8);
        ck(hn_memcpy_h2d(ru.p, hru.data(), 8 * m, st), "H2D");
        ck(hn_memcpy_h2d(cu.p, hcu.data(), 8 * n, st), "H2D");
        double kv[4] = {0, 0, 0, 0}, kref[4] = {0, 0, 0, 0};
        long ref_iter = -1;
        auto measure = [&]() {
            ck(hn_ipm_kkt((int64_t)n, (int64_t)m, x.d(), lam.d(), b.d(), c.d(), rp.d(), rd.d(), ru.d(), cu.d(), koff,
                          kkt.d(), st),
               "hn_ipm_kkt");
            ck(hn_memcpy_d2h(kv, kkt.p, sizeof(kv), st), "D2H kkt");
        };
        auto flags = [&]() {
            std::uint64_t fl;
            std::memcpy(&fl, &sc[HN_IPM_FLAGS], 8);
            return fl;
        };

        bool done = false, time_up = false, interrupted = false, numerical_error = false;
        auto deadline_passed = [&]() {
            return O.time_limit_seconds > 0.0 && ms_since(start) >= O.time_limit_seconds * 1e3;
        };
        DenseLDLT fac;
        SparseLDLT sfac;  // the pattern of N is fixed: analysed once, refactorised per iteration
        if (sparse_fac) {
            auto ta = Clock::now();
            sfac.analyze(m, N.rp.data(), N.ci.data());
            result.factor_ms += ms_since(ta);
        }
        std::vector<double> hrhs(m), hdlam(m);
        auto solve_normal = [&](const DevBuf& rhs_dev) {
            auto t = Clock::now();
            ck(hn_memcpy_d2h(hrhs.data(), rhs_dev.p, 8 * m, st), "D2H rhs");
            hdlam = hrhs;
            if (sparse_fac) {
                sfac.solve(hdlam);
                refine(sfac, N, hdlam, hrhs);
            } else {
                fac.solve(hdlam);
                refine(fac, N, hdlam, hrhs);
            }
            ck(hn_memcpy_h2d(dlam.p, hdlam.data(), 8 * m, st), "H2D dlam");
            result.solve_ms += ms_since(t);
        };

        const std::size_t max_it = static_cast<std::size_t>(std::max(O.max_iterations, 0));
        std::size_t iter = 0;
        for (iter = 0; iter < max_it; ++iter) {
            if (O.interrupt_callback && O.interrupt_callback()) {
                interrupted = true;
                break;
            }
            if (deadline_passed()) {
                time_up = true;
                break;
            }
            auto t0 = Clock::now();
            ck(hn_ipm_residuals(M, x.d(), lam.d(), z.d(), b.d(), c.d(), mx.d(), rp.d(), rd.d(), D.d(), Drd.d(),
                                scal.d(), st),
               "hn_ipm_residuals");
            read_scal();
            measure();
            const double mu = sc[HN_IPM_MU];
            if (ref_iter < 0 && sc[HN_IPM_NRP] < O.convergence_tol && sc[HN_IPM_NRD] < O.convergence_tol &&
                mu < O.complementarity_tol) {  // the reference's rule (:525-530)
                ref_iter = (long)iter;
                std::memcpy(kref, kv, sizeof(kv));
                if (tighten) {
                    ck(hn_memcpy_d2d(xb.p, x.p, 8 * n, st), "save x");
                    ck(hn_memcpy_d2d(zb.p, z.p, 8 * n, st), "save z");
                    ck(hn_memcpy_d2d(lb.p, lam.p, 8 * m, st), "save lam");
                }
            }
            if (ref_iter >= 0 &&
                (!tighten || kv[0] <= O.kkt_tol || (long)iter - ref_iter >= O.kkt_extra_iterations)) {
                done = true;
                result.device_ms += ms_since(t0);
                break;
            }
            ck(hn_ada_numeric(P, D.d(), O.regularization, nval.d(), dyn.d(), st), "hn_ada_numeric");
            ck(hn_memcpy_d2h(N.val.data(), nval.p, 8 * (std::size_t)pnnz, st), "D2H N");
            result.device_ms += ms_since(t0);
            if (deadline_passed()) {
                time_up = true;
                break;
            }
            auto tf = Clock::now();
            if (sparse_fac) {
                sfac.factorize(N.val.data(), O.singular_tol);
            } else {
                N.to_dense();
                fac.factorize(N.dense, m, O.singular_tol);
            }
            result.factor_ms += ms_since(tf);
            if (deadline_passed()) {
                time_up = true;
                break;
            }
            t0 = Clock::now();
            ck(hn_ipm_rhs(M, Drd.d(), rp.d(), mx.d(), rhs_pred.d(), st), "hn_ipm_rhs");
            result.device_ms += ms_since(t0);
            solve_normal(rhs_pred);
            t0 = Clock::now();
            ck(hn_ipm_direction(M, dlam.d(), D.d(), rd.d(), x.d(), nullptr, dx.d(), dz.d(), st), "hn_ipm_direction");
            ck(hn_ipm_step_lengths((int64_t)n, (int64_t)m, x.d(), dx.d(), z.d(), dz.d(), dlam.d(), scal.d(), st),
               "hn_ipm_step_lengths");
            read_scal();
            if (flags() & 1ull) {
                numerical_error = true;
                break;
            }
            ck(hn_ipm_corrector(M, x.d(), dx.d(), z.d(), dz.d(), rhs_pred.d(), zs.d(), rhs.d(), scal.d(), st),
               "hn_ipm_corrector");
            result.device_ms += ms_since(t0);
            solve_normal(rhs);
            t0 = Clock::now();
            ck(hn_ipm_direction(M, dlam.d(), D.d(), rd.d(), x.d(), zs.d(), dx.d(), dz.d(), st), "hn_ipm_direction");
            ck(hn_ipm_step_lengths((int64_t)n, (int64_t)m, x.d(), dx.d(), z.d(), dz.d(), dlam.d(), scal.d(), st),
               "hn_ipm_step_lengths");
            read_scal();
            if (flags() & 1ull) {
                numerical_error = true;
                break;
            }
            ck(hn_ipm_update((int64_t)n, (int64_t)m, x.d(), dx.d(), z.d(), dz.d(), lam.d(), dlam.d(), scal.d(), st),
               "hn_ipm_update");
            read_scal();
            result.device_ms += ms_since(t0);
            if (flags() & 2ull) {
                numerical_error = true;
                break;
            }
            if (O.verbose) {
                double dreg = 0.0;
                ck(hn_memcpy_d2h(&dreg, dyn.p, 8, st), "D2H dyn_reg");
                std::fprintf(stderr, "IPM it=%zu mu=%g rp=%g rd=%g ap=%g ad=%g dyn_reg=%g kkt=%g (%g %g %g)\n", iter,
                             mu, sc[HN_IPM_NRP], sc[HN_IPM_NRD], sc[HN_IPM_AP], sc[HN_IPM_AD], dreg, kv[0], kv[1],
                             kv[2], kv[3]);
            }
            result.iterations = iter + 1;
        }
        double last_nrp = 0.0;
        {
            ck(hn_ipm_residuals(M, x.d(), lam.d(), z.d(), b.d(), c.d(), mx.d(), rp.d(), rd.d(), D.d(), Drd.d(),
                                scal.d(), st),
               "hn_ipm_residuals");
            read_scal();
            measure();
            last_nrp = sc[HN_IPM_NRP];
            if (ref_iter >= 0) {
                // the reference stopped here as OPTIMAL; whatever the
                // tightening met afterwards, return the better iterate
                if (tighten && (numerical_error || !(kv[0] <= kref[0]))) {
                    ck(hn_memcpy_d2d(x.p, xb.p, 8 * n, st), "restore x");
                    ck(hn_memcpy_d2d(z.p, zb.p, 8 * n, st), "restore z");
                    ck(hn_memcpy_d2d(lam.p, lb.p, 8 * m, st), "restore lam");
                    std::memcpy(kv, kref, sizeof(kv));
                    result.iterations = (std::size_t)ref_iter;
                }
                done = true;
                numerical_error = interrupted = time_up = false;
            }
            // relaxed acceptance after the loop (:727-753); crossover is not
            // part of this solver, so the strict 1e-4 primal threshold applies
            if (!done && !interrupted && sc[HN_IPM_NRP] < 1e-4 && sc[HN_IPM_NRD] < 1e-4 && sc[HN_IPM_MU] < 1e-4)
                done = true;
            result.kkt = kv[0];
            result.kkt_primal = kv[1];
            result.kkt_dual = kv[2];
            result.kkt_gap = kv[3];
            result.reference_iterations = ref_iter;
        }
        ck(hn_memcpy_d2h(hx.data(), x.p, 8 * n, st), "D2H x");
        std::vector<double> primal = to_original_primal(f, hx);
        double obj = 0.0;
        bool obj_ok = std::isfinite(problem.obj_offset);
        for (std::size_t j = 0; j < problem.num_cols && obj_ok; ++j) {
            const double term = problem.objective[j] * primal[j];
            if (!std::isfinite(term)) obj_ok = false;
            obj += term;
        }
        if (obj_ok) obj += problem.obj_offset;
        if (!obj_ok) numerical_error = true;
        result.objective_value = obj_ok ? obj : 0.0;
        result.primal = primal;
        result.dual.assign(problem.num_rows, 0.0);
        {
            std::vector<double> hl(m);
            ck(hn_memcpy_d2h(hl.data(), lam.p, 8 * m, st), "D2H lam");
            original_duals(f, problem, hl.data(), result.dual_estimate, result.reduced_cost_estimate);
        }
        const bool feasible_incumbent = last_nrp <= O.feasibility_tol;
        result.status = numerical_error ? ProblemStatus::NUMERICAL_ERROR
                        : interrupted   ? ProblemStatus::INTERRUPTED
                        : done          ? ProblemStatus::OPTIMAL
                        : feasible_incumbent ? ProblemStatus::SUBOPTIMAL
                        : time_up            ? ProblemStatus::TIME_LIMIT
                                             : ProblemStatus::ITER_LIMIT;
    } catch (const std::exception& e) {
        result.status = ProblemStatus::NUMERICAL_ERROR;
        result.error = e.what();
    }
    result.solve_time_ms = ms_since(start);
    return result;
}

}  // namespace hn::lp
