// extern "C" shim over the reference's problem readers (model::MPSParser,
// core/model/mps_parser.cpp; model::LPParser, core/model/lp_parser.cpp),
// compiled from the reference's own sources into oracle/_ref/libhnref.so by
// oracle/Makefile.
//
// TEST INFRASTRUCTURE ONLY: the checker for tests/ and bench.py's CPU leg.
// Nothing in the product links or calls it.
//
//   hnref_mps_parse   -> MPSParser::parse_string (default settings, or the
//                        layout forced through set_free_format)
//   hnref_mps_shape / hnref_mps_arrays -> the parsed Problem: constraint
//                        matrix (CSR from SparseMatrix::from_triplets), rows,
//                        columns, objective sense
//   hnref_mps_parse_ms -> wall time of one parse_string (CPU baseline)
//   hnref_lp_parse    -> LPParser::parse_string; read with the same accessors
#include "lp_parser.hpp"
#include "mps_parser.hpp"

#include <chrono>
#include <cstdint>
#include <cstring>
#include <string>

using hypernova::model::LPParser;
using hypernova::model::MPSParser;

namespace {
struct RefMps {  // the parts of MPSParseResult / LPParseResult read here
    struct {
        hypernova::model::Problem problem;
        bool success = false;
        std::vector<std::string> warnings, errors;
    } r;
};

template <class R>
void keep(RefMps* h, R&& res) {
    h->r.problem = std::move(res.problem);
    h->r.success = res.success;
    h->r.warnings = res.warnings;
    h->r.errors = res.errors;
}
}  // namespace

extern "C" {

void* hnref_mps_parse(const char* text, int64_t len, int format) {
    MPSParser p;
    if (format >= 0) p.set_free_format(format == 0);
    auto* h = new RefMps;
    keep(h, p.parse_string(std::string(text, static_cast<std::size_t>(len))));
    return h;
}

// LPParser::parse_string; an exception escaping it (the reference finalises
// pending statements outside its per-line try block) counts as a failed read
void* hnref_lp_parse(const char* text, int64_t len) {
    LPParser p;
    auto* h = new RefMps;
    try {
        keep(h, p.parse_string(std::string(text, static_cast<std::size_t>(len))));
    } catch (const std::exception& e) {
        h->r.success = false;
        h->r.errors.push_back(e.what());
    }
    return h;
}

int64_t hnref_parse_errors(const void* hv) {
    return static_cast<int64_t>(static_cast<const RefMps*>(hv)->r.errors.size());
}

int hnref_mps_shape(const void* hv, int64_t* m, int64_t* n, int64_t* nnz, int* maximize, int* success,
                    int64_t* warnings) {
    const auto* h = static_cast<const RefMps*>(hv);
    const auto& P = h->r.problem;
    *m = static_cast<int64_t>(P.constraints.size());
    *n = static_cast<int64_t>(P.variables.size());
    *nnz = static_cast<int64_t>(P.constraint_matrix.values().size());
    *maximize = P.obj_sense == hypernova::model::ObjectiveSense::MAXIMIZE ? 1 : 0;
    *success = h->r.success ? 1 : 0;
    *warnings = static_cast<int64_t>(h->r.warnings.size());
    return 0;
}

int hnref_mps_arrays(const void* hv, uint64_t* rp, uint64_t* ci, double* val, double* c, double* rhs,
                     int32_t* sense, double* lb, double* ub, double* range_lo, double* range_hi, int32_t* vtype) {
    const auto* h = static_cast<const RefMps*>(hv);
    const auto& P = h->r.problem;
    const auto& A = P.constraint_matrix;
    const std::size_t m = P.constraints.size(), n = P.variables.size();
    const auto& arp = A.row_ptr();
    for (std::size_t i = 0; i <= m; ++i) rp[i] = i < arp.size() ? arp[i] : (arp.empty() ? 0 : arp.back());
    for (std::size_t k = 0; k < A.values().size(); ++k) {
        ci[k] = A.col_indices()[k];
        val[k] = A.values()[k];
    }
    for (std::size_t j = 0; j < n; ++j) {
        const auto& v = P.variables[j];
        c[j] = v.objective_coeff;
        lb[j] = v.lower_bound;
        ub[j] = v.upper_bound;
        vtype[j] = static_cast<int32_t>(v.type);
    }
    for (std::size_t i = 0; i < m; ++i) {
        const auto& k = P.constraints[i];
        rhs[i] = k.rhs;
        sense[i] = static_cast<int32_t>(k.sense);
        range_lo[i] = k.lower_bound;
        range_hi[i] = k.upper_bound;
    }
    return 0;
}

const char* hnref_mps_name(const void* hv, int what, int64_t i) {
    const auto& P = static_cast<const RefMps*>(hv)->r.problem;
    if (what < 0) return P.name.c_str();
    if (what == 0) return P.constraints[static_cast<std::size_t>(i)].name.c_str();
    return P.variables[static_cast<std::size_t>(i)].name.c_str();
}

void hnref_mps_free(void* hv) { delete static_cast<RefMps*>(hv); }

double hnref_mps_parse_ms(const char* text, int64_t len) {
    const std::string s(text, static_cast<std::size_t>(len));
    MPSParser p;
    const auto t0 = std::chrono::steady_clock::now();
    auto r = p.parse_string(s);
    const auto t1 = std::chrono::steady_clock::now();
    return r.success ? std::chrono::duration<double, std::milli>(t1 - t0).count() : -1.0;
}

}  // extern "C"
