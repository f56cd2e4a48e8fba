// MPS reader: HyperNova's MPSParser (core/model/mps_parser.cpp) restated with
// the same results on the same text -- sections, free/fixed layouts and their
// detection, the lenient fall-backs -- but without its quadratic name
// lookups: rows and columns are found through hash maps (first occurrence
// wins, as the reference's first-match linear searches do), so a file with
// millions of coefficients reads in linear time. The output is the
// problem's arrays plus the constraint coefficients as triplets in file
// order; hn_csr_create_coo turns those into the device CSR with
// SparseMatrix::from_triplets semantics (sparse_matrix.cpp:8-53).
//
// Number reading follows the two routes of the reference: stream extraction
// (`iss >> double`: libstdc++'s float grammar, then strtod over the collected
// characters, failing unless all of them are used, and failing on overflow)
// and std::stod (strtod over a prefix; out_of_range/invalid_argument caught
// where the reference catches them).
#include <cerrno>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <limits>
#include <optional>
#include <sstream>
#include <string>
#include <string_view>
#include <tuple>
#include <unordered_map>
#include <vector>

#include "hn_host.h"
#include "hn_mps.hpp"
#include "hn_sm100.h"

namespace hn::model {
namespace {

constexpr double kInf = std::numeric_limits<double>::infinity();

enum class Section { NONE, NAME, ROWS, COLUMNS, RHS, RANGES, BOUNDS, SOS, QUADOBJ, QCMATRIX, OBJSENSE, ENDATA };
enum VarType : int32_t { CONTINUOUS = 0, INTEGER = 1, BINARY = 2, SEMI_CONTINUOUS = 3, SEMI_INTEGER = 4 };

inline bool is_ws(char ch) {  // isspace in the C locale
    return ch == ' ' || ch == '\t' || ch == '\n' || ch == '\v' || ch == '\f' || ch == '\r';
}

std::string upper(std::string_view s) {
    std::string u(s);
    for (char& ch : u)
        if (ch >= 'a' && ch <= 'z') ch = static_cast<char>(ch - 'a' + 'A');
    return u;
}

// A cursor over one line with the extraction rules of std::istringstream:
// strings are whitespace-delimited tokens; a double reads the longest prefix
// of libstdc++'s float grammar (sign, digits with one point, exponent after a
// digit) and converts it with strtod, failing unless strtod used all of it or
// when the value overflows. Any failure sticks (later extractions fail).
class Tokens {
public:
    explicit Tokens(std::string_view s) : s_(s) {}
    bool str(std::string& out) {
        if (fail_) return false;
        skip();
        if (p_ >= s_.size()) {
            fail_ = true;  // the sentry fails: `out` is left as it was
            return false;
        }
        const size_t b = p_;
        while (p_ < s_.size() && !is_ws(s_[p_])) ++p_;
        out.assign(s_.substr(b, p_ - b));
        return true;
    }
    bool num(double& out) {
        if (fail_) return false;
        skip();
        std::string acc;
        size_t q = p_;
        bool mant = false, point = false, sci = false;
        if (q < s_.size() && (s_[q] == '+' || s_[q] == '-')) acc += s_[q++];
        while (q < s_.size()) {
            const char ch = s_[q];
            if (ch >= '0' && ch <= '9') {
                acc += ch;
                mant = true;
            } else if (ch == '.' && !point && !sci) {
                acc += ch;
                point = true;
            } else if ((ch == 'e' || ch == 'E') && mant && !sci) {
                acc += ch;
                sci = true;
                ++q;
                if (q < s_.size() && (s_[q] == '+' || s_[q] == '-')) acc += s_[q++];
                while (q < s_.size() && s_[q] >= '0' && s_[q] <= '9') acc += s_[q++];
                break;
            } else {
                break;
            }
            ++q;
        }
        p_ = q;
        out = 0.0;
        if (acc.empty()) {
            fail_ = true;
            return false;
        }
        char* end = nullptr;
        const double v = std::strtod(acc.c_str(), &end);
        if (end != acc.c_str() + acc.size()) {
            fail_ = true;
            return false;
        }
        if (std::isinf(v)) {
            out = v > 0 ? std::numeric_limits<double>::max() : -std::numeric_limits<double>::max();
            fail_ = true;
            return false;
        }
        out = v;
        return true;
    }

private:
    void skip() {
        while (p_ < s_.size() && is_ws(s_[p_])) ++p_;
    }
    std::string_view s_;
    size_t p_ = 0;
    bool fail_ = false;
};

std::vector<std::string> split(std::string_view s) {
    std::vector<std::string> out;
    Tokens t(s);
    std::string w;
    while (t.str(w)) out.push_back(w);
    return out;
}

// std::stod: strtod over a prefix; throws (here: nullopt) on no conversion or
// ERANGE; `used` gets the characters consumed
std::optional<double> stod_like(const std::string& s, size_t* used) {
    const char* b = s.c_str();
    char* end = nullptr;
    errno = 0;
    const double v = std::strtod(b, &end);
    if (end == b || errno == ERANGE) return std::nullopt;
    if (used) *used = static_cast<size_t>(end - b);
    return v;
}

bool is_numeric(const std::string& s) {
    if (s.empty()) return false;
    size_t used = 0;
    const auto v = stod_like(s, &used);
    return v && used == s.size();
}

std::string trim_ends(std::string_view s, const char* set) {
    const size_t b = s.find_first_not_of(set);
    if (b == std::string_view::npos) return "";
    const size_t e = s.find_last_not_of(set);
    return std::string(s.substr(b, e - b + 1));
}

using Record = std::tuple<std::string, std::string, double, std::string, double>;

Section detect_section(std::string_view line) {
    Tokens t(line);
    std::string first, second;
    t.str(first);
    const bool single = !t.str(second);
    const std::string u = upper(first);
    if (u == "NAME") return Section::NAME;
    if (u == "OBJSENSE") return Section::OBJSENSE;
    if (!single) return Section::NONE;
    if (u == "ROWS") return Section::ROWS;
    if (u == "COLUMNS") return Section::COLUMNS;
    if (u == "RHS") return Section::RHS;
    if (u == "RANGES") return Section::RANGES;
    if (u == "BOUNDS") return Section::BOUNDS;
    if (u == "SOS") return Section::SOS;
    if (u == "QUADOBJ") return Section::QUADOBJ;
    if (u == "QCMATRIX") return Section::QCMATRIX;
    if (u == "ENDATA") return Section::ENDATA;
    return Section::NONE;
}

// the reference's layout probe (mps_parser.cpp:124-158): over the first 8
// COLUMNS data lines, the position of the second non-blank character; fixed
// layout when at least 3 were sampled and half of them sit at index 14
bool detect_free(const std::vector<std::string_view>& lines) {
    bool in_columns = false;
    int samples = 0, aligned = 0;
    for (std::string_view line : lines) {
        const size_t lead = line.find_first_not_of(" \t\r\n");
        if (lead == std::string_view::npos) continue;
        std::string_view trimmed = line.substr(lead);
        if (trimmed[0] == '*') continue;
        const Section sec = detect_section(trimmed);
        if (sec != Section::NONE) {
            in_columns = (sec == Section::COLUMNS);
            continue;
        }
        if (!in_columns) continue;
        const size_t a = line.find_first_not_of(" \t");
        if (a == std::string_view::npos) continue;
        const size_t b = line.find_first_not_of(" \t", a + 1);
        if (b == std::string_view::npos) continue;
        ++samples;
        if (b == 14) ++aligned;
        if (samples >= 8) break;
    }
    return !(samples >= 3 && aligned * 2 >= samples);
}

class Reader {
public:
    explicit Reader(MpsProblem& out) : P(out) {}

    void run(std::string_view text, int format) {
        std::vector<std::string_view> lines;
        size_t b = 0;
        while (b < text.size()) {  // std::getline on '\n'
            size_t e = text.find('\n', b);
            if (e == std::string_view::npos) e = text.size();
            lines.push_back(text.substr(b, e - b));
            b = e + 1;
        }
        free_ = format < 0 ? detect_free(lines) : format == 0;
        Section cur = Section::NONE;
        for (std::string_view line : lines) {
            const std::string trimmed = trim_ends(line, " \t\r\n");
            if (trimmed.empty() || trimmed[0] == '*') continue;
            const Section sec = detect_section(trimmed);
            if (sec != Section::NONE) {
                cur = sec;
                if (sec == Section::NAME) {
                    name_line(trimmed);
                } else if (sec == Section::OBJSENSE) {
                    Tokens t(trimmed);
                    std::string s;
                    t.str(s);
                    t.str(s);
                    objsense(s);
                }
                continue;
            }
            switch (cur) {
                case Section::NAME: name_line(line); break;
                case Section::ROWS: rows(line); break;
                case Section::COLUMNS: columns(line); break;
                case Section::RHS: rhs(line); break;
                case Section::RANGES: ranges(line); break;
                case Section::BOUNDS: bounds(line); break;
                case Section::SOS: ++P.sos_records; break;
                case Section::QUADOBJ:
                case Section::QCMATRIX: ++P.quadratic_records; break;
                case Section::OBJSENSE: {
                    Tokens t(trimmed);
                    std::string s;
                    t.str(s);
                    objsense(s);
                    break;
                }
                default: break;
            }
        }
        // INTEGER columns confined to [0, 1] are BINARY (mps_parser.cpp:100-104)
        for (size_t j = 0; j < P.vtype.size(); ++j)
            if (P.vtype[j] == INTEGER && P.lb[j] >= 0.0 && P.ub[j] <= 1.0) P.vtype[j] = BINARY;
    }

private:
    MpsProblem& P;
    bool free_ = true;
    bool in_int_ = false;
    std::string obj_row_;
    std::unordered_map<std::string, int64_t> row_of_, col_of_;

    void warn(std::string msg) { P.warnings.push_back(std::move(msg)); }

    void objsense(const std::string& s) {
        const std::string u = upper(s);
        if (u == "MAX" || u == "MAXIMIZE") P.maximize = 1;
    }

    void name_line(std::string_view line) {
        Tokens t(line);
        std::string s;
        t.str(s);
        if (t.str(s)) P.name = s;
    }

    std::optional<Record> record(std::string_view line) { return free_ ? free_record(line) : fixed_record(line); }

    static std::optional<Record> free_record(std::string_view line) {
        Tokens t(line);
        std::string a, b, c;
        double v1 = 0.0, v2 = 0.0;
        if (!t.str(a) || !t.str(b) || !t.num(v1)) return std::nullopt;
        if (!t.str(c)) c.clear();
        if (!t.num(v2)) v2 = 0.0;
        return Record{a, b, v1, c, v2};
    }

    static std::optional<Record> fixed_record(std::string_view line) {
        // whole-token reading first (right-justified writers), then the fixed
        // column windows 5-12, 15-22, 25-36, 40-47, 50-61
        const std::vector<std::string> tok = split(line);
        if (tok.size() == 3 && !is_numeric(tok[0]) && !is_numeric(tok[1]) && is_numeric(tok[2]))
            return Record{tok[0], tok[1], *stod_like(tok[2], nullptr), std::string(), 0.0};
        if (tok.size() == 5 && !is_numeric(tok[0]) && !is_numeric(tok[1]) && is_numeric(tok[2]) &&
            !is_numeric(tok[3]) && is_numeric(tok[4]))
            return Record{tok[0], tok[1], *stod_like(tok[2], nullptr), tok[3], *stod_like(tok[4], nullptr)};
        auto field = [&](size_t off, size_t width) -> std::string {
            if (off > line.size()) return "";
            return std::string(line.substr(off, std::min(width, line.size() - off)));
        };
        auto value = [&](size_t off) {
            const auto v = stod_like(trim_ends(field(off, 12), " \t"), nullptr);
            return v ? *v : 0.0;
        };
        return Record{trim_ends(field(4, 8), " \t"), trim_ends(field(14, 8), " \t"), value(24),
                      trim_ends(field(39, 8), " \t"), value(49)};
    }

    void rows(std::string_view line) {
        Tokens t(line);
        std::string kind, name;
        t.str(kind);
        t.str(name);
        if (kind == "N") {
            obj_row_ = name;
            return;
        }
        int32_t sense = 0;  // LE
        if (kind == "L")
            sense = 0;
        else if (kind == "G")
            sense = 1;
        else if (kind == "E")
            sense = 2;
        else
            warn("Unknown row type: " + kind + " for row " + name);
        const int64_t i = static_cast<int64_t>(P.sense.size());
        if (name.empty()) name = "c" + std::to_string(i);
        row_of_.emplace(name, i);  // first row of a name answers lookups
        P.row_names.push_back(name);
        P.sense.push_back(sense);
        P.rhs.push_back(0.0);
        P.range_lo.push_back(-kInf);
        P.range_hi.push_back(kInf);
    }

    int64_t row(const std::string& name) const {
        const auto it = row_of_.find(name);
        return it == row_of_.end() ? -1 : it->second;
    }

    static bool marker(std::string_view line, bool& in_int) {
        std::vector<std::string> t = split(line);
        for (std::string& w : t) {
            if (w.size() >= 2 && w.front() == '\'') w.erase(0, 1);
            if (!w.empty() && w.back() == '\'') w.pop_back();
        }
        if (t.size() < 2) return false;
        bool has = false;
        std::string kind;
        for (const std::string& w : t) {
            const std::string u = upper(w);
            if (u == "MARKER") {
                has = true;
                continue;
            }
            if (u == "INTORG" || u == "INTEND") {
                kind = u;
                break;
            }
        }
        if (!has) return false;
        if (kind == "INTORG") in_int = true;
        if (kind == "INTEND") in_int = false;
        return true;
    }

    void columns(std::string_view line) {
        if (marker(line, in_int_)) return;
        const auto rec = record(line);
        if (!rec) return;
        const auto& [col, r1, v1, r2, v2] = *rec;
        if (col == "MARKER") return;
        int64_t j;
        const auto it = col_of_.find(col);
        if (it == col_of_.end()) {
            j = static_cast<int64_t>(P.c.size());
            col_of_.emplace(col, j);
            P.col_names.push_back(col);
            P.c.push_back(0.0);
            P.lb.push_back(0.0);
            P.ub.push_back(kInf);
            P.vtype.push_back(in_int_ ? INTEGER : CONTINUOUS);
        } else {
            j = it->second;
        }
        coeff(j, r1, v1);
        coeff(j, r2, v2);
    }

    void coeff(int64_t j, const std::string& r, double v) {
        if (r.empty() || v == 0.0) return;
        if (r == obj_row_) {
            P.c[j] = v;
            return;
        }
        const int64_t i = row(r);
        if (i >= 0) {
            P.trow.push_back(i);
            P.tcol.push_back(j);
            P.tval.push_back(v);
            return;
        }
        if (obj_row_.empty()) {  // no N row: the first unknown row is the objective
            obj_row_ = r;
            P.c[j] = v;
            warn("Implicit objective row '" + r + "' (no N row declared in ROWS)");
            return;
        }
        warn("Unknown row '" + r + "' referenced in COLUMNS is ignored");
    }

    bool set_rhs(const std::string& r, double v) {
        const int64_t i = row(r);
        if (i < 0) return false;
        P.rhs[i] = v;
        return true;
    }

    // the fixed-layout retry of an RHS line that free reading misplaced
    // (mps_parser.cpp:318-346); returns whether its first row matched
    bool rhs_retry(std::string_view line) {
        if (!(free_ && line.size() >= 50)) return false;
        const auto f = fixed_record(line);
        if (!f) return false;
        const auto& [fn, f1, fv1, f2, fv2] = *f;
        if (!f1.empty() && set_rhs(f1, fv1)) {
            if (!f2.empty()) set_rhs(f2, fv2);
            return true;
        }
        return false;
    }

    void rhs(std::string_view line) {
        const auto rec = record(line);
        if (!rec) return;
        const auto& [nm, r1, v1, r2, v2] = *rec;
        const bool m1 = !r1.empty() && set_rhs(r1, v1);
        if (!m1 && !r1.empty()) {
            if (rhs_retry(line)) return;
        } else if (r1.empty()) {
            if (!r2.empty()) set_rhs(r2, v2);
        }
        if (!r2.empty() && !set_rhs(r2, v2)) rhs_retry(line);
    }

    void range(const std::string& r, double v) {
        const int64_t i = row(r);
        if (i < 0) return;
        const double b = P.rhs[i];
        if (P.sense[i] == 0) {
            P.range_hi[i] = b + v;
            P.range_lo[i] = b;
        } else if (P.sense[i] == 1) {
            P.range_lo[i] = b - v;
            P.range_hi[i] = b;
        } else {
            P.range_lo[i] = b - std::abs(v);
            P.range_hi[i] = b + std::abs(v);
        }
    }

    void ranges(std::string_view line) {
        const auto rec = record(line);
        if (!rec) return;
        const auto& [nm, r1, v1, r2, v2] = *rec;
        if (!r1.empty()) range(r1, v1);
        if (!r2.empty()) range(r2, v2);
    }

    void bounds(std::string_view line) {
        // type, bound-set name and column are always read as three tokens
        Tokens t(line);
        std::string type, set, col;
        double v = 0.0;
        t.str(type);
        t.str(set);
        t.str(col);
        if (type != "FR" && type != "MI" && type != "PL") t.num(v);
        const auto it = col_of_.find(col);
        if (it == col_of_.end()) return;
        const int64_t j = it->second;
        if (type == "LO") {
            P.lb[j] = v;
        } else if (type == "UP") {
            P.ub[j] = v;
        } else if (type == "FX") {
            P.lb[j] = v;
            P.ub[j] = v;
        } else if (type == "FR") {
            P.lb[j] = -kInf;
            P.ub[j] = kInf;
        } else if (type == "MI") {
            P.lb[j] = -kInf;
        } else if (type == "PL") {
            P.ub[j] = kInf;
        } else if (type == "BV") {
            P.vtype[j] = BINARY;
            P.lb[j] = 0.0;
            P.ub[j] = 1.0;
        } else if (type == "UI") {
            P.vtype[j] = INTEGER;
            P.ub[j] = v;
        } else if (type == "LI") {
            P.vtype[j] = INTEGER;
            P.lb[j] = v;
        } else if (type == "SC") {
            P.vtype[j] = SEMI_CONTINUOUS;
            P.lb[j] = v;
        } else if (type == "SI") {
            P.vtype[j] = SEMI_INTEGER;
            P.lb[j] = v;
        }
    }
};

}  // namespace

void read_mps(std::string_view text, int format, MpsProblem& out) {
    out = MpsProblem{};
    Reader(out).run(text, format);
}

}  // namespace hn::model

// ---- C ABI ----
struct hn_mps {
    hn::model::MpsProblem p;
};

namespace {
int mps_fail(int code, const std::string& msg) {
    hn::set_host_error(msg);
    return code;
}
}  // namespace

extern "C" {

int hn_mps_read_string(const char* text, int64_t len, int format, hn_mps** out) {
    if (!out || (!text && len > 0) || len < 0 || format < -1 || format > 1)
        return mps_fail(HN_ERR_INVALID_ARG, "hn_mps_read_string: bad arguments");
    try {
        auto* h = new hn_mps;
        hn::model::read_mps(std::string_view(text ? text : "", static_cast<size_t>(len)), format, h->p);
        *out = h;
        return HN_OK;
    } catch (const std::bad_alloc&) {
        return mps_fail(HN_ERR_OUT_OF_MEMORY, "hn_mps_read_string: out of host memory");
    }
}

int hn_mps_read_file(const char* path, int format, hn_mps** out) {
    if (!path || !out) return mps_fail(HN_ERR_INVALID_ARG, "hn_mps_read_file: bad arguments");
    std::ifstream f(path, std::ios::binary);
    if (!f.is_open()) return mps_fail(HN_ERR_INVALID_ARG, std::string("Cannot open file: ") + path);
    std::ostringstream buf;
    buf << f.rdbuf();
    const std::string text = buf.str();
    return hn_mps_read_string(text.data(), static_cast<int64_t>(text.size()), format, out);
}

int hn_mps_shape(const hn_mps* h, int64_t* m, int64_t* n, int64_t* ntriplets, int* maximize) {
    if (!h) return mps_fail(HN_ERR_INVALID_ARG, "hn_mps_shape: null handle");
    if (m) *m = static_cast<int64_t>(h->p.sense.size());
    if (n) *n = static_cast<int64_t>(h->p.c.size());
    if (ntriplets) *ntriplets = static_cast<int64_t>(h->p.tval.size());
    if (maximize) *maximize = h->p.maximize;
    return HN_OK;
}

int hn_mps_arrays(const hn_mps* h, int64_t* trow, int64_t* tcol, double* tval, double* c, double* rhs,
                  int32_t* sense, double* lb, double* ub, double* range_lo, double* range_hi, int32_t* vtype) {
    if (!h) return mps_fail(HN_ERR_INVALID_ARG, "hn_mps_arrays: null handle");
    const auto& p = h->p;
    auto put = [](auto* dst, const auto& v) {
        if (dst && !v.empty()) std::memcpy(dst, v.data(), sizeof(v[0]) * v.size());
    };
    put(trow, p.trow);
    put(tcol, p.tcol);
    put(tval, p.tval);
    put(c, p.c);
    put(rhs, p.rhs);
    put(sense, p.sense);
    put(lb, p.lb);
    put(ub, p.ub);
    put(range_lo, p.range_lo);
    put(range_hi, p.range_hi);
    put(vtype, p.vtype);
    return HN_OK;
}

int hn_mps_counts(const hn_mps* h, int64_t* warnings, int64_t* sos_records, int64_t* quadratic_records) {
    if (!h) return mps_fail(HN_ERR_INVALID_ARG, "hn_mps_counts: null handle");
    if (warnings) *warnings = static_cast<int64_t>(h->p.warnings.size());
    if (sos_records) *sos_records = h->p.sos_records;
    if (quadratic_records) *quadratic_records = h->p.quadratic_records;
    return HN_OK;
}

const char* hn_mps_warning(const hn_mps* h, int64_t i) {
    if (!h || i < 0 || i >= static_cast<int64_t>(h->p.warnings.size())) return nullptr;
    return h->p.warnings[static_cast<size_t>(i)].c_str();
}

const char* hn_mps_name(const hn_mps* h, int what, int64_t i) {
    if (!h) return nullptr;
    if (what < 0) return h->p.name.c_str();
    const auto& v = what == 0 ? h->p.row_names : h->p.col_names;
    if (i < 0 || i >= static_cast<int64_t>(v.size())) return nullptr;
    return v[static_cast<size_t>(i)].c_str();
}

int hn_mps_free(hn_mps* h) {
    delete h;
    return HN_OK;
}

}  // extern "C"
