// Problem readers. MPS: HyperNova's MPSParser (core/model/mps_parser.cpp) restated with
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
#include <charconv>
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
#include "hn_read.hpp"
#include "hn_sm100.h"

namespace hn::model {
namespace {

constexpr double kInf = std::numeric_limits<double>::infinity();

enum class Section { NONE, NAME, ROWS, COLUMNS, RHS, RANGES, BOUNDS, SOS, QUADOBJ, QCMATRIX, OBJSENSE, ENDATA };
enum VarType : int32_t { CONTINUOUS = 0, INTEGER = 1, BINARY = 2, SEMI_CONTINUOUS = 3, SEMI_INTEGER = 4 };

using sv = std::string_view;

inline bool is_ws(char ch) {  // isspace in the C locale
    return ch == ' ' || ch == '\t' || ch == '\n' || ch == '\v' || ch == '\f' || ch == '\r';
}
inline char up(char ch) { return ch >= 'a' && ch <= 'z' ? static_cast<char>(ch - 'a' + 'A') : ch; }

// a == kw after upper-casing a (kw is upper case)
bool ieq(sv a, sv kw) {
    if (a.size() != kw.size()) return false;
    for (size_t i = 0; i < a.size(); ++i)
        if (up(a[i]) != kw[i]) return false;
    return true;
}

// strtod over a copy of s (NUL-terminated); `end` = characters used
double strtod_sv(sv s, size_t* used, bool* erange) {
    char buf[96];
    std::string big;
    const char* b = buf;
    if (s.size() < sizeof(buf)) {
        if (!s.empty()) std::memcpy(buf, s.data(), s.size());
        buf[s.size()] = '\0';
    } else {
        big.assign(s);
        b = big.c_str();
    }
    char* end = nullptr;
    errno = 0;
    const double v = std::strtod(b, &end);
    if (erange) *erange = errno == ERANGE;
    *used = static_cast<size_t>(end - b);
    return v;
}

// A cursor over one line with the extraction rules of std::istringstream:
// strings are whitespace-delimited tokens; a double reads the longest prefix
// of libstdc++'s float grammar (sign, digits with one point, exponent after a
// digit) and converts all of it (failing otherwise) with correct rounding,
// failing on overflow. Any failure sticks (later extractions fail).
class Tokens {
public:
    explicit Tokens(sv s) : s_(s) {}
    bool str(sv& out) {
        if (fail_) return false;
        skip();
        if (p_ >= s_.size()) {
            fail_ = true;  // the sentry fails: `out` is left as it was
            return false;
        }
        const size_t b = p_;
        while (p_ < s_.size() && !is_ws(s_[p_])) ++p_;
        out = s_.substr(b, p_ - b);
        return true;
    }
    bool num(double& out) {
        if (fail_) return false;
        skip();
        const size_t b = p_;
        size_t q = p_;
        bool mant = false, point = false;
        if (q < s_.size() && (s_[q] == '+' || s_[q] == '-')) ++q;
        while (q < s_.size()) {
            const char ch = s_[q];
            if (ch >= '0' && ch <= '9') {
                mant = true;
            } else if (ch == '.' && !point) {
                point = true;
            } else if ((ch == 'e' || ch == 'E') && mant) {
                ++q;
                if (q < s_.size() && (s_[q] == '+' || s_[q] == '-')) ++q;
                while (q < s_.size() && s_[q] >= '0' && s_[q] <= '9') ++q;
                break;
            } else {
                break;
            }
            ++q;
        }
        p_ = q;
        out = 0.0;
        sv acc = s_.substr(b, q - b);
        if (acc.empty()) return fail();
        // from_chars takes no '+'; its result is strtod's (both round correctly)
        sv digits = acc[0] == '+' ? acc.substr(1) : acc;
        double v = 0.0;
        const auto r = std::from_chars(digits.data(), digits.data() + digits.size(), v);
        if (r.ec == std::errc() && r.ptr == digits.data() + digits.size()) {
            out = v;
            return true;
        }
        // the rare cases (range errors, malformed text): strtod's own answer
        size_t used = 0;
        v = strtod_sv(acc, &used, nullptr);
        if (used != acc.size()) return fail();
        if (std::isinf(v)) {
            out = v > 0 ? std::numeric_limits<double>::max() : -std::numeric_limits<double>::max();
            return fail();
        }
        out = v;
        return true;
    }

private:
    bool fail() {
        fail_ = true;
        return false;
    }
    void skip() {
        while (p_ < s_.size() && is_ws(s_[p_])) ++p_;
    }
    sv s_;
    size_t p_ = 0;
    bool fail_ = false;
};

template <size_t N>
size_t split(sv s, sv (&out)[N]) {  // up to N tokens; returns the total count
    Tokens t(s);
    sv w;
    size_t k = 0;
    while (t.str(w)) {
        if (k < N) out[k] = w;
        ++k;
    }
    return k;
}

// std::stod: strtod over a prefix; throws (here: nullopt) on no conversion or
// ERANGE; `used` gets the characters consumed
std::optional<double> stod_like(sv s, size_t* used) {
    size_t u = 0;
    bool erange = false;
    const double v = strtod_sv(s, &u, &erange);
    if (u == 0 || erange) return std::nullopt;
    if (used) *used = u;
    return v;
}

bool is_numeric(sv s) {
    if (s.empty()) return false;
    size_t used = 0;
    const auto v = stod_like(s, &used);
    return v && used == s.size();
}

sv trim_ends(sv s, const char* set) {
    const size_t b = s.find_first_not_of(set);
    if (b == sv::npos) return sv();
    const size_t e = s.find_last_not_of(set);
    return s.substr(b, e - b + 1);
}

struct Record {
    sv a, b;
    double v1;
    sv c;
    double v2;
};

Section detect_section(sv line) {
    Tokens t(line);
    sv first, second;
    t.str(first);
    const bool single = !t.str(second);
    if (first.size() < 3 || first.size() > 8) return Section::NONE;
    if (ieq(first, "NAME")) return Section::NAME;
    if (ieq(first, "OBJSENSE")) return Section::OBJSENSE;
    if (!single) return Section::NONE;
    if (ieq(first, "ROWS")) return Section::ROWS;
    if (ieq(first, "COLUMNS")) return Section::COLUMNS;
    if (ieq(first, "RHS")) return Section::RHS;
    if (ieq(first, "RANGES")) return Section::RANGES;
    if (ieq(first, "BOUNDS")) return Section::BOUNDS;
    if (ieq(first, "SOS")) return Section::SOS;
    if (ieq(first, "QUADOBJ")) return Section::QUADOBJ;
    if (ieq(first, "QCMATRIX")) return Section::QCMATRIX;
    if (ieq(first, "ENDATA")) return Section::ENDATA;
    return Section::NONE;
}

// the reference's layout probe (mps_parser.cpp:124-158): over the first 8
// COLUMNS data lines, the position of the second non-blank character; fixed
// layout when at least 3 were sampled and half of them sit at index 14
bool detect_free(const std::vector<sv>& lines) {
    bool in_columns = false;
    int samples = 0, aligned = 0;
    for (sv line : lines) {
        const size_t lead = line.find_first_not_of(" \t\r\n");
        if (lead == sv::npos) continue;
        sv trimmed = line.substr(lead);
        if (trimmed[0] == '*') continue;
        const Section sec = detect_section(trimmed);
        if (sec != Section::NONE) {
            in_columns = (sec == Section::COLUMNS);
            continue;
        }
        if (!in_columns) continue;
        const size_t a = line.find_first_not_of(" \t");
        if (a == sv::npos) continue;
        const size_t b = line.find_first_not_of(" \t", a + 1);
        if (b == sv::npos) continue;
        ++samples;
        if (b == 14) ++aligned;
        if (samples >= 8) break;
    }
    return !(samples >= 3 && aligned * 2 >= samples);
}

// Names -> first index: open addressing over (hash, index) slots, the names
// themselves kept by the caller's vector; a slot is compared by hash first.
class NameIndex {
public:
    explicit NameIndex(const std::vector<std::string>& names) : names_(names) { slots_.assign(64, Slot{0, -1}); }
    int64_t find(sv name) const {
        const uint64_t h = hash(name);
        for (size_t i = h & (slots_.size() - 1);; i = (i + 1) & (slots_.size() - 1)) {
            const Slot& s = slots_[i];
            if (s.idx < 0) return -1;
            if (s.h == h && names_[static_cast<size_t>(s.idx)] == name) return s.idx;
        }
    }
    // records names_[idx] unless the name is already present (first wins)
    void add(int64_t idx) {
        if (4 * (count_ + 1) > 3 * slots_.size()) grow();
        const sv name = names_[static_cast<size_t>(idx)];
        const uint64_t h = hash(name);
        for (size_t i = h & (slots_.size() - 1);; i = (i + 1) & (slots_.size() - 1)) {
            Slot& s = slots_[i];
            if (s.idx < 0) {
                s = Slot{h, idx};
                ++count_;
                return;
            }
            if (s.h == h && names_[static_cast<size_t>(s.idx)] == name) return;
        }
    }

private:
    struct Slot {
        uint64_t h;
        int64_t idx;
    };
    static uint64_t hash(sv s) {  // FNV-1a, then a 64-bit finaliser
        uint64_t h = 1469598103934665603ull;
        for (const char ch : s) h = (h ^ static_cast<unsigned char>(ch)) * 1099511628211ull;
        h ^= h >> 33;
        h *= 0xff51afd7ed558ccdull;
        h ^= h >> 33;
        return h;
    }
    void grow() {
        std::vector<Slot> old;
        old.swap(slots_);
        slots_.assign(old.size() * 2, Slot{0, -1});
        for (const Slot& o : old) {
            if (o.idx < 0) continue;
            size_t i = o.h & (slots_.size() - 1);
            while (slots_[i].idx >= 0) i = (i + 1) & (slots_.size() - 1);
            slots_[i] = o;
        }
    }
    const std::vector<std::string>& names_;
    std::vector<Slot> slots_;
    size_t count_ = 0;
};

class Reader {
public:
    explicit Reader(ReadProblem& out) : P(out), row_of_(out.row_names), col_of_(out.col_names) {}

    void run(sv text, int format) {
        std::vector<sv> lines;
        size_t b = 0;
        while (b < text.size()) {  // std::getline on '\n'
            size_t e = text.find('\n', b);
            if (e == sv::npos) e = text.size();
            lines.push_back(text.substr(b, e - b));
            b = e + 1;
        }
        free_ = format < 0 ? detect_free(lines) : format == 0;
        Section cur = Section::NONE;
        for (sv line : lines) {
            const sv trimmed = trim_ends(line, " \t\r\n");
            if (trimmed.empty() || trimmed[0] == '*') continue;
            const Section sec = detect_section(trimmed);
            if (sec != Section::NONE) {
                cur = sec;
                if (sec == Section::NAME) {
                    name_line(trimmed);
                } else if (sec == Section::OBJSENSE) {
                    Tokens t(trimmed);
                    sv s;
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
                    sv s;
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
    ReadProblem& P;
    bool free_ = true;
    bool in_int_ = false;
    std::string obj_row_;
    NameIndex row_of_, col_of_;
    int64_t last_col_ = -1;  // COLUMNS lists a column's entries together

    void warn(std::string msg) { P.warnings.push_back(std::move(msg)); }

    void objsense(sv s) {
        if (ieq(s, "MAX") || ieq(s, "MAXIMIZE")) P.maximize = 1;
    }

    void name_line(sv line) {
        Tokens t(line);
        sv s;
        t.str(s);
        if (t.str(s)) P.name.assign(s);
    }

    std::optional<Record> record(sv line) const { return free_ ? free_record(line) : fixed_record(line); }

    static std::optional<Record> free_record(sv line) {
        Tokens t(line);
        Record r{sv(), sv(), 0.0, sv(), 0.0};
        if (!t.str(r.a) || !t.str(r.b) || !t.num(r.v1)) return std::nullopt;
        if (!t.str(r.c)) r.c = sv();
        if (!t.num(r.v2)) r.v2 = 0.0;
        return r;
    }

    static std::optional<Record> fixed_record(sv line) {
        // whole-token reading first (right-justified writers), then the fixed
        // column windows 5-12, 15-22, 25-36, 40-47, 50-61
        sv tok[6];
        const size_t nt = split(line, tok);
        if (nt == 3 && !is_numeric(tok[0]) && !is_numeric(tok[1]) && is_numeric(tok[2]))
            return Record{tok[0], tok[1], *stod_like(tok[2], nullptr), sv(), 0.0};
        if (nt == 5 && !is_numeric(tok[0]) && !is_numeric(tok[1]) && is_numeric(tok[2]) && !is_numeric(tok[3]) &&
            is_numeric(tok[4]))
            return Record{tok[0], tok[1], *stod_like(tok[2], nullptr), tok[3], *stod_like(tok[4], nullptr)};
        auto field = [&](size_t off, size_t width) -> sv {
            if (off > line.size()) return sv();
            return line.substr(off, std::min(width, line.size() - off));
        };
        auto value = [&](size_t off) {
            const auto v = stod_like(trim_ends(field(off, 12), " \t"), nullptr);
            return v ? *v : 0.0;
        };
        return Record{trim_ends(field(4, 8), " \t"), trim_ends(field(14, 8), " \t"), value(24),
                      trim_ends(field(39, 8), " \t"), value(49)};
    }

    void rows(sv line) {
        Tokens t(line);
        sv kind, nm;
        t.str(kind);
        t.str(nm);
        if (kind == "N") {
            obj_row_.assign(nm);
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
            warn("Unknown row type: " + std::string(kind) + " for row " + std::string(nm));
        const int64_t i = static_cast<int64_t>(P.sense.size());
        P.row_names.push_back(nm.empty() ? "c" + std::to_string(i) : std::string(nm));
        row_of_.add(i);  // the first row of a name answers lookups
        P.sense.push_back(sense);
        P.rhs.push_back(0.0);
        P.range_lo.push_back(-kInf);
        P.range_hi.push_back(kInf);
    }

    int64_t row(sv name) const { return row_of_.find(name); }

    static bool marker(sv line, bool& in_int) {
        // a marker record has a token "MARKER" (quotes stripped, any case):
        // no such substring, no marker
        bool any = false;
        for (size_t i = 0; i + 6 <= line.size() && !any; ++i)
            any = up(line[i]) == 'M' && ieq(line.substr(i, 6), "MARKER");
        if (!any) return false;
        sv t[64];
        const size_t nt = split(line, t);
        if (nt < 2) return false;
        bool has = false;
        int kind = 0;  // 1 INTORG, 2 INTEND
        for (size_t i = 0; i < nt && i < 64; ++i) {
            sv w = t[i];
            if (w.size() >= 2 && w.front() == '\'') w.remove_prefix(1);
            if (!w.empty() && w.back() == '\'') w.remove_suffix(1);
            if (ieq(w, "MARKER")) {
                has = true;
                continue;
            }
            if (ieq(w, "INTORG")) {
                kind = 1;
                break;
            }
            if (ieq(w, "INTEND")) {
                kind = 2;
                break;
            }
        }
        if (!has) return false;
        if (kind == 1) in_int = true;
        if (kind == 2) in_int = false;
        return true;
    }

    void columns(sv line) {
        if (marker(line, in_int_)) return;
        const auto rec = record(line);
        if (!rec) return;
        if (rec->a == "MARKER") return;
        int64_t j = last_col_ >= 0 && P.col_names[static_cast<size_t>(last_col_)] == rec->a ? last_col_
                                                                                            : col_of_.find(rec->a);
        if (j < 0) {
            j = static_cast<int64_t>(P.c.size());
            P.col_names.emplace_back(rec->a);
            col_of_.add(j);
            P.c.push_back(0.0);
            P.lb.push_back(0.0);
            P.ub.push_back(kInf);
            P.vtype.push_back(in_int_ ? INTEGER : CONTINUOUS);
        }
        last_col_ = j;
        coeff(j, rec->b, rec->v1);
        coeff(j, rec->c, rec->v2);
    }

    void coeff(int64_t j, sv r, double v) {
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
            obj_row_.assign(r);
            P.c[j] = v;
            warn("Implicit objective row '" + std::string(r) + "' (no N row declared in ROWS)");
            return;
        }
        warn("Unknown row '" + std::string(r) + "' referenced in COLUMNS is ignored");
    }

    bool set_rhs(sv r, double v) {
        const int64_t i = row(r);
        if (i < 0) return false;
        P.rhs[i] = v;
        return true;
    }

    // the fixed-layout retry of an RHS line that free reading misplaced
    // (mps_parser.cpp:318-346); returns whether its first row matched
    bool rhs_retry(sv line) {
        if (!(free_ && line.size() >= 50)) return false;
        const auto f = fixed_record(line);
        if (!f) return false;
        if (!f->b.empty() && set_rhs(f->b, f->v1)) {
            if (!f->c.empty()) set_rhs(f->c, f->v2);
            return true;
        }
        return false;
    }

    void rhs(sv line) {
        const auto rec = record(line);
        if (!rec) return;
        const sv r1 = rec->b, r2 = rec->c;
        const bool m1 = !r1.empty() && set_rhs(r1, rec->v1);
        if (!m1 && !r1.empty()) {
            if (rhs_retry(line)) return;
        } else if (r1.empty()) {
            if (!r2.empty()) set_rhs(r2, rec->v2);
        }
        if (!r2.empty() && !set_rhs(r2, rec->v2)) rhs_retry(line);
    }

    void range(sv r, double v) {
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

    void ranges(sv line) {
        const auto rec = record(line);
        if (!rec) return;
        if (!rec->b.empty()) range(rec->b, rec->v1);
        if (!rec->c.empty()) range(rec->c, rec->v2);
    }

    void bounds(sv line) {
        // type, bound-set name and column are always read as three tokens
        Tokens t(line);
        sv type, set, col;
        double v = 0.0;
        t.str(type);
        t.str(set);
        t.str(col);
        if (type != "FR" && type != "MI" && type != "PL") t.num(v);
        const int64_t j = col_of_.find(col);
        if (j < 0) return;
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

// ---- LP text: model::LPParser (core/model/lp_parser.cpp) restated ----
// Variables are created where the reference creates them: at their first
// mention in the objective's linear part, then its bracketed quadratic
// groups, then constraint left-hand sides and the QUADRATIC section, so the
// column order matches. Every place where the reference would record an
// error or let std::stod throw makes the read fail.

inline bool c_space(char ch) { return ch == ' ' || (ch >= '\t' && ch <= '\r'); }  // isspace, C locale
inline bool c_digit(char ch) { return ch >= '0' && ch <= '9'; }
inline bool c_alpha(char ch) { return (ch >= 'a' && ch <= 'z') || (ch >= 'A' && ch <= 'Z'); }
inline bool c_alnum(char ch) { return c_digit(ch) || c_alpha(ch); }

struct LpFail : std::exception {};

double stod_or_throw(sv s) {  // std::stod: prefix conversion, throws on none or ERANGE
    const auto v = stod_like(s, nullptr);
    if (!v) throw LpFail();
    return *v;
}

class LpReader {
public:
    explicit LpReader(ReadProblem& out) : P(out), col_of_(out.col_names) {}

    void run(sv text) {
        enum class Sec { NONE, OBJ, CONSTRAINTS, BOUNDS, GENERAL, BINARY, SEMI, SOS, QUADRATIC, END };
        auto section = [&](sv t) -> Sec {
            if (ieq(t, "MINIMIZE") || ieq(t, "MAXIMIZE") || ieq(t, "MIN") || ieq(t, "MAX")) {
                P.maximize = (ieq(t, "MAXIMIZE") || ieq(t, "MAX")) ? 1 : 0;
                return Sec::OBJ;
            }
            if (ieq(t, "SUBJECT TO") || ieq(t, "ST") || ieq(t, "S.T.") || ieq(t, "CONSTRAINTS")) return Sec::CONSTRAINTS;
            if (ieq(t, "BOUNDS")) return Sec::BOUNDS;
            if (ieq(t, "GENERAL") || ieq(t, "GENERALS")) return Sec::GENERAL;
            if (ieq(t, "BINARY") || ieq(t, "BINARIES")) return Sec::BINARY;
            if (ieq(t, "SEMI-CONTINUOUS") || ieq(t, "SEMI-CONT") || ieq(t, "SEMI-INTEGER") || ieq(t, "SEMI-INT"))
                return Sec::SEMI;
            if (ieq(t, "SOS")) return Sec::SOS;
            if (ieq(t, "QUADRATIC") || ieq(t, "Q")) return Sec::QUADRATIC;
            if (ieq(t, "END")) return Sec::END;
            return Sec::NONE;
        };
        Sec cur = Sec::NONE;
        int64_t line_no = 0;
        size_t b = 0;
        while (b < text.size()) {  // std::getline on '\n'
            size_t e = text.find('\n', b);
            if (e == sv::npos) e = text.size();
            const sv line = text.substr(b, e - b);
            b = e + 1;
            ++line_no;
            const sv t = trim_ends(line, " \t\r\n");
            if (t.empty() || t[0] == '\\' || (t.size() >= 2 && t[0] == '*' && t[1] == '*')) continue;
            const Sec ns = section(t);
            if (ns != Sec::NONE) {
                // the reference finalises outside its per-line try block
                guarded(line_no, [&] {
                    if (cur == Sec::OBJ) finalize_obj();
                    if (cur == Sec::CONSTRAINTS) finalize_constraint();
                });
                cur = ns;
                continue;
            }
            if (cur == Sec::END) break;
            guarded(line_no, [&] {
                switch (cur) {
                    case Sec::OBJ: {
                        sv ex = t;
                        const size_t colon = ex.find(':');
                        if (colon != sv::npos) ex = ex.substr(colon + 1);
                        obj_buf_ += ' ';
                        obj_buf_ += ex;
                        break;
                    }
                    case Sec::CONSTRAINTS: {
                        const size_t colon = t.find(':');
                        if (colon != sv::npos) {
                            if (!acc_.empty()) {
                                error("Unterminated constraint before: " + std::string(t));
                                acc_.clear();
                                acc_name_.clear();
                            }
                            acc_name_.assign(trim_ends(t.substr(0, colon), " \t\r\n"));
                            acc_.assign(trim_ends(t.substr(colon + 1), " \t\r\n"));
                        } else {
                            acc_ += ' ';
                            acc_ += t;
                        }
                        if (acc_.find("<=") != std::string::npos || acc_.find(">=") != std::string::npos ||
                            acc_.find('=') != std::string::npos)
                            finalize_constraint();
                        break;
                    }
                    case Sec::BOUNDS: bounds(t); break;
                    case Sec::GENERAL: types(t, false); break;
                    case Sec::BINARY: types(t, true); break;
                    case Sec::SOS: ++P.sos_records; break;
                    case Sec::QUADRATIC: P.quadratic_records += quadratic_expr(t); break;
                    default: break;
                }
            });
        }
        guarded(line_no, [&] {
            if (cur == Sec::OBJ) finalize_obj();
            if (cur == Sec::CONSTRAINTS) finalize_constraint();
        });
    }

private:
    ReadProblem& P;
    NameIndex col_of_;
    std::string obj_buf_, acc_, acc_name_;

    void error(std::string msg) { P.errors.push_back(std::move(msg)); }

    template <class F>
    void guarded(int64_t line_no, F&& f) {
        try {
            f();
        } catch (const LpFail&) {
            error("Line " + std::to_string(line_no) + ": stod");
        }
    }

    int64_t column(sv name) {
        int64_t j = col_of_.find(name);
        if (j >= 0) return j;
        j = static_cast<int64_t>(P.c.size());
        P.col_names.emplace_back(name);
        col_of_.add(j);
        P.c.push_back(0.0);
        P.lb.push_back(0.0);
        P.ub.push_back(kInf);
        P.vtype.push_back(CONTINUOUS);
        return j;
    }

    // LPParser::parse_linear_expr (lp_parser.cpp:384-443)
    std::vector<std::pair<int64_t, double>> linear_expr(sv s) {
        std::vector<std::pair<int64_t, double>> terms;
        size_t pos = 0;
        const size_t n = s.size();
        while (pos < n) {
            while (pos < n && c_space(s[pos])) ++pos;
            if (pos >= n) break;
            double sign = 1.0;
            if (s[pos] == '+') {
                ++pos;
            } else if (s[pos] == '-') {
                sign = -1.0;
                ++pos;
            }
            while (pos < n && c_space(s[pos])) ++pos;
            const size_t old = pos;
            double coeff = 1.0;
            size_t ce = pos;
            while (ce < n && (c_digit(s[ce]) || s[ce] == '.')) ++ce;
            if (ce < n && (s[ce] == 'e' || s[ce] == 'E')) {
                size_t en = ce + 1;
                if (en < n && (s[en] == '+' || s[en] == '-')) ++en;
                size_t ed = en;
                while (ed < n && c_digit(s[ed])) ++ed;
                if (ed > en) ce = ed;
            }
            if (ce > pos) {
                coeff = stod_or_throw(s.substr(pos, ce - pos));
                pos = ce;
            }
            while (pos < n && c_space(s[pos])) ++pos;
            const size_t vs = pos;
            while (pos < n && (c_alnum(s[pos]) || s[pos] == '_')) ++pos;
            if (pos > vs) {
                const int64_t j = column(s.substr(vs, pos - vs));
                terms.emplace_back(j, sign * coeff);
            } else if (pos == old) {
                ++pos;
            }
        }
        return terms;
    }

    // LPParser::parse_quadratic_expr (lp_parser.cpp:445-584): only its
    // variable creation matters to an LP; returns the number of terms
    int64_t quadratic_expr(sv ex) {
        enum class K { NUM, NAME, SEP, POWER };
        struct Tok {
            K k;
            sv name;
        };
        std::vector<Tok> toks;
        size_t pos = 0;
        const size_t n = ex.size();
        auto skip = [&] {
            while (pos < n && c_space(ex[pos])) ++pos;
        };
        while (pos < n) {
            skip();
            if (pos >= n) break;
            char ch = ex[pos];
            if (ch == '\\') break;
            if (ch == '*' || ch == '/') {
                toks.push_back({K::SEP, sv()});
                ++pos;
                continue;
            }
            if (ch == '^') {
                toks.push_back({K::POWER, sv()});
                ++pos;
                continue;
            }
            if (ch == '[' || ch == ']' || ch == '"' || ch == ',') {
                ++pos;
                continue;
            }
            if (ch == '+' || ch == '-') {
                ++pos;
                skip();
                if (pos >= n) break;
                ch = ex[pos];
            }
            if (c_digit(ch) || ch == '.') {
                const size_t st = pos;
                while (pos < n && (c_digit(ex[pos]) || ex[pos] == '.' || ex[pos] == 'e' || ex[pos] == 'E' ||
                                   ex[pos] == '+' || ex[pos] == '-'))
                    ++pos;
                stod_or_throw(ex.substr(st, pos - st));
                toks.push_back({K::NUM, sv()});
                continue;
            }
            if (c_alpha(ch) || ch == '_') {
                const size_t st = pos;
                while (pos < n && (c_alnum(ex[pos]) || ex[pos] == '_')) ++pos;
                toks.push_back({K::NAME, ex.substr(st, pos - st)});
                continue;
            }
            ++pos;  // stray character
        }
        int64_t count = 0;
        size_t i = 0;
        const size_t nt = toks.size();
        while (i < nt) {
            if (toks[i].k == K::SEP || toks[i].k == K::POWER) {
                ++i;
                continue;
            }
            bool lead = false;
            if (toks[i].k == K::NUM) {
                lead = true;
                ++i;
                while (i < nt && (toks[i].k == K::SEP || toks[i].k == K::POWER)) ++i;
            }
            if (i >= nt) break;
            if (toks[i].k != K::NAME) {
                if (toks[i].k == K::NUM) ++i;
                continue;
            }
            const sv v1 = toks[i].name;
            ++i;
            sv v2 = v1;
            if (i < nt && toks[i].k == K::POWER) {
                ++i;
                if (i < nt && toks[i].k == K::NUM) ++i;
            } else if (i < nt && toks[i].k == K::SEP) {
                ++i;
                if (i < nt && toks[i].k == K::NAME) {
                    v2 = toks[i].name;
                    ++i;
                }
            } else if (i < nt && toks[i].k == K::NAME) {
                v2 = toks[i].name;
                ++i;
            }
            if (!lead && i < nt && toks[i].k == K::NUM) ++i;
            column(v1);
            column(v2);
            ++count;
        }
        return count;
    }

    void finalize_obj() {
        if (obj_buf_.empty()) return;
        std::string linear, cur;
        std::vector<std::string> groups;
        int depth = 0;
        for (const char ch : obj_buf_) {
            if (ch == '[') {
                ++depth;
                continue;
            }
            if (ch == ']') {
                if (depth > 0 && --depth == 0) {
                    groups.emplace_back(trim_ends(cur, " \t\r\n"));
                    cur.clear();
                }
                continue;
            }
            (depth > 0 ? cur : linear) += ch;
        }
        if (depth > 0 && !trim_ends(cur, " \t\r\n").empty()) groups.emplace_back(trim_ends(cur, " \t\r\n"));
        for (const auto& [j, v] : linear_expr(linear)) P.c[static_cast<size_t>(j)] = v;
        for (const std::string& g : groups)
            if (!g.empty()) P.quadratic_records += quadratic_expr(g);
        obj_buf_.clear();
    }

    void finalize_constraint() {
        if (acc_.empty() && acc_name_.empty()) return;
        const std::string ex = acc_;
        int32_t sense = 0;
        size_t sp = std::string::npos;
        for (size_t i = 0; i + 1 < ex.size(); ++i) {
            if (ex[i] == '<' && ex[i + 1] == '=') {
                sp = i;
                sense = 0;
                break;
            }
            if (ex[i] == '>' && ex[i + 1] == '=') {
                sp = i;
                sense = 1;
                break;
            }
        }
        if (sp == std::string::npos) {
            sp = ex.find('=');
            if (sp != std::string::npos) sense = 2;
        }
        if (sp == std::string::npos) {
            error("Invalid constraint format: " + ex);
            acc_.clear();
            acc_name_.clear();
            return;
        }
        const sv lhs = trim_ends(sv(ex).substr(0, sp), " \t\r\n");
        const sv rhs_s = trim_ends(sv(ex).substr(sp + (sense == 2 ? 1 : 2)), " \t\r\n");
        if (rhs_s.empty()) return;  // the reference keeps the text for the next line
        const auto rhs = stod_like(rhs_s, nullptr);
        if (!rhs) {
            error("Invalid constraint RHS: " + std::string(rhs_s));
            acc_.clear();
            acc_name_.clear();
            return;
        }
        const auto terms = linear_expr(lhs);
        const int64_t i = static_cast<int64_t>(P.sense.size());
        P.row_names.push_back(acc_name_.empty() ? "c" + std::to_string(i) : acc_name_);
        P.sense.push_back(sense);
        P.rhs.push_back(*rhs);
        P.range_lo.push_back(-kInf);
        P.range_hi.push_back(kInf);
        for (const auto& [j, v] : terms) {
            P.trow.push_back(i);
            P.tcol.push_back(j);
            P.tval.push_back(v);
        }
        acc_.clear();
        acc_name_.clear();
    }

    // NUM of the bound patterns: -?(\d+\.?\d*|\.\d+|inf)
    static bool bound_num(sv s, size_t& p, sv& out) {
        const size_t st = p;
        size_t q = p;
        if (q < s.size() && s[q] == '-') ++q;
        if (s.substr(q, 3) == "inf") {
            q += 3;
        } else if (q < s.size() && c_digit(s[q])) {
            while (q < s.size() && c_digit(s[q])) ++q;
            if (q < s.size() && s[q] == '.') ++q;
            while (q < s.size() && c_digit(s[q])) ++q;
        } else if (q + 1 < s.size() && s[q] == '.' && c_digit(s[q + 1])) {
            ++q;
            while (q < s.size() && c_digit(s[q])) ++q;
        } else {
            return false;
        }
        out = s.substr(st, q - st);
        p = q;
        return true;
    }
    // NAME of the bound patterns: [a-zA-Z_][a-zA-Z0-9_]*
    static bool bound_name(sv s, size_t& p, sv& out) {
        if (p >= s.size() || !(c_alpha(s[p]) || s[p] == '_')) return false;
        const size_t st = p++;
        while (p < s.size() && (c_alnum(s[p]) || s[p] == '_')) ++p;
        out = s.substr(st, p - st);
        return true;
    }
    static void ws(sv s, size_t& p) {
        while (p < s.size() && c_space(s[p])) ++p;
    }
    static bool lit(sv s, size_t& p, sv op) {
        if (s.substr(p, op.size()) != op) return false;
        p += op.size();
        return true;
    }
    static double bound_value(sv tok) {
        std::string low(tok);
        for (char& ch : low)
            if (ch >= 'A' && ch <= 'Z') ch = static_cast<char>(ch - 'A' + 'a');
        if (low == "inf" || low == "+inf" || low == "infinity") return kInf;
        if (low == "-inf" || low == "-infinity") return -kInf;
        return stod_or_throw(tok);
    }

    // LPParser::parse_bounds (lp_parser.cpp:242-313): the five whole-line
    // patterns in the reference's order
    void bounds(sv line) {
        sv name, a, c;
        bool has_lb = false, has_ub = false, fixed = false;
        double lb = -kInf, ub = kInf;
        auto at_end = [&](size_t p) {
            ws(line, p);
            return p == line.size();
        };
        size_t p = 0;
        bool ok = false;
        // NUM <= NAME <= NUM  |  NUM <= NAME
        ws(line, p);
        if (bound_num(line, p, a) && (ws(line, p), lit(line, p, "<=")) && (ws(line, p), bound_name(line, p, name))) {
            const size_t after = p;
            size_t q = p;
            ws(line, q);
            if (lit(line, q, "<=") && (ws(line, q), bound_num(line, q, c)) && at_end(q)) {
                lb = bound_value(a);
                ub = bound_value(c);
                has_lb = has_ub = ok = true;
            } else if (at_end(after)) {
                lb = bound_value(a);
                has_lb = ok = true;
            }
        }
        if (!ok) {
            // NAME <= NUM  |  NAME >= NUM  |  NAME = NUM
            p = 0;
            ws(line, p);
            sv nm;
            if (bound_name(line, p, nm)) {
                ws(line, p);
                const sv ops[3] = {"<=", ">=", "="};
                for (int k = 0; k < 3 && !ok; ++k) {
                    size_t q = p;
                    if (lit(line, q, ops[k]) && (ws(line, q), bound_num(line, q, c)) && at_end(q)) {
                        name = nm;
                        const double v = bound_value(c);
                        if (k == 0) {
                            ub = v;
                            has_ub = true;
                        } else if (k == 1) {
                            lb = v;
                            has_lb = true;
                        } else {
                            lb = ub = v;
                            has_lb = has_ub = fixed = true;
                        }
                        ok = true;
                    }
                }
            }
        }
        if (!ok) name = line;  // no pattern: the whole line as a name
        const int64_t j = col_of_.find(name);
        if (j < 0) return;
        if (fixed) {
            P.lb[j] = lb;
            P.ub[j] = ub;
        } else {
            if (has_lb) P.lb[j] = lb;
            if (has_ub) P.ub[j] = ub;
        }
    }

    void types(sv line, bool binary) {
        Tokens t(line);
        sv w;
        while (t.str(w)) {
            const int64_t j = col_of_.find(w);
            if (j < 0) continue;
            P.vtype[j] = binary ? BINARY : INTEGER;
            if (binary) {
                P.lb[j] = 0.0;
                P.ub[j] = 1.0;
            }
        }
    }
};

}  // namespace

void read_mps(std::string_view text, int format, ReadProblem& out) {
    out = ReadProblem{};
    Reader(out).run(text, format);
}

void read_lp(std::string_view text, ReadProblem& out) {
    out = ReadProblem{};
    LpReader(out).run(text);
}

}  // namespace hn::model

// ---- C ABI ----
struct hn_mps {
    hn::model::ReadProblem p;
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

int hn_lp_read_string(const char* text, int64_t len, hn_mps** out) {
    if (!out || (!text && len > 0) || len < 0) return mps_fail(HN_ERR_INVALID_ARG, "hn_lp_read_string: bad arguments");
    *out = nullptr;
    try {
        auto* h = new hn_mps;
        hn::model::read_lp(std::string_view(text ? text : "", static_cast<size_t>(len)), h->p);
        if (!h->p.errors.empty()) {
            const std::string msg = "LP text rejected (" + std::to_string(h->p.errors.size()) +
                                    " errors), first: " + h->p.errors.front();
            delete h;
            return mps_fail(HN_ERR_INVALID_ARG, msg);
        }
        *out = h;
        return HN_OK;
    } catch (const std::bad_alloc&) {
        return mps_fail(HN_ERR_OUT_OF_MEMORY, "hn_lp_read_string: out of host memory");
    }
}

int hn_lp_read_file(const char* path, hn_mps** out) {
    if (!path || !out) return mps_fail(HN_ERR_INVALID_ARG, "hn_lp_read_file: bad arguments");
    std::ifstream f(path, std::ios::binary);
    if (!f.is_open()) return mps_fail(HN_ERR_INVALID_ARG, std::string("Cannot open file: ") + path);
    std::ostringstream buf;
    buf << f.rdbuf();
    const std::string text = buf.str();
    return hn_lp_read_string(text.data(), static_cast<int64_t>(text.size()), out);
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
