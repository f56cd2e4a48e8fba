// MPS reader of the host layer (hn_mps.cpp): the problem as arrays, the
// constraint coefficients as triplets in file order.
#pragma once
#include <cstdint>
#include <string>
#include <string_view>
#include <vector>

namespace hn::model {

struct MpsProblem {
    std::string name;
    int maximize = 0;
    // rows: sense 0 LE, 1 GE, 2 EQ (model::ConstraintSense); rhs; the RANGES
    // interval (-inf, +inf when none)
    std::vector<std::string> row_names;
    std::vector<int32_t> sense;
    std::vector<double> rhs, range_lo, range_hi;
    // columns: objective coefficient, bounds, model::VarType
    std::vector<std::string> col_names;
    std::vector<double> c, lb, ub;
    std::vector<int32_t> vtype;
    // constraint coefficients in file order (duplicates kept)
    std::vector<int64_t> trow, tcol;
    std::vector<double> tval;
    std::vector<std::string> warnings;
    int64_t sos_records = 0, quadratic_records = 0;  // read past, not kept
};

// format: -1 detect as the reference does, 0 free, 1 fixed
void read_mps(std::string_view text, int format, MpsProblem& out);

}  // namespace hn::model

namespace hn {
void set_host_error(const std::string& msg);  // text for hn_host_last_error
}
