// Problem readers of the host layer (hn_read.cpp): MPS and LP text to the
// problem as arrays, the constraint coefficients as triplets in file order.
#pragma once
#include <cstdint>
#include <string>
#include <string_view>
#include <vector>

namespace hn::model {

struct ReadProblem {
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
    std::vector<std::string> errors;  // the reference would report the read as failed
    int64_t sos_records = 0, quadratic_records = 0;  // read past, not kept
};

// format: -1 detect as the reference does, 0 free, 1 fixed
void read_mps(std::string_view text, int format, ReadProblem& out);
// CPLEX-style LP text with model::LPParser's results
void read_lp(std::string_view text, ReadProblem& out);

}  // namespace hn::model

namespace hn {
void set_host_error(const std::string& msg);  // text for hn_host_last_error
}
