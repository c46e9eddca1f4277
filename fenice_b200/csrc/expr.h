// Case-file expressions as programs for the device.
//
// The reference evaluates the values of a case file that are not plain numbers (the source terms source_rho ..
// source_mz, the time-dependent boundary values u_in, v_in, rho_in, p_out, the initial states) with TinyExpr (its
// vendored cpp/third_party/tinyexpr, built with TE_POW_FROM_RIGHT), binding x, y, z, t, every numeric run parameter and
// the mesh's Lx, Ly, Lz, nx, ny, nz (the Evaluator of cpp/src/CaseFile.cpp:299-377). Here one compiler (expr.cu) reads
// the same grammar, folds every part that depends on neither x, y, z nor t with the host's C library (so those parts
// carry the reference's bits), and emits a postfix program of Op codes over a constant pool. The program runs on the
// host (the C library's functions: the reference's values) and on the device (expr.cuh: CUDA's functions, within their
// documented ulp bounds of the C library's).
#pragma once

#include <string>
#include <vector>

namespace fvg {
namespace expr {

// operations of a postfix program; arguments: kConst the constant's index, kVar the variable (0 x, 1 y, 2 z, 3 t),
// kTable the offset of a time table in the pool (n, then n times, then n values), kEnd nothing
enum OpCode : int {
    kEnd = 0, kConst, kVar, kTable,
    // one operand
    kNeg, kNot, kNotNot, kNegNot, kNegNotNot,
    kAbs, kAcos, kAsin, kAtan, kCeil, kCos, kCosh, kExp, kFac, kFloor, kLn, kLog10, kSin, kSinh, kSqrt, kTan, kTanh,
    // two operands
    kAdd, kSub, kMul, kDiv, kMod, kPow, kAtan2, kNcr, kNpr,
    kGt, kGe, kLt, kLe, kEq, kNe, kAnd, kOr, kComma,
};
constexpr int kVarX = 0, kVarY = 1, kVarZ = 2, kVarT = 3;
constexpr int kMaxStack = 32;   // the device evaluator's stack; deeper programs are refused when compiled

struct Op {
    int code, arg;
};

inline bool unary(int c) { return c >= kNeg && c <= kTanh; }
inline bool binary(int c) { return c >= kAdd && c <= kComma; }

// The programs of one run: the code of every entry (each ends in kEnd) and their constant pool.
struct Program {
    std::vector<Op> code;
    std::vector<double> pool;
    int depth = 0;   // the deepest stack of any entry

    // The names an expression may use besides x, y, z, t: later entries of the same name replace earlier ones.
    std::vector<std::string> names;
    std::vector<double> values;
    void bind(const std::string& name, double v);

    // Compiles `src` (a number: kept exact, as the reference's Evaluator::compile; otherwise an expression) and returns
    // the entry's first op. Throws std::invalid_argument("<what>: cannot evaluate ...") for a malformed expression.
    int add(const std::string& src, const std::string& what);
    // A boundary time table (read_time_table / table_value, cpp/src/SimulationInternal.hpp:62-111): rows of (t, value),
    // at least two, strictly increasing times, finite values; throws std::invalid_argument otherwise.
    int add_table(const double* rows, int n, const std::string& what);
    // Whether the entry's program reads variable v.
    bool reads(int entry, int v) const;
    // Whether the entry is the constant c and nothing else.
    bool constant(int entry, double* c) const;
    // Evaluates an entry on the host at (x, y, z, t).
    double eval(int entry, double x, double y, double z, double t) const;
};

// Whether a whole string is a number, as the reference's parse_number (strtod over all of it, cpp/src/CaseFile.cpp:164).
bool parse_number(const std::string& s, double& out);

}  // namespace expr
}  // namespace fvg
