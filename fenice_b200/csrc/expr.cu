// The compiler of case-file expressions (expr.h) and the host entry point fvg_expr_eval.
//
// The grammar is TinyExpr's with TE_POW_FROM_RIGHT, as the reference builds it (cpp/third_party/tinyexpr/tinyexpr.c:
// next_token 334-443, base 463-560, power 563-616, factor 619-676, term .. list 717-865):
//   list     = expr {"," expr}                         (the value of the last)
//   expr     = and {"||" and};  and = eq {"&&" eq};  eq = rel {("==" | "!=") rel};  rel = sum {("<" | "<=" | ">" | ">=") sum}
//   sum      = term {("+" | "-") term};  term = factor {("*" | "/" | "%") factor}
//   factor   = power {"^" power}                       (right to left; a unary operator written before the first power
//                                                       applies to the whole chain, one before a later power to the rest)
//   power    = {"+" | "-"} {"+" | "-" | "!"} base
//   base     = number | name | function0 ["(" ")"] | function1 power | function2 "(" expr "," expr ")" | "(" list ")"
// Numbers are read TinyExpr's way (digits accumulated in a double, then scaled by pow(10, exponent); hex 0x...), names
// start with a letter and go on with letters, digits and '_'. A name is x, y, z, t, a bound parameter, or a function:
// abs acos asin atan atan2 ceil cos cosh e exp fac floor ln log (base 10) log10 ncr npr pi pow sin sinh sqrt tan tanh.
// Every operation whose operands are known without x, y, z, t is folded on the host, as TinyExpr's optimize folds the
// constant parts (its parameters are fixed for the run, so folding them too gives the values TinyExpr computes).
#include <cctype>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/fenice_gpu.h"
#include "expr.cuh"

namespace fvg {
namespace expr {
namespace {

enum Tok { TNull, TEnd, TNum, TName, TFun0, TFun1, TFun2, TInfix, TOpen, TClose, TSep, TError };

struct Builtin {
    const char* name;
    int arity;
    int op;        // the operation of a function of one or two arguments
    double value;  // a function of none
};
const Builtin kBuiltins[] = {
    {"abs", 1, kAbs, 0}, {"acos", 1, kAcos, 0}, {"asin", 1, kAsin, 0}, {"atan", 1, kAtan, 0}, {"atan2", 2, kAtan2, 0},
    {"ceil", 1, kCeil, 0}, {"cos", 1, kCos, 0}, {"cosh", 1, kCosh, 0}, {"e", 0, 0, 2.71828182845904523536}, {"exp", 1, kExp, 0},
    {"fac", 1, kFac, 0}, {"floor", 1, kFloor, 0}, {"ln", 1, kLn, 0}, {"log", 1, kLog10, 0}, {"log10", 1, kLog10, 0},
    {"ncr", 2, kNcr, 0}, {"npr", 2, kNpr, 0}, {"pi", 0, 0, 3.14159265358979323846}, {"pow", 2, kPow, 0}, {"sin", 1, kSin, 0},
    {"sinh", 1, kSinh, 0}, {"sqrt", 1, kSqrt, 0}, {"tan", 1, kTan, 0}, {"tanh", 1, kTanh, 0},
};

// A node of the parse tree: a constant, a variable (op = which) or an operation (op) of one (a) or two (a, b) operands.
struct Node {
    int kind;   // 0 constant, 1 variable, 2 operation
    int op;
    double value;
    int a, b;
};

struct Failed {
    size_t at;
};

class Parser {
public:
    Parser(const std::string& src, const Program& prog) : start_(src.c_str()), p_(src.c_str()), prog_(prog) {}

    int parse() {
        next_token();
        const int r = list();
        if (type_ != TEnd) fail();
        return r;
    }
    std::vector<Node> nodes;

private:
    const char* start_;
    const char* p_;
    const Program& prog_;
    int type_ = TNull, fn_ = 0, var_ = 0;
    double value_ = 0.0;
    bool applied_unary_ = false;
    int depth_ = 0;

    [[noreturn]] void fail() { throw Failed{(size_t)(p_ - start_) > 0 ? (size_t)(p_ - start_) : 1}; }

    int node(int kind, int op, double value, int a = -1, int b = -1) {
        nodes.push_back({kind, op, value, a, b});
        return (int)nodes.size() - 1;
    }

    double number() {
        const char* p = p_;
        double value = 0.0;
        if (p[0] == '0' && (p[1] == 'x' || p[1] == 'X') && isxdigit((unsigned char)p[2])) {
            p += 2;
            while (isxdigit((unsigned char)p[0])) {
                const char c = p[0];
                const int d = isdigit((unsigned char)c) ? c - '0' : (c >= 'a' ? c - 'a' + 10 : c - 'A' + 10);
                value = value * 16.0 + d;
                ++p;
            }
        } else {
            int exponent = 0, digits = 0;
            while (isdigit((unsigned char)p[0])) {
                value = value * 10.0 + (p[0] - '0');
                ++p;
                ++digits;
            }
            if (p[0] == '.') {
                ++p;
                while (isdigit((unsigned char)p[0])) {
                    value = value * 10.0 + (p[0] - '0');
                    ++p;
                    ++digits;
                    --exponent;
                }
            }
            if (digits == 0) {
                type_ = TError;
                return 0.0;
            }
            if (p[0] == 'e' || p[0] == 'E') {   // an exponent only when digits follow ("1e" is 1 then the name e)
                const char* ep = p + 1;
                int esign = 1, e = 0;
                if (ep[0] == '+') ++ep;
                else if (ep[0] == '-') {
                    esign = -1;
                    ++ep;
                }
                if (isdigit((unsigned char)ep[0])) {
                    while (isdigit((unsigned char)ep[0])) {
                        if (e < 100000000) e = e * 10 + (ep[0] - '0');
                        ++ep;
                    }
                    exponent += esign * e;
                    p = ep;
                }
            }
            if (exponent && value != 0.0) value *= std::pow(10.0, exponent);
        }
        type_ = TNum;
        p_ = p;
        return value;
    }

    void next_token() {
        type_ = TNull;
        do {
            if (!*p_) {
                type_ = TEnd;
                return;
            }
            if ((p_[0] >= '0' && p_[0] <= '9') || p_[0] == '.') {
                value_ = number();
            } else if (isalpha((unsigned char)p_[0])) {
                const char* s = p_;
                while (isalpha((unsigned char)p_[0]) || isdigit((unsigned char)p_[0]) || p_[0] == '_') ++p_;
                const std::string name(s, p_ - s);
                if (name == "x" || name == "y" || name == "z" || name == "t") {
                    type_ = TName;
                    var_ = name == "x" ? kVarX : name == "y" ? kVarY : name == "z" ? kVarZ : kVarT;
                    continue;
                }
                int bound = -1;
                for (size_t i = 0; i < prog_.names.size(); ++i)
                    if (prog_.names[i] == name) bound = (int)i;
                if (bound >= 0) {   // a parameter: a constant of the run
                    type_ = TNum;
                    value_ = prog_.values[bound];
                    continue;
                }
                type_ = TError;
                for (const Builtin& b : kBuiltins)
                    if (name == b.name) {
                        type_ = b.arity == 0 ? TFun0 : b.arity == 1 ? TFun1 : TFun2;
                        fn_ = b.op;
                        value_ = b.value;
                    }
            } else {
                const char c = *p_++;
                switch (c) {
                case '+': type_ = TInfix; fn_ = kAdd; break;
                case '-': type_ = TInfix; fn_ = kSub; break;
                case '*': type_ = TInfix; fn_ = kMul; break;
                case '/': type_ = TInfix; fn_ = kDiv; break;
                case '^': type_ = TInfix; fn_ = kPow; break;
                case '%': type_ = TInfix; fn_ = kMod; break;
                case '!':
                    if (*p_ == '=') {
                        ++p_;
                        type_ = TInfix;
                        fn_ = kNe;
                    } else {
                        type_ = TInfix;
                        fn_ = kNot;
                    }
                    break;
                case '=':
                    if (*p_ == '=') {
                        ++p_;
                        type_ = TInfix;
                        fn_ = kEq;
                    } else type_ = TError;
                    break;
                case '<':
                    type_ = TInfix;
                    fn_ = kLt;
                    if (*p_ == '=') {
                        ++p_;
                        fn_ = kLe;
                    }
                    break;
                case '>':
                    type_ = TInfix;
                    fn_ = kGt;
                    if (*p_ == '=') {
                        ++p_;
                        fn_ = kGe;
                    }
                    break;
                case '&':
                    if (*p_ == '&') {
                        ++p_;
                        type_ = TInfix;
                        fn_ = kAnd;
                    } else type_ = TError;
                    break;
                case '|':
                    if (*p_ == '|') {
                        ++p_;
                        type_ = TInfix;
                        fn_ = kOr;
                    } else type_ = TError;
                    break;
                case '(': type_ = TOpen; break;
                case ')': type_ = TClose; break;
                case ',': type_ = TSep; break;
                case ' ': case '\t': case '\n': case '\r': break;
                default: type_ = TError; break;
                }
            }
        } while (type_ == TNull);
        if (type_ == TError) fail();
    }

    int base() {
        if (depth_ >= 512) fail();
        ++depth_;
        int r = -1;
        switch (type_) {
        case TNum:
            r = node(0, 0, value_);
            next_token();
            break;
        case TName:
            r = node(1, var_, 0.0);
            next_token();
            break;
        case TFun0:
            r = node(0, 0, value_);
            next_token();
            if (type_ == TOpen) {
                next_token();
                if (type_ != TClose) fail();
                next_token();
            }
            break;
        case TFun1: {
            const int op = fn_;
            next_token();
            const int a = power();
            r = node(2, op, 0.0, a);
            break;
        }
        case TFun2: {
            const int op = fn_;
            next_token();
            if (type_ != TOpen) fail();
            next_token();
            const int a = expr();
            if (type_ != TSep) fail();
            next_token();
            const int b = expr();
            if (type_ != TClose) fail();
            next_token();
            r = node(2, op, 0.0, a, b);
            break;
        }
        case TOpen:
            next_token();
            r = list();
            if (type_ != TClose) fail();
            next_token();
            break;
        default: fail();
        }
        --depth_;
        return r;
    }

    int power() {
        int sign = 1;
        while (type_ == TInfix && (fn_ == kAdd || fn_ == kSub)) {
            if (fn_ == kSub) sign = -sign;
            next_token();
        }
        int logical = 0;
        while (type_ == TInfix && (fn_ == kAdd || fn_ == kSub || fn_ == kNot)) {
            if (fn_ == kNot) logical = logical == 0 ? -1 : -logical;
            next_token();
        }
        int r;
        if (sign == 1) {
            r = base();
            if (logical != 0) r = node(2, logical == -1 ? kNot : kNotNot, 0.0, r);
        } else {
            r = base();
            r = node(2, logical == 0 ? kNeg : logical == -1 ? kNegNot : kNegNotNot, 0.0, r);
        }
        applied_unary_ = sign != 1 || logical != 0;
        return r;
    }

    int& child(int n, int which) { return which == 0 ? nodes[n].a : nodes[n].b; }

    int factor() {
        int r = power();
        int left = -1;
        if (applied_unary_) {   // the unary operator in front applies to the whole chain of powers
            left = nodes[r].op;
            r = nodes[r].a;
        }
        int slot = -1, which = 0;   // where the next exponent goes
        while (type_ == TInfix && fn_ == kPow) {
            next_token();
            const int p = power();
            const bool p_unary = applied_unary_;
            if (slot >= 0) {
                const int ins = node(2, kPow, 0.0, child(slot, which), p);
                child(slot, which) = ins;
                slot = p_unary ? p : ins;
                which = p_unary ? 0 : 1;
            } else {
                r = node(2, kPow, 0.0, r, p);
                slot = p_unary ? p : r;
                which = p_unary ? 0 : 1;
            }
        }
        if (left >= 0) r = node(2, left, 0.0, r);
        return r;
    }

    template <typename Next> int chain(Next next, std::initializer_list<int> ops) {
        int r = next();
        for (;;) {
            bool match = false;
            for (int o : ops) match |= type_ == TInfix && fn_ == o;
            if (!match) return r;
            const int op = fn_;
            next_token();
            const int b = next();
            r = node(2, op, 0.0, r, b);
        }
    }
    int term() { return chain([&] { return factor(); }, {kMul, kDiv, kMod}); }
    int sum() { return chain([&] { return term(); }, {kAdd, kSub}); }
    int rel() { return chain([&] { return sum(); }, {kGt, kGe, kLt, kLe}); }
    int eq() { return chain([&] { return rel(); }, {kEq, kNe}); }
    int conj() { return chain([&] { return eq(); }, {kAnd}); }
    int expr() { return chain([&] { return conj(); }, {kOr}); }
    int list() {
        int r = expr();
        while (type_ == TSep) {
            next_token();
            const int b = expr();
            r = node(2, kComma, 0.0, r, b);
        }
        return r;
    }
};

// folds the operations whose operands are constants (host functions: the C library's)
void fold(std::vector<Node>& n, int i) {
    if (n[i].kind != 2) return;
    fold(n, n[i].a);
    if (n[i].b >= 0) fold(n, n[i].b);
    const bool known = n[n[i].a].kind == 0 && (n[i].b < 0 || n[n[i].b].kind == 0);
    if (!known) return;
    n[i].value = n[i].b < 0 ? apply1(n[i].op, n[n[i].a].value) : apply2(n[i].op, n[n[i].a].value, n[n[i].b].value);
    n[i].kind = 0;
}

// postfix code of node i; returns the stack depth it needs
int emit(const std::vector<Node>& n, int i, Program& p) {
    const Node& d = n[i];
    if (d.kind == 0) {
        p.pool.push_back(d.value);
        p.code.push_back({kConst, (int)p.pool.size() - 1});
        return 1;
    }
    if (d.kind == 1) {
        p.code.push_back({kVar, d.op});
        return 1;
    }
    const int da = emit(n, d.a, p);
    int need = da;
    if (d.b >= 0) {
        const int db = emit(n, d.b, p);
        need = da > 1 + db ? da : 1 + db;
    }
    p.code.push_back({d.op, 0});
    return need;
}

}  // namespace

bool parse_number(const std::string& s, double& out) {
    if (s.empty()) return false;
    char* end = nullptr;
    out = std::strtod(s.c_str(), &end);
    return end && *end == '\0';
}

void Program::bind(const std::string& name, double v) {
    for (size_t i = 0; i < names.size(); ++i)
        if (names[i] == name) {
            values[i] = v;
            return;
        }
    names.push_back(name);
    values.push_back(v);
}

int Program::add(const std::string& src, const std::string& what) {
    const int entry = (int)code.size();
    double c = 0.0;
    if (parse_number(src, c)) {
        pool.push_back(c);
        code.push_back({kConst, (int)pool.size() - 1});
        code.push_back({kEnd, 0});
        if (depth < 1) depth = 1;
        return entry;
    }
    Parser parser(src, *this);
    int root = -1;
    try {
        root = parser.parse();
    } catch (const Failed& f) {
        throw std::invalid_argument(what + ": cannot evaluate \"" + src + "\" (error at character " + std::to_string(f.at) + ")");
    }
    fold(parser.nodes, root);
    const int need = emit(parser.nodes, root, *this);
    code.push_back({kEnd, 0});
    if (need > kMaxStack) {
        code.resize(entry);
        throw std::invalid_argument(what + ": \"" + src + "\" nests deeper than the device evaluator's stack of " + std::to_string(kMaxStack));
    }
    if (need > depth) depth = need;
    return entry;
}

int Program::add_table(const double* rows, int n, const std::string& what) {
    if (n < 2) throw std::invalid_argument(what + " must contain at least two (t,value) rows");
    for (int i = 0; i < n; ++i) {
        if (!std::isfinite(rows[2 * i]) || !std::isfinite(rows[2 * i + 1])) throw std::invalid_argument(what + ": values must be finite");
        if (i > 0 && !(rows[2 * i] > rows[2 * i - 2])) throw std::invalid_argument(what + ": times must be strictly increasing");
    }
    const int off = (int)pool.size();
    pool.push_back((double)n);
    for (int i = 0; i < n; ++i) pool.push_back(rows[2 * i]);
    for (int i = 0; i < n; ++i) pool.push_back(rows[2 * i + 1]);
    const int entry = (int)code.size();
    code.push_back({kVar, kVarT});
    code.push_back({kTable, off});
    code.push_back({kEnd, 0});
    if (depth < 1) depth = 1;
    return entry;
}

bool Program::reads(int entry, int v) const {
    for (int pc = entry; code[pc].code != kEnd; ++pc)
        if (code[pc].code == kVar && code[pc].arg == v) return true;
    return false;
}

bool Program::constant(int entry, double* c) const {
    if (code[entry].code == kConst && code[entry + 1].code == kEnd) {
        if (c) *c = pool[code[entry].arg];
        return true;
    }
    return false;
}

double Program::eval(int entry, double x, double y, double z, double t) const { return run(code.data(), pool.data(), entry, x, y, z, t); }

}  // namespace expr
}  // namespace fvg

extern "C" {

int fvg_expr_eval(const char* src, const char* const* names, const double* values, int nnames, const double* x, const double* y,
                  const double* z, double t, size_t n, double* out, char* err, size_t errlen) {
    try {
        if (!src || (n && !out) || (nnames && (!names || !values))) throw std::invalid_argument("fvg_expr_eval: null argument");
        fvg::expr::Program p;
        for (int i = 0; i < nnames; ++i) p.bind(names[i] ? names[i] : "", values[i]);
        const int e = p.add(src, "expression");
        for (size_t i = 0; i < n; ++i) out[i] = p.eval(e, x ? x[i] : 0.0, y ? y[i] : 0.0, z ? z[i] : 0.0, t);
        return FVG_OK;
    } catch (const std::exception& ex) {
        if (err && errlen) {
            std::strncpy(err, ex.what(), errlen - 1);
            err[errlen - 1] = '\0';
        }
        return FVG_ERR_CONFIG;
    }
}

}  // extern "C"
