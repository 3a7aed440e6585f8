// Element-wise expressions over containers (ironArray's iarray_expr_* / iarray_eval,
// src/iarray_expression.c:59-780), evaluated on the GPU.
//
// The reference compiles the expression string to machine code (LLVM) and runs it as a
// Blosc2 prefilter over the output blocks.  Here the string is parsed once on the host into
// a postfix program (operands: bound containers, bound scalars and literals; the arithmetic
// operators + - * / and **, unary minus, and the math functions of the reference's tests,
// with numpy's names as aliases), and one CUDA kernel runs the program for every element of
// the decoded operands, in the expression's data type.  The program travels in the kernel's
// parameters; each thread keeps its evaluation stack in registers / local memory.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <cctype>
#include <string>
#include <vector>

#include "common.cuh"
#include "expr.h"

namespace iab {

// ============================================================================ parser
namespace {
struct Fn {
    const char *name;
    int code;   // F_*
    int arity;
};
const Fn kFns[] = {
    {"abs", F_ABS, 1},     {"absolute", F_ABS, 1}, {"fabs", F_ABS, 1},     {"sqrt", F_SQRT, 1},
    {"exp", F_EXP, 1},     {"expm1", F_EXPM1, 1},  {"log", F_LOG, 1},      {"log10", F_LOG10, 1},
    {"log1p", F_LOG1P, 1}, {"sin", F_SIN, 1},      {"cos", F_COS, 1},      {"tan", F_TAN, 1},
    {"asin", F_ASIN, 1},   {"arcsin", F_ASIN, 1},  {"acos", F_ACOS, 1},    {"arccos", F_ACOS, 1},
    {"atan", F_ATAN, 1},   {"arctan", F_ATAN, 1},  {"sinh", F_SINH, 1},    {"cosh", F_COSH, 1},
    {"tanh", F_TANH, 1},   {"ceil", F_CEIL, 1},    {"floor", F_FLOOR, 1},  {"negative", F_NEG, 1},
    {"atan2", F_ATAN2, 2}, {"arctan2", F_ATAN2, 2}, {"pow", F_POW, 2},     {"power", F_POW, 2},
    {"min", F_MIN, 2},     {"minimum", F_MIN, 2},  {"max", F_MAX, 2},      {"maximum", F_MAX, 2},
    {"fmod", F_FMOD, 2},
};

struct Parser {
    const char *s;
    size_t p = 0;
    const std::vector<std::string> &vars;
    const std::vector<std::pair<std::string, double>> &scalars;
    std::vector<ExprOp> *out;
    std::string err;

    void ws() { while (s[p] && isspace((unsigned char)s[p])) p++; }
    bool eat(const char *t)
    {
        ws();
        const size_t n = strlen(t);
        if (strncmp(s + p, t, n) != 0) return false;
        // "*" must not eat the first half of "**"
        if (n == 1 && t[0] == '*' && s[p + 1] == '*') return false;
        p += n;
        return true;
    }
    void emit(int code, int arg = 0, double v = 0) { out->push_back(ExprOp{code, arg, v}); }
    bool fail(const std::string &m) { if (err.empty()) err = m; return false; }

    bool expr()
    {
        if (!term()) return false;
        for (;;) {
            if (eat("+")) { if (!term()) return false; emit(OP_ADD); }
            else if (eat("-")) { if (!term()) return false; emit(OP_SUB); }
            else return true;
        }
    }
    bool term()
    {
        if (!unary()) return false;
        for (;;) {
            if (eat("*")) { if (!unary()) return false; emit(OP_MUL); }
            else if (eat("/")) { if (!unary()) return false; emit(OP_DIV); }
            else return true;
        }
    }
    bool unary()
    {
        if (eat("-")) { if (!unary()) return false; emit(OP_F1, F_NEG); return true; }
        if (eat("+")) return unary();
        return power();
    }
    bool power()                                   // right-associative, binds tighter than unary minus on its left
    {
        if (!primary()) return false;
        if (eat("**")) { if (!unary()) return false; emit(OP_F2, F_POW); }
        return true;
    }
    bool primary()
    {
        ws();
        if (eat("(")) {
            if (!expr()) return false;
            return eat(")") || fail("missing ')'");
        }
        const char c = s[p];
        if (isdigit((unsigned char)c) || c == '.') {
            char *end = nullptr;
            const double v = strtod(s + p, &end);
            if (end == s + p) return fail("bad number");
            p = (size_t)(end - s);
            emit(OP_CONST, 0, v);
            return true;
        }
        if (isalpha((unsigned char)c) || c == '_') {
            const size_t b = p;
            while (isalnum((unsigned char)s[p]) || s[p] == '_') p++;
            const std::string name(s + b, p - b);
            ws();
            if (s[p] == '(') {
                p++;
                const Fn *f = nullptr;
                for (const Fn &x : kFns)
                    if (name == x.name) f = &x;
                if (!f) return fail("unknown function '" + name + "'");
                for (int a = 0; a < f->arity; a++) {
                    if (a && !eat(",")) return fail("function '" + name + "' takes " + std::to_string(f->arity) + " arguments");
                    if (!expr()) return false;
                }
                if (!eat(")")) return fail("missing ')' after the arguments of '" + name + "'");
                emit(f->arity == 1 ? OP_F1 : OP_F2, f->code);
                return true;
            }
            for (size_t i = 0; i < vars.size(); i++)
                if (vars[i] == name) { emit(OP_VAR, (int)i); return true; }
            for (const auto &sc : scalars)
                if (sc.first == name) { emit(OP_CONST, 0, sc.second); return true; }
            if (name == "pi") { emit(OP_CONST, 0, 3.14159265358979323846); return true; }
            if (name == "e") { emit(OP_CONST, 0, 2.71828182845904523536); return true; }
            return fail("unbound variable '" + name + "'");
        }
        return fail(std::string("unexpected character '") + (c ? c : '?') + "'");
    }
};
}  // namespace

bool expr_compile(const std::string &text, const std::vector<std::string> &vars,
                  const std::vector<std::pair<std::string, double>> &scalars, std::vector<ExprOp> *prog,
                  std::string *err)
{
    prog->clear();
    Parser ps{text.c_str(), 0, vars, scalars, prog, {}};
    bool ok = ps.expr();
    ps.ws();
    if (ok && text[ps.p]) ok = ps.fail("trailing characters");
    if (ok && (int)prog->size() > EXPR_MAX_OPS) ok = ps.fail("expression too long");
    // stack depth
    int sp = 0, mx = 0;
    for (const ExprOp &o : *prog) {
        if (o.code == OP_VAR || o.code == OP_CONST) sp++;
        else if (o.code != OP_F1) sp--;
        mx = std::max(mx, sp);
    }
    if (ok && mx > EXPR_MAX_STACK) ok = ps.fail("expression nests too deeply");
    if (!ok && err) *err = ps.err;
    return ok;
}

// ============================================================================ evaluation
template <typename T>
__device__ __forceinline__ T f1(int f, T x)
{
    switch (f) {
    case F_ABS: return fabs(x);
    case F_SQRT: return sqrt(x);
    case F_EXP: return exp(x);
    case F_EXPM1: return expm1(x);
    case F_LOG: return log(x);
    case F_LOG10: return log10(x);
    case F_LOG1P: return log1p(x);
    case F_SIN: return sin(x);
    case F_COS: return cos(x);
    case F_TAN: return tan(x);
    case F_ASIN: return asin(x);
    case F_ACOS: return acos(x);
    case F_ATAN: return atan(x);
    case F_SINH: return sinh(x);
    case F_COSH: return cosh(x);
    case F_TANH: return tanh(x);
    case F_CEIL: return ceil(x);
    case F_FLOOR: return floor(x);
    case F_NEG: return -x;
    default: return x;
    }
}

template <typename T>
__device__ __forceinline__ T f2(int f, T a, T b)
{
    switch (f) {
    case F_ATAN2: return atan2(a, b);
    case F_POW: return pow(a, b);
    case F_MIN: return a < b ? a : (b < a ? b : (a != a ? a : b));   // NaN wins, like numpy's minimum
    case F_MAX: return a > b ? a : (b > a ? b : (a != a ? a : b));
    case F_FMOD: return fmod(a, b);
    default: return a;
    }
}

template <typename T>
__global__ void __launch_bounds__(256) k_expr(int64_t rows, int64_t cols, ExprArgs args, T *__restrict__ out, int64_t ldo)
{
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < rows * cols;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = e / cols, j = e - i * cols;
        T st[EXPR_MAX_STACK];
        int sp = 0;
        for (int k = 0; k < args.nops; k++) {
            const ExprOp o = args.ops[k];
            switch (o.code) {
            case OP_VAR: st[sp++] = reinterpret_cast<const T *>(args.in[o.arg])[i * args.ld[o.arg] + j]; break;
            case OP_CONST: st[sp++] = (T)o.value; break;
            case OP_ADD: sp--; st[sp - 1] = st[sp - 1] + st[sp]; break;
            case OP_SUB: sp--; st[sp - 1] = st[sp - 1] - st[sp]; break;
            case OP_MUL: sp--; st[sp - 1] = st[sp - 1] * st[sp]; break;
            case OP_DIV: sp--; st[sp - 1] = st[sp - 1] / st[sp]; break;
            case OP_F1: st[sp - 1] = f1<T>(o.arg, st[sp - 1]); break;
            case OP_F2: sp--; st[sp - 1] = f2<T>(o.arg, st[sp - 1], st[sp]); break;
            default: break;
            }
        }
        out[i * ldo + j] = sp > 0 ? st[sp - 1] : (T)0;
    }
}

void expr_eval(int itemsize, int64_t rows, int64_t cols, const ExprArgs &args, void *out, int64_t ldo, cudaStream_t st)
{
    if (rows * cols == 0) return;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const unsigned grid = (unsigned)std::max<int64_t>(1, std::min<int64_t>((rows * cols + 255) / 256, (int64_t)sms * 16));
    if (itemsize == 8)
        IAB_TIMED("k_expr", st, k_expr<double><<<grid, 256, 0, st>>>(rows, cols, args, (double *)out, ldo));
    else
        IAB_TIMED("k_expr", st, k_expr<float><<<grid, 256, 0, st>>>(rows, cols, args, (float *)out, ldo));
}

}  // namespace iab
