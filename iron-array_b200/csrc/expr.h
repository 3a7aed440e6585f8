// Element-wise expression programs (expr.cu): postfix programs compiled on the host from an
// expression string and evaluated by one CUDA kernel over dense operands.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <utility>
#include <vector>

namespace iab {

enum ExprCode : int32_t { OP_VAR = 0, OP_CONST, OP_ADD, OP_SUB, OP_MUL, OP_DIV, OP_F1, OP_F2 };
enum ExprFn : int32_t {
    F_ABS = 0, F_SQRT, F_EXP, F_EXPM1, F_LOG, F_LOG10, F_LOG1P, F_SIN, F_COS, F_TAN, F_ASIN, F_ACOS, F_ATAN,
    F_SINH, F_COSH, F_TANH, F_CEIL, F_FLOOR, F_NEG,
    F_ATAN2, F_POW, F_MIN, F_MAX, F_FMOD
};

struct ExprOp {
    int32_t code;   // ExprCode
    int32_t arg;    // OP_VAR: operand index; OP_F1 / OP_F2: ExprFn
    double value;   // OP_CONST
};

constexpr int EXPR_MAX_OPS = 96;
constexpr int EXPR_MAX_STACK = 16;
constexpr int EXPR_MAX_OPERANDS = 16;

// Kernel arguments: the program and the dense operands (row-major, leading dimensions in
// items), passed by value.
struct ExprArgs {
    const void *in[EXPR_MAX_OPERANDS];
    int64_t ld[EXPR_MAX_OPERANDS];
    int nops;
    ExprOp ops[EXPR_MAX_OPS];
};

// Parses `text` over the operand names `vars` (OP_VAR i refers to vars[i]) and the bound
// scalars; false with a message in *err on a syntax error, an unknown name or function, or a
// program beyond EXPR_MAX_OPS / EXPR_MAX_STACK.
bool expr_compile(const std::string &text, const std::vector<std::string> &vars,
                  const std::vector<std::pair<std::string, double>> &scalars, std::vector<ExprOp> *prog,
                  std::string *err);

// out[i, j] = program(operands[i, j]) for a rows x cols output, float64 (itemsize 8) or
// float32 (4).
void expr_eval(int itemsize, int64_t rows, int64_t cols, const ExprArgs &args, void *out, int64_t ldo, cudaStream_t st);

}  // namespace iab
