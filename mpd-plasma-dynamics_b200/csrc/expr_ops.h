// Opcodes of the expression bytecode shared by the host compiler (expr.cpp)
// and the host/device interpreter (eval_code in lf_core.cuh).
#pragma once

#include <stdint.h>

namespace mpd {

enum ExprOp : int32_t {
    OP_END = 0,
    OP_CONST,  // push consts[arg]
    OP_VAR,    // push sym[arg]
    OP_NEG,
    OP_ADD,
    OP_SUB,
    OP_MUL,
    OP_DIV,
    OP_MOD,
    OP_POW,
    OP_FN1,    // arg = Fn1 id, unary function
    OP_ATAN2,
    OP_MIN2,
    OP_MAX2,
    OP_CLAMP,  // clamp(lo, x, hi)
};

enum ExprFn1 : int32_t {
    FN_SIN = 0, FN_COS, FN_TAN, FN_ASIN, FN_ACOS, FN_ATAN, FN_EXP, FN_LOG, FN_LOG2,
    FN_LOG10, FN_SQRT, FN_ABS, FN_SIGN
};

constexpr int kExprMaxStack = 16;

}  // namespace mpd
