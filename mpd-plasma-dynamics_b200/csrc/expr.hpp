// Expression compiler: the arithmetic subset of the exprtk language used by
// the reference's per-field boundary conditions (src/bcs/per_field_bc.cpp:35-182)
// and expression initial condition (src/ics/expression_ic.cpp:48-188),
// compiled on the host into a postfix bytecode that both the host and the
// device interpret (interpreter: eval_code in lf_core.cuh).
//
// Grammar, precedence low to high (left-associative except '^'):
//   expr  := term  (('+'|'-') term)*
//   term  := unary (('*'|'/'|'%') unary)*
//   unary := ('-'|'+') unary | power
//   power := primary ('^' unary)?
//   primary := NUMBER | NAME | NAME '(' expr (',' expr)* ')' | '(' expr ')'
// Functions: sin cos tan asin acos atan atan2 exp log log2 log10 sqrt pow abs
// sign min max (2..8 args) clamp(lo, x, hi).  No constant folding and no
// reassociation: each operator is one IEEE-754 operation in source order, so
// + - * / expressions evaluate bit-identically on host and device.
#pragma once

#include <cstdint>
#include <map>
#include <string>
#include <vector>

#include "expr_ops.h"

namespace mpd {



struct ExprCode {
    std::vector<int32_t> code;    // (arg << 8) | op, terminated by OP_END
    std::vector<double> consts;
    std::vector<int> vars_used;   // symbol indices referenced
    int max_depth = 0;
};

// Compile `src` against the ordered symbol list (OP_VAR operands index into
// it) and named constants (folded into the constant pool as values).
// Returns false and sets `err` on a syntax error or unknown name.
bool CompileExpr(const std::string &src, const std::vector<std::string> &symbols,
                 const std::map<std::string, double> &constants, ExprCode &out,
                 std::string &err);

}  // namespace mpd
