/*
 * Oracle expression evaluator — TEST INFRASTRUCTURE ONLY.
 *
 * A small tree-walking evaluator for the arithmetic subset of the exprtk
 * language that the reference's boundary conditions and initial conditions
 * use (exprtk 0.0.2, pinned at cmake/Dependencies.cmake:6 of the reference,
 * not vendored and not installed here).  Call sites it stands in for:
 *   src/bcs/per_field_bc.cpp:35-182   (PerFieldBC::ExprImpl)
 *   src/ics/expression_ic.cpp:48-188  (ExpressionIC::Impl)
 *
 * Grammar (precedence low to high, all binary operators left-associative
 * except '^'):
 *     expr   := term  (('+' | '-') term)*
 *     term   := unary (('*' | '/' | '%') unary)*
 *     unary  := ('-' | '+') unary | power
 *     power  := primary ('^' unary)?
 *     primary:= NUMBER | NAME | NAME '(' expr (',' expr)* ')' | '(' expr ')'
 * Functions: sin cos tan asin acos atan atan2 exp log log2 log10 sqrt pow abs
 * sign min max (variadic, >= 2 args) clamp(lo, x, hi).
 * Numbers are converted with strtod (correctly rounded).  No constant folding
 * and no reassociation: every operator is one IEEE-754 double operation in
 * source order.
 *
 * Only tests/, the oracle harness and the CPU-baseline leg of bench.py use
 * this file; the product path has its own compiler (bytecode, device
 * interpreter).
 */
#ifndef MPD_ORACLE_EXPR_EVAL_H
#define MPD_ORACLE_EXPR_EVAL_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct oe_symtab oe_symtab;
typedef struct oe_expr oe_expr;

oe_symtab *oe_symtab_new(void);
void oe_symtab_free(oe_symtab *st);
/* Register a variable read through `ref` at evaluation time. 0 = ok, -1 = duplicate/bad name. */
int oe_symtab_add_var(oe_symtab *st, const char *name, double *ref);
/* Register a constant; the value is copied. 0 = ok, -1 = duplicate/bad name. */
int oe_symtab_add_const(oe_symtab *st, const char *name, double value);
int oe_symtab_has(const oe_symtab *st, const char *name);

/* Compile `src` against `st`.  Returns NULL and writes a diagnostic into
 * err (if non-NULL) on failure.  The symbol table must outlive the expr. */
oe_expr *oe_compile(const char *src, const oe_symtab *st, char *err, int errlen);
double oe_eval(const oe_expr *e);
void oe_free(oe_expr *e);

#ifdef __cplusplus
}
#endif
#endif
