/*
 * Oracle expression evaluator — TEST INFRASTRUCTURE ONLY (see expr_eval.h).
 * Recursive-descent parser building an AST that is walked at evaluation time.
 */
#include "expr_eval.h"

#include <ctype.h>
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define OE_MAX_SYMS 96
#define OE_NAME_LEN 32

struct oe_symtab {
    int n;
    char name[OE_MAX_SYMS][OE_NAME_LEN];
    double *ref[OE_MAX_SYMS];
    double cval[OE_MAX_SYMS];
    int is_const[OE_MAX_SYMS];
};

enum { N_NUM, N_VAR, N_NEG, N_ADD, N_SUB, N_MUL, N_DIV, N_MOD, N_POW, N_FN };
enum { F_SIN, F_COS, F_TAN, F_ASIN, F_ACOS, F_ATAN, F_ATAN2, F_EXP, F_LOG, F_LOG2,
       F_LOG10, F_SQRT, F_POW, F_ABS, F_SIGN, F_MIN, F_MAX, F_CLAMP };

typedef struct node {
    int kind;
    double num;
    const double *var;
    int fn;
    int nargs;
    struct node *a[8];
} node;

struct oe_expr {
    node *root;
};

static const struct { const char *name; int id; int min_args; int max_args; } k_funcs[] = {
    {"sin", F_SIN, 1, 1},   {"cos", F_COS, 1, 1},     {"tan", F_TAN, 1, 1},
    {"asin", F_ASIN, 1, 1}, {"acos", F_ACOS, 1, 1},   {"atan", F_ATAN, 1, 1},
    {"atan2", F_ATAN2, 2, 2}, {"exp", F_EXP, 1, 1},   {"log", F_LOG, 1, 1},
    {"log2", F_LOG2, 1, 1}, {"log10", F_LOG10, 1, 1}, {"sqrt", F_SQRT, 1, 1},
    {"pow", F_POW, 2, 2},   {"abs", F_ABS, 1, 1},     {"sign", F_SIGN, 1, 1},
    {"min", F_MIN, 2, 8},   {"max", F_MAX, 2, 8},     {"clamp", F_CLAMP, 3, 3},
};

oe_symtab *oe_symtab_new(void) { return (oe_symtab *)calloc(1, sizeof(oe_symtab)); }
void oe_symtab_free(oe_symtab *st) { free(st); }

static int find_sym(const oe_symtab *st, const char *name) {
    for (int i = 0; i < st->n; ++i)
        if (strcmp(st->name[i], name) == 0) return i;
    return -1;
}

int oe_symtab_has(const oe_symtab *st, const char *name) { return find_sym(st, name) >= 0; }

static int add_sym(oe_symtab *st, const char *name, double *ref, double v, int c) {
    if (!name || !*name || strlen(name) >= OE_NAME_LEN || st->n >= OE_MAX_SYMS) return -1;
    if (find_sym(st, name) >= 0) return -1;
    for (size_t i = 0; i < sizeof(k_funcs) / sizeof(k_funcs[0]); ++i)
        if (strcmp(k_funcs[i].name, name) == 0) return -1;
    strcpy(st->name[st->n], name);
    st->ref[st->n] = ref;
    st->cval[st->n] = v;
    st->is_const[st->n] = c;
    st->n++;
    return 0;
}

int oe_symtab_add_var(oe_symtab *st, const char *name, double *ref) {
    return add_sym(st, name, ref, 0.0, 0);
}
int oe_symtab_add_const(oe_symtab *st, const char *name, double value) {
    return add_sym(st, name, NULL, value, 1);
}

/* ------------------------------------------------------------------ parser */
typedef struct {
    const char *s;
    int pos;
    const oe_symtab *st;
    char *err;
    int errlen;
    int failed;
} parser;

static void perr(parser *p, const char *fmt, ...) {
    if (p->failed) return;
    p->failed = 1;
    if (p->err && p->errlen > 0) {
        va_list ap;
        va_start(ap, fmt);
        int k = snprintf(p->err, (size_t)p->errlen, "at %d: ", p->pos);
        if (k < p->errlen) vsnprintf(p->err + k, (size_t)(p->errlen - k), fmt, ap);
        va_end(ap);
    }
}

static void skip_ws(parser *p) {
    while (p->s[p->pos] && isspace((unsigned char)p->s[p->pos])) p->pos++;
}

static node *mk(int kind) {
    node *n = (node *)calloc(1, sizeof(node));
    n->kind = kind;
    return n;
}

static void free_node(node *n) {
    if (!n) return;
    for (int i = 0; i < 8; ++i) free_node(n->a[i]);
    free(n);
}

static node *parse_expr(parser *p);
static node *parse_unary(parser *p);

static node *parse_primary(parser *p) {
    skip_ws(p);
    char c = p->s[p->pos];
    if (c == '(') {
        p->pos++;
        node *e = parse_expr(p);
        skip_ws(p);
        if (p->s[p->pos] != ')') { perr(p, "expected ')'"); free_node(e); return NULL; }
        p->pos++;
        return e;
    }
    if (isdigit((unsigned char)c) || (c == '.' && isdigit((unsigned char)p->s[p->pos + 1]))) {
        const char *start = p->s + p->pos;
        int k = p->pos;
        while (isdigit((unsigned char)p->s[k])) k++;
        if (p->s[k] == '.') { k++; while (isdigit((unsigned char)p->s[k])) k++; }
        if (p->s[k] == 'e' || p->s[k] == 'E') {
            int k2 = k + 1;
            if (p->s[k2] == '+' || p->s[k2] == '-') k2++;
            if (isdigit((unsigned char)p->s[k2])) {
                k = k2;
                while (isdigit((unsigned char)p->s[k])) k++;
            }
        }
        char buf[64];
        int len = k - p->pos;
        if (len >= (int)sizeof(buf)) { perr(p, "number too long"); return NULL; }
        memcpy(buf, start, (size_t)len);
        buf[len] = 0;
        node *n = mk(N_NUM);
        n->num = strtod(buf, NULL);
        p->pos = k;
        return n;
    }
    if (isalpha((unsigned char)c) || c == '_') {
        char name[OE_NAME_LEN];
        int len = 0;
        while (isalnum((unsigned char)p->s[p->pos]) || p->s[p->pos] == '_') {
            if (len < OE_NAME_LEN - 1) name[len++] = p->s[p->pos];
            p->pos++;
        }
        name[len] = 0;
        skip_ws(p);
        if (p->s[p->pos] == '(') {
            int fi = -1;
            for (size_t i = 0; i < sizeof(k_funcs) / sizeof(k_funcs[0]); ++i)
                if (strcmp(k_funcs[i].name, name) == 0) fi = (int)i;
            if (fi < 0) { perr(p, "unknown function '%s'", name); return NULL; }
            p->pos++;
            node *n = mk(N_FN);
            n->fn = k_funcs[fi].id;
            for (;;) {
                if (n->nargs >= 8) { perr(p, "too many arguments"); free_node(n); return NULL; }
                n->a[n->nargs] = parse_expr(p);
                if (!n->a[n->nargs]) { free_node(n); return NULL; }
                n->nargs++;
                skip_ws(p);
                if (p->s[p->pos] == ',') { p->pos++; continue; }
                if (p->s[p->pos] == ')') { p->pos++; break; }
                perr(p, "expected ',' or ')'");
                free_node(n);
                return NULL;
            }
            if (n->nargs < k_funcs[fi].min_args || n->nargs > k_funcs[fi].max_args) {
                perr(p, "wrong number of arguments to '%s'", name);
                free_node(n);
                return NULL;
            }
            return n;
        }
        int si = find_sym(p->st, name);
        if (si < 0) { perr(p, "undefined symbol '%s'", name); return NULL; }
        if (p->st->is_const[si]) {
            node *n = mk(N_NUM);
            n->num = p->st->cval[si];
            return n;
        }
        node *n = mk(N_VAR);
        n->var = p->st->ref[si];
        return n;
    }
    if (c == 0) perr(p, "unexpected end of expression");
    else perr(p, "unexpected character '%c'", c);
    return NULL;
}

static node *parse_power(parser *p) {
    node *b = parse_primary(p);
    if (!b) return NULL;
    skip_ws(p);
    if (p->s[p->pos] == '^') {
        p->pos++;
        node *e = parse_unary(p);
        if (!e) { free_node(b); return NULL; }
        node *n = mk(N_POW);
        n->a[0] = b;
        n->a[1] = e;
        return n;
    }
    return b;
}

static node *parse_unary(parser *p) {
    skip_ws(p);
    if (p->s[p->pos] == '-') {
        p->pos++;
        node *x = parse_unary(p);
        if (!x) return NULL;
        node *n = mk(N_NEG);
        n->a[0] = x;
        return n;
    }
    if (p->s[p->pos] == '+') {
        p->pos++;
        return parse_unary(p);
    }
    return parse_power(p);
}

static node *parse_term(parser *p) {
    node *l = parse_unary(p);
    while (l) {
        skip_ws(p);
        char c = p->s[p->pos];
        int kind = c == '*' ? N_MUL : c == '/' ? N_DIV : c == '%' ? N_MOD : -1;
        if (kind < 0) break;
        p->pos++;
        node *r = parse_unary(p);
        if (!r) { free_node(l); return NULL; }
        node *n = mk(kind);
        n->a[0] = l;
        n->a[1] = r;
        l = n;
    }
    return l;
}

static node *parse_expr(parser *p) {
    node *l = parse_term(p);
    while (l) {
        skip_ws(p);
        char c = p->s[p->pos];
        int kind = c == '+' ? N_ADD : c == '-' ? N_SUB : -1;
        if (kind < 0) break;
        p->pos++;
        node *r = parse_term(p);
        if (!r) { free_node(l); return NULL; }
        node *n = mk(kind);
        n->a[0] = l;
        n->a[1] = r;
        l = n;
    }
    return l;
}

oe_expr *oe_compile(const char *src, const oe_symtab *st, char *err, int errlen) {
    parser p = {src ? src : "", 0, st, err, errlen, 0};
    if (err && errlen > 0) err[0] = 0;
    node *root = parse_expr(&p);
    skip_ws(&p);
    if (root && !p.failed && p.s[p.pos] != 0) perr(&p, "trailing input");
    if (p.failed || !root) {
        free_node(root);
        if (!p.failed) perr(&p, "empty expression");
        return NULL;
    }
    oe_expr *e = (oe_expr *)calloc(1, sizeof(oe_expr));
    e->root = root;
    return e;
}

static double ev(const node *n) {
    switch (n->kind) {
        case N_NUM: return n->num;
        case N_VAR: return *n->var;
        case N_NEG: return -ev(n->a[0]);
        case N_ADD: return ev(n->a[0]) + ev(n->a[1]);
        case N_SUB: return ev(n->a[0]) - ev(n->a[1]);
        case N_MUL: return ev(n->a[0]) * ev(n->a[1]);
        case N_DIV: return ev(n->a[0]) / ev(n->a[1]);
        case N_MOD: return fmod(ev(n->a[0]), ev(n->a[1]));
        case N_POW: return pow(ev(n->a[0]), ev(n->a[1]));
        case N_FN: {
            double x = ev(n->a[0]);
            switch (n->fn) {
                case F_SIN: return sin(x);
                case F_COS: return cos(x);
                case F_TAN: return tan(x);
                case F_ASIN: return asin(x);
                case F_ACOS: return acos(x);
                case F_ATAN: return atan(x);
                case F_ATAN2: return atan2(x, ev(n->a[1]));
                case F_EXP: return exp(x);
                case F_LOG: return log(x);
                case F_LOG2: return log2(x);
                case F_LOG10: return log10(x);
                case F_SQRT: return sqrt(x);
                case F_POW: return pow(x, ev(n->a[1]));
                case F_ABS: return fabs(x);
                case F_SIGN: return x > 0.0 ? 1.0 : (x < 0.0 ? -1.0 : 0.0);
                case F_MIN: {
                    double r = x;
                    for (int i = 1; i < n->nargs; ++i) { double y = ev(n->a[i]); r = y < r ? y : r; }
                    return r;
                }
                case F_MAX: {
                    double r = x;
                    for (int i = 1; i < n->nargs; ++i) { double y = ev(n->a[i]); r = y > r ? y : r; }
                    return r;
                }
                case F_CLAMP: {
                    double v = ev(n->a[1]), hi = ev(n->a[2]);
                    return v < x ? x : (v > hi ? hi : v);
                }
            }
            return NAN;
        }
    }
    return NAN;
}

double oe_eval(const oe_expr *e) { return ev(e->root); }

void oe_free(oe_expr *e) {
    if (!e) return;
    free_node(e->root);
    free(e);
}
