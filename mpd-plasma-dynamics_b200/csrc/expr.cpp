// Expression compiler (see expr.hpp).  Recursive descent that emits postfix
// code directly; the stack depth is tracked so the interpreter can use a
// fixed-size register stack.
#include "expr.hpp"

#include <cctype>
#include <cstdlib>
#include <cstring>

namespace mpd {
namespace {

struct FnInfo {
    const char *name;
    int op;       // OP_FN1 / OP_ATAN2 / OP_POW / OP_MIN2 / OP_MAX2 / OP_CLAMP
    int fn1;      // ExprFn1 for OP_FN1
    int min_args, max_args;
};

const FnInfo kFns[] = {
    {"sin", OP_FN1, FN_SIN, 1, 1},     {"cos", OP_FN1, FN_COS, 1, 1},
    {"tan", OP_FN1, FN_TAN, 1, 1},     {"asin", OP_FN1, FN_ASIN, 1, 1},
    {"acos", OP_FN1, FN_ACOS, 1, 1},   {"atan", OP_FN1, FN_ATAN, 1, 1},
    {"exp", OP_FN1, FN_EXP, 1, 1},     {"log", OP_FN1, FN_LOG, 1, 1},
    {"log2", OP_FN1, FN_LOG2, 1, 1},   {"log10", OP_FN1, FN_LOG10, 1, 1},
    {"sqrt", OP_FN1, FN_SQRT, 1, 1},   {"abs", OP_FN1, FN_ABS, 1, 1},
    {"sign", OP_FN1, FN_SIGN, 1, 1},   {"atan2", OP_ATAN2, 0, 2, 2},
    {"pow", OP_POW, 0, 2, 2},          {"min", OP_MIN2, 0, 2, 8},
    {"max", OP_MAX2, 0, 2, 8},         {"clamp", OP_CLAMP, 0, 3, 3},
};

class Compiler {
public:
    Compiler(const std::string &src, const std::vector<std::string> &syms,
             const std::map<std::string, double> &consts, ExprCode &out)
        : s_(src), syms_(syms), consts_(consts), out_(out) {}

    bool Run(std::string &err) {
        out_.code.clear();
        out_.consts.clear();
        out_.vars_used.clear();
        out_.max_depth = 0;
        Expr();
        SkipWs();
        if (!failed_ && pos_ < s_.size()) Fail("trailing input");
        if (!failed_ && depth_ != 1) Fail("empty expression");
        if (!failed_ && out_.max_depth > kExprMaxStack) Fail("expression nests too deeply");
        if (failed_) {
            err = err_;
            return false;
        }
        out_.code.push_back(OP_END);
        return true;
    }

private:
    void Fail(const std::string &msg) {
        if (failed_) return;
        failed_ = true;
        err_ = "at " + std::to_string(pos_) + ": " + msg;
    }
    void SkipWs() {
        while (pos_ < s_.size() && std::isspace(static_cast<unsigned char>(s_[pos_]))) pos_++;
    }
    char Peek() {
        SkipWs();
        return pos_ < s_.size() ? s_[pos_] : '\0';
    }
    void Emit(int op, int arg, int stack_delta) {
        out_.code.push_back((arg << 8) | op);
        depth_ += stack_delta;
        if (depth_ > out_.max_depth) out_.max_depth = depth_;
    }
    void EmitConst(double v) {
        out_.consts.push_back(v);
        Emit(OP_CONST, static_cast<int>(out_.consts.size() - 1), +1);
    }

    void Expr() {
        Term();
        for (;;) {
            if (failed_) return;
            const char c = Peek();
            if (c != '+' && c != '-') return;
            pos_++;
            Term();
            Emit(c == '+' ? OP_ADD : OP_SUB, 0, -1);
        }
    }
    void Term() {
        Unary();
        for (;;) {
            if (failed_) return;
            const char c = Peek();
            if (c != '*' && c != '/' && c != '%') return;
            pos_++;
            Unary();
            Emit(c == '*' ? OP_MUL : c == '/' ? OP_DIV : OP_MOD, 0, -1);
        }
    }
    void Unary() {
        const char c = Peek();
        if (c == '-') {
            pos_++;
            Unary();
            Emit(OP_NEG, 0, 0);
            return;
        }
        if (c == '+') {
            pos_++;
            Unary();
            return;
        }
        Power();
    }
    void Power() {
        Primary();
        if (failed_) return;
        if (Peek() == '^') {
            pos_++;
            Unary();
            Emit(OP_POW, 0, -1);
        }
    }
    void Primary() {
        if (failed_) return;
        const char c = Peek();
        if (c == '(') {
            pos_++;
            Expr();
            if (Peek() != ')') return Fail("expected ')'");
            pos_++;
            return;
        }
        const bool digit = std::isdigit(static_cast<unsigned char>(c)) != 0;
        const bool dot_digit = c == '.' && pos_ + 1 < s_.size() &&
                               std::isdigit(static_cast<unsigned char>(s_[pos_ + 1]));
        if (digit || dot_digit) {
            std::size_t k = pos_;
            while (k < s_.size() && std::isdigit(static_cast<unsigned char>(s_[k]))) k++;
            if (k < s_.size() && s_[k] == '.') {
                k++;
                while (k < s_.size() && std::isdigit(static_cast<unsigned char>(s_[k]))) k++;
            }
            if (k < s_.size() && (s_[k] == 'e' || s_[k] == 'E')) {
                std::size_t k2 = k + 1;
                if (k2 < s_.size() && (s_[k2] == '+' || s_[k2] == '-')) k2++;
                if (k2 < s_.size() && std::isdigit(static_cast<unsigned char>(s_[k2]))) {
                    k = k2;
                    while (k < s_.size() && std::isdigit(static_cast<unsigned char>(s_[k]))) k++;
                }
            }
            const std::string num = s_.substr(pos_, k - pos_);
            pos_ = k;
            EmitConst(std::strtod(num.c_str(), nullptr));
            return;
        }
        if (std::isalpha(static_cast<unsigned char>(c)) || c == '_') {
            std::size_t k = pos_;
            while (k < s_.size() &&
                   (std::isalnum(static_cast<unsigned char>(s_[k])) || s_[k] == '_'))
                k++;
            const std::string name = s_.substr(pos_, k - pos_);
            pos_ = k;
            if (Peek() == '(') return Call(name);
            for (std::size_t i = 0; i < syms_.size(); ++i) {
                if (syms_[i] == name) {
                    Emit(OP_VAR, static_cast<int>(i), +1);
                    out_.vars_used.push_back(static_cast<int>(i));
                    return;
                }
            }
            auto it = consts_.find(name);
            if (it != consts_.end()) return EmitConst(it->second);
            return Fail("undefined symbol '" + name + "'");
        }
        if (c == '\0') return Fail("unexpected end of expression");
        return Fail(std::string("unexpected character '") + c + "'");
    }
    void Call(const std::string &name) {
        const FnInfo *fn = nullptr;
        for (const auto &f : kFns)
            if (name == f.name) fn = &f;
        if (!fn) return Fail("unknown function '" + name + "'");
        pos_++;  // '('
        int nargs = 0;
        for (;;) {
            Expr();
            if (failed_) return;
            nargs++;
            // variadic min/max fold left to right as the arguments arrive
            if ((fn->op == OP_MIN2 || fn->op == OP_MAX2) && nargs >= 2) Emit(fn->op, 0, -1);
            const char c = Peek();
            if (c == ',') {
                pos_++;
                continue;
            }
            if (c == ')') {
                pos_++;
                break;
            }
            return Fail("expected ',' or ')'");
        }
        if (nargs < fn->min_args || nargs > fn->max_args)
            return Fail("wrong number of arguments to '" + name + "'");
        switch (fn->op) {
            case OP_FN1: Emit(OP_FN1, fn->fn1, 0); break;
            case OP_ATAN2:
            case OP_POW: Emit(fn->op, 0, -1); break;
            case OP_CLAMP: Emit(OP_CLAMP, 0, -2); break;
            default: break;  // min/max already emitted
        }
    }

    const std::string &s_;
    const std::vector<std::string> &syms_;
    const std::map<std::string, double> &consts_;
    ExprCode &out_;
    std::size_t pos_ = 0;
    int depth_ = 0;
    bool failed_ = false;
    std::string err_;
};

}  // namespace

bool CompileExpr(const std::string &src, const std::vector<std::string> &symbols,
                 const std::map<std::string, double> &constants, ExprCode &out,
                 std::string &err) {
    Compiler c(src, symbols, constants, out);
    return c.Run(err);
}

}  // namespace mpd
