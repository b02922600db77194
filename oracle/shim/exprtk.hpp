/*
 * exprtk-API stand-in — TEST INFRASTRUCTURE ONLY.
 *
 * exprtk 0.0.2 (pinned at cmake/Dependencies.cmake:6 of the reference) is
 * neither vendored nor installed.  The reference uses exactly this part of
 * its API (src/bcs/per_field_bc.cpp:35-182, src/ics/expression_ic.cpp:48-188):
 *   symbol_table<T>::add_variable(name, T&), add_constant(name, T)
 *   expression<T>::register_symbol_table(symbol_table&), value()
 *   parser<T>::compile(src, expression&), error_count(), get_error(i).diagnostic
 * which this header provides on top of the oracle's evaluator
 * (oracle/expr_eval.c).  Like exprtk, symbol tables and expressions are
 * shared handles: copies refer to the same underlying object.
 * Project-written; not derived from exprtk's source.
 */
#ifndef MPD_ORACLE_EXPRTK_SHIM_HPP
#define MPD_ORACLE_EXPRTK_SHIM_HPP

#include <cstddef>
#include <limits>
#include <memory>
#include <string>
#include <vector>

#include "../expr_eval.h"

namespace exprtk {

template <typename T>
class symbol_table {
public:
    symbol_table() : st_(oe_symtab_new(), oe_symtab_free) {}
    bool add_variable(const std::string &name, T &ref, bool = false) {
        return oe_symtab_add_var(st_.get(), name.c_str(), &ref) == 0;
    }
    bool add_constant(const std::string &name, const T &value) {
        return oe_symtab_add_const(st_.get(), name.c_str(), value) == 0;
    }
    oe_symtab *raw() const { return st_.get(); }

private:
    std::shared_ptr<oe_symtab> st_;
};

template <typename T>
class parser;

template <typename T>
class expression {
public:
    void register_symbol_table(symbol_table<T> &st) { tabs_.push_back(st); }
    T value() const { return e_ ? oe_eval(e_.get()) : std::numeric_limits<T>::quiet_NaN(); }

private:
    friend class parser<T>;
    std::shared_ptr<oe_expr> e_;
    std::vector<symbol_table<T>> tabs_;
};

template <typename T>
class parser {
public:
    struct error_t {
        std::string diagnostic;
    };

    bool compile(const std::string &src, expression<T> &expr) {
        errors_.clear();
        if (expr.tabs_.empty()) {
            errors_.push_back({"no symbol table registered"});
            return false;
        }
        char err[256];
        oe_expr *e = oe_compile(src.c_str(), expr.tabs_.front().raw(), err, sizeof(err));
        if (!e) {
            errors_.push_back({err});
            return false;
        }
        expr.e_ = std::shared_ptr<oe_expr>(e, oe_free);
        return true;
    }
    std::size_t error_count() const { return errors_.size(); }
    error_t get_error(std::size_t i) const { return errors_.at(i); }

private:
    std::vector<error_t> errors_;
};

}  // namespace exprtk

#endif
