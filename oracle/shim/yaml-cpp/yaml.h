/*
 * Minimal YAML::Node stand-in — TEST INFRASTRUCTURE ONLY.
 *
 * yaml-cpp 0.8.0 (pinned at cmake/Dependencies.cmake:4 of the reference) is
 * not installed here.  The reference's geometry plugins (src/geometries/*.cpp)
 * and ExpressionIC (src/ics/expression_ic.cpp:199-247) only read a map of
 * scalars through operator bool / IsNull / IsMap / IsScalar / operator[] /
 * as<T>() / map iteration, so this node supports exactly that: Null, Scalar
 * and a flat Map of scalars, built by the oracle harness from key=value text.
 * Project-written.
 */
#ifndef MPD_ORACLE_YAML_SHIM_H
#define MPD_ORACLE_YAML_SHIM_H

#include <cstdlib>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace YAML {

class Node {
public:
    enum Kind { Undefined, Null, Scalar, Map };

    Node() : kind_(Null) {}
    static Node MakeScalar(const std::string &s) {
        Node n;
        n.kind_ = Scalar;
        n.scalar_ = s;
        return n;
    }
    static Node MakeMap() {
        Node n;
        n.kind_ = Map;
        n.items_ = std::make_shared<std::vector<std::pair<Node, Node>>>();
        return n;
    }
    void Set(const std::string &key, const Node &value) {
        items_->emplace_back(MakeScalar(key), value);
    }

    explicit operator bool() const { return kind_ != Undefined; }
    bool IsNull() const { return kind_ == Null; }
    bool IsMap() const { return kind_ == Map; }
    bool IsScalar() const { return kind_ == Scalar; }
    bool IsSequence() const { return false; }

    Node operator[](const std::string &key) const {
        if (kind_ == Map)
            for (const auto &kv : *items_)
                if (kv.first.scalar_ == key) return kv.second;
        Node n;
        n.kind_ = Undefined;
        return n;
    }

    template <typename T>
    T as() const {
        if (kind_ != Scalar) throw std::runtime_error("yaml shim: not a scalar");
        std::istringstream is(scalar_);
        T v{};
        is >> v;
        if (is.fail()) throw std::runtime_error("yaml shim: bad conversion of '" + scalar_ + "'");
        return v;
    }

    using const_iterator = std::vector<std::pair<Node, Node>>::const_iterator;
    const_iterator begin() const { return items_ ? items_->begin() : empty().begin(); }
    const_iterator end() const { return items_ ? items_->end() : empty().end(); }

private:
    static const std::vector<std::pair<Node, Node>> &empty() {
        static const std::vector<std::pair<Node, Node>> e;
        return e;
    }
    Kind kind_;
    std::string scalar_;
    std::shared_ptr<std::vector<std::pair<Node, Node>>> items_;
};

template <>
inline std::string Node::as<std::string>() const {
    if (kind_ != Scalar) throw std::runtime_error("yaml shim: not a scalar");
    return scalar_;
}

template <>
inline double Node::as<double>() const {
    if (kind_ != Scalar) throw std::runtime_error("yaml shim: not a scalar");
    char *end = nullptr;
    const double v = std::strtod(scalar_.c_str(), &end);
    if (end == scalar_.c_str()) throw std::runtime_error("yaml shim: bad double '" + scalar_ + "'");
    return v;
}

}  // namespace YAML

#endif
