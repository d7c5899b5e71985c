// Minimal stand-in for yaml-cpp's YAML::Node -- test infrastructure only.
//
// The reference's Integrator.hpp includes "yaml-cpp/yaml.h" (IntegratorConfig::
// ompConfig is a YAML::Node) and yaml-cpp is not installed here.  This header
// declares just the surface B200BDFIntegrator touches (operator[] by key, the
// "is defined" test, as<std::string>()) so that csrc/host/b200_bdf_integrator.cpp
// compiles against the reference's own headers (-DB200ODE_WITH_REFERENCE_HEADERS):
// the compile proves that its overrides bind to the reference's virtuals.  It is
// not a YAML parser and nothing links it into the product.
#pragma once

#include <map>
#include <memory>
#include <sstream>
#include <string>

namespace YAML {

class Node {
public:
    Node() = default;
    explicit Node(const std::string& scalar) : scalar_(std::make_shared<std::string>(scalar)) {}

    Node operator[](const std::string& key) const {
        if (!map_) return Node();
        auto it = map_->find(key);
        return it == map_->end() ? Node() : it->second;
    }
    Node operator[](const char* key) const { return (*this)[std::string(key)]; }
    Node& operator[](const std::string& key) {
        if (!map_) map_ = std::make_shared<std::map<std::string, Node>>();
        return (*map_)[key];
    }

    explicit operator bool() const { return scalar_ || map_; }
    bool operator!() const { return !static_cast<bool>(*this); }

    template <class T>
    T as() const {
        T out{};
        std::istringstream in(scalar_ ? *scalar_ : std::string());
        in >> out;
        return out;
    }

private:
    std::shared_ptr<std::string> scalar_;
    std::shared_ptr<std::map<std::string, Node>> map_;
};

template <>
inline std::string Node::as<std::string>() const { return scalar_ ? *scalar_ : std::string(); }

}  // namespace YAML
