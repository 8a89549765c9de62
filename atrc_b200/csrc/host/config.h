// Config tree for the Atrc JSON scene format.
//
// Mirrors the reference's ConfigGroup / ConfigArray / ConfigValue
// (src/tracer/include/agz/tracer/utility/config.h:44-120) and the JSON
// conversion of src/factory/src/utility/config_cvt.cpp:50-105: every scalar
// is kept as a string, booleans become "1"/"0" and floating-point numbers are
// formatted with std::to_string (6 decimals) before being read back with
// std::stof, exactly as the reference does (config_cvt.cpp:43-44,
// src/tracer/src/utility/config.cpp:843).
#pragma once

#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "vecmath.h"

namespace atrc {

class ConfigError : public std::runtime_error {
public:
    using std::runtime_error::runtime_error;
};

class ConfigGroup;
class ConfigArray;
class ConfigValue;

class ConfigNode {
public:
    virtual ~ConfigNode() = default;
    virtual bool is_group() const { return false; }
    virtual bool is_array() const { return false; }
    virtual bool is_value() const { return false; }
    const ConfigGroup& as_group() const;
    const ConfigArray& as_array() const;
    const ConfigValue& as_value() const;
    virtual const char* kind() const = 0;
};

class ConfigValue : public ConfigNode {
    std::string str_;
public:
    explicit ConfigValue(std::string s) : str_(std::move(s)) {}
    bool is_value() const override { return true; }
    const char* kind() const override { return "value"; }
    const std::string& as_str() const { return str_; }
    int as_int() const;
    float as_real() const;
};

class ConfigArray : public ConfigNode {
    std::vector<std::shared_ptr<ConfigNode>> elems_;
public:
    bool is_array() const override { return true; }
    const char* kind() const override { return "array"; }
    void push_back(std::shared_ptr<ConfigNode> n) { elems_.push_back(std::move(n)); }
    size_t size() const { return elems_.size(); }
    const ConfigNode& at(size_t i) const;
    float at_real(size_t i) const { return at(i).as_value().as_real(); }
    int at_int(size_t i) const { return at(i).as_value().as_int(); }
    const std::string& at_str(size_t i) const { return at(i).as_value().as_str(); }
};

class ConfigGroup : public ConfigNode {
    std::map<std::string, std::shared_ptr<ConfigNode>> children_;
public:
    bool is_group() const override { return true; }
    const char* kind() const override { return "group"; }
    void insert(const std::string& k, std::shared_ptr<ConfigNode> n) { children_[k] = std::move(n); }
    const std::map<std::string, std::shared_ptr<ConfigNode>>& children() const { return children_; }

    const ConfigNode* find_child(const std::string& name) const;
    const ConfigGroup* find_child_group(const std::string& name) const;
    const ConfigArray* find_child_array(const std::string& name) const;
    const ConfigNode& child(const std::string& name) const;
    const ConfigGroup& child_group(const std::string& name) const;
    const ConfigArray& child_array(const std::string& name) const;

    std::string child_str(const std::string& name) const;
    std::string child_str_or(const std::string& name, const std::string& d) const;
    int child_int(const std::string& name) const;
    int child_int_or(const std::string& name, int d) const;
    float child_real(const std::string& name) const;
    float child_real_or(const std::string& name, float d) const;
    Vec2 child_vec2(const std::string& name) const;
    Vec2 child_vec2_or(const std::string& name, Vec2 d) const;
    Vec3 child_vec3(const std::string& name) const;
    Vec3 child_vec3_or(const std::string& name, Vec3 d) const;
    Vec3 child_spectrum(const std::string& name) const { return child_vec3(name); }
    Vec3 child_spectrum_or(const std::string& name, Vec3 d) const { return child_vec3_or(name, d); }
    int child_vec3i_perm(const std::string& name, int out[3]) const;
    // Transform list (config.cpp:195-297): a group or an array of groups,
    // composed left-to-right, so the LAST element acts on the object first.
    Affine child_transform3(const std::string& name) const;
    Affine child_transform3_or_identity(const std::string& name) const;
    Affine2 child_transform2_or_identity(const std::string& name) const;
};

// Parse JSON text into a config tree (objects -> groups, arrays -> arrays,
// scalars -> values with the reference's string conversions).
std::shared_ptr<ConfigGroup> parse_json_config(const std::string& text);

Vec2 node_to_vec2(const ConfigNode& n);
Vec3 node_to_vec3(const ConfigNode& n);
Affine node_to_transform3(const ConfigNode& n);
Affine2 node_to_transform2(const ConfigNode& n);

bool ends_with(const std::string& s, const std::string& suffix);

}  // namespace atrc
