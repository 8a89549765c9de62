// JSON -> config tree, typed getters and transform parsing.
// Follows src/factory/src/utility/config_cvt.cpp:50-105 and
// src/tracer/src/utility/config.cpp:1-297,800-860.
#include "config.h"

#include <cctype>
#include <cmath>
#include <cstdlib>
#include <cstring>

namespace atrc {

namespace {

const float kPi = 3.14159265358979323846f;

// --------------------------------------------------------------------- JSON
class JsonParser {
public:
    explicit JsonParser(const std::string& s) : s_(s) {}

    std::shared_ptr<ConfigNode> parse_root() {
        skip_ws();
        auto n = parse_value();
        skip_ws();
        if (pos_ != s_.size()) fail("trailing characters after JSON value");
        return n;
    }

private:
    const std::string& s_;
    size_t pos_ = 0;

    [[noreturn]] void fail(const std::string& what) const {
        size_t line = 1;
        for (size_t i = 0; i < pos_ && i < s_.size(); ++i)
            if (s_[i] == '\n') ++line;
        throw ConfigError("JSON parse error at line " + std::to_string(line) + ": " + what);
    }
    void skip_ws() {
        while (pos_ < s_.size()) {
            char c = s_[pos_];
            if (c == ' ' || c == '\t' || c == '\n' || c == '\r') { ++pos_; continue; }
            // tolerate // and /* */ comments (the reference's nlohmann parser does not;
            // accepting them is harmless and eases hand-written scenes)
            if (c == '/' && pos_ + 1 < s_.size() && s_[pos_ + 1] == '/') {
                while (pos_ < s_.size() && s_[pos_] != '\n') ++pos_;
                continue;
            }
            if (c == '/' && pos_ + 1 < s_.size() && s_[pos_ + 1] == '*') {
                size_t e = s_.find("*/", pos_ + 2);
                if (e == std::string::npos) fail("unterminated comment");
                pos_ = e + 2;
                continue;
            }
            break;
        }
    }
    char peek() const { return pos_ < s_.size() ? s_[pos_] : '\0'; }
    void expect(char c) {
        if (peek() != c) fail(std::string("expected '") + c + "'");
        ++pos_;
    }

    std::string parse_string_raw() {
        expect('"');
        std::string out;
        while (true) {
            if (pos_ >= s_.size()) fail("unterminated string");
            char c = s_[pos_++];
            if (c == '"') break;
            if (c == '\\') {
                if (pos_ >= s_.size()) fail("bad escape");
                char e = s_[pos_++];
                switch (e) {
                case '"': out += '"'; break;
                case '\\': out += '\\'; break;
                case '/': out += '/'; break;
                case 'b': out += '\b'; break;
                case 'f': out += '\f'; break;
                case 'n': out += '\n'; break;
                case 'r': out += '\r'; break;
                case 't': out += '\t'; break;
                case 'u': {
                    if (pos_ + 4 > s_.size()) fail("bad \\u escape");
                    unsigned cp = std::strtoul(s_.substr(pos_, 4).c_str(), nullptr, 16);
                    pos_ += 4;
                    if (cp < 0x80) out += char(cp);
                    else if (cp < 0x800) { out += char(0xC0 | (cp >> 6)); out += char(0x80 | (cp & 0x3F)); }
                    else { out += char(0xE0 | (cp >> 12)); out += char(0x80 | ((cp >> 6) & 0x3F)); out += char(0x80 | (cp & 0x3F)); }
                    break;
                }
                default: fail("bad escape");
                }
            } else {
                out += c;
            }
        }
        return out;
    }

    std::shared_ptr<ConfigNode> parse_value() {
        skip_ws();
        char c = peek();
        if (c == '{') return parse_object();
        if (c == '[') return parse_array();
        if (c == '"') return std::make_shared<ConfigValue>(parse_string_raw());
        if (s_.compare(pos_, 4, "true") == 0) { pos_ += 4; return std::make_shared<ConfigValue>("1"); }
        if (s_.compare(pos_, 5, "false") == 0) { pos_ += 5; return std::make_shared<ConfigValue>("0"); }
        if (s_.compare(pos_, 4, "null") == 0) fail("null values are not supported");
        return parse_number();
    }

    std::shared_ptr<ConfigNode> parse_number() {
        size_t start = pos_;
        bool is_float = false;
        if (peek() == '-' || peek() == '+') ++pos_;
        while (pos_ < s_.size()) {
            char c = s_[pos_];
            if (std::isdigit((unsigned char)c)) { ++pos_; continue; }
            if (c == '.' || c == 'e' || c == 'E') { is_float = true; ++pos_; continue; }
            if ((c == '-' || c == '+') && (s_[pos_ - 1] == 'e' || s_[pos_ - 1] == 'E')) { ++pos_; continue; }
            break;
        }
        if (start == pos_) fail("unexpected character");
        std::string tok = s_.substr(start, pos_ - start);
        if (is_float) {
            // config_cvt.cpp:43: std::to_string(val.get<real>()) -- the JSON
            // number becomes a float, then a 6-decimal string.
            float f = std::strtof(tok.c_str(), nullptr);
            return std::make_shared<ConfigValue>(std::to_string(f));
        }
        // config_cvt.cpp:45: std::to_string(val.get<int>())
        long long v = std::strtoll(tok.c_str(), nullptr, 10);
        return std::make_shared<ConfigValue>(std::to_string(int(v)));
    }

    std::shared_ptr<ConfigNode> parse_object() {
        expect('{');
        auto g = std::make_shared<ConfigGroup>();
        skip_ws();
        if (peek() == '}') { ++pos_; return g; }
        while (true) {
            skip_ws();
            std::string key = parse_string_raw();
            skip_ws();
            expect(':');
            auto v = parse_value();
            g->insert(key, v);
            skip_ws();
            if (peek() == ',') { ++pos_; continue; }
            expect('}');
            break;
        }
        return g;
    }

    std::shared_ptr<ConfigNode> parse_array() {
        expect('[');
        auto a = std::make_shared<ConfigArray>();
        skip_ws();
        if (peek() == ']') { ++pos_; return a; }
        while (true) {
            a->push_back(parse_value());
            skip_ws();
            if (peek() == ',') { ++pos_; continue; }
            expect(']');
            break;
        }
        return a;
    }
};

// -------------------------------------------------------- affine helpers
void mat_mul(const float* a, const float* b, float* out) {  // 3x4 * 3x4 (affine)
    double r[12];
    for (int i = 0; i < 3; ++i) {
        for (int j = 0; j < 4; ++j) {
            double s = 0;
            for (int k = 0; k < 3; ++k) s += double(a[4 * i + k]) * double(b[4 * k + j]);
            if (j == 3) s += a[4 * i + 3];
            r[4 * i + j] = s;
        }
    }
    for (int i = 0; i < 12; ++i) out[i] = float(r[i]);
}

bool mat_inverse(const float* m, float* inv) {
    const double a = m[0], b = m[1], c = m[2], d = m[4], e = m[5], f = m[6], g = m[8], h = m[9], i = m[10];
    const double A = e * i - f * h, B = -(d * i - f * g), C = d * h - e * g;
    const double det = a * A + b * B + c * C;
    if (det == 0.0 || !std::isfinite(det)) return false;
    const double id = 1.0 / det;
    double r[9] = {A * id, -(b * i - c * h) * id, (b * f - c * e) * id,
                   B * id, (a * i - c * g) * id, -(a * f - c * d) * id,
                   C * id, -(a * h - b * g) * id, (a * e - b * d) * id};
    for (int row = 0; row < 3; ++row) {
        inv[4 * row + 0] = float(r[3 * row + 0]);
        inv[4 * row + 1] = float(r[3 * row + 1]);
        inv[4 * row + 2] = float(r[3 * row + 2]);
        double t = -(r[3 * row + 0] * m[3] + r[3 * row + 1] * m[7] + r[3 * row + 2] * m[11]);
        inv[4 * row + 3] = float(t);
    }
    return true;
}

Affine make_affine(const float* m) {
    Affine a;
    for (int i = 0; i < 12; ++i) a.m[i] = m[i];
    if (!mat_inverse(a.m, a.inv)) throw ConfigError("singular transform");
    return a;
}

Affine identity_affine() {
    Affine a;
    affine_identity(a.m);
    affine_identity(a.inv);
    return a;
}

Affine compose(const Affine& lhs, const Affine& rhs) {  // lhs * rhs
    float m[12];
    mat_mul(lhs.m, rhs.m, m);
    return make_affine(m);
}

Affine rotation(Vec3 axis, float rad) {
    // Rodrigues' rotation about a normalised axis (right-handed).
    double ax = axis.x, ay = axis.y, az = axis.z;
    double len = std::sqrt(ax * ax + ay * ay + az * az);
    if (len == 0) throw ConfigError("zero rotation axis");
    ax /= len; ay /= len; az /= len;
    double c = std::cos(double(rad)), s = std::sin(double(rad)), t = 1 - c;
    float m[12] = {float(t * ax * ax + c), float(t * ax * ay - s * az), float(t * ax * az + s * ay), 0,
                   float(t * ax * ay + s * az), float(t * ay * ay + c), float(t * ay * az - s * ax), 0,
                   float(t * ax * az - s * ay), float(t * ay * az + s * ax), float(t * az * az + c), 0};
    return make_affine(m);
}

float read_angle(const ConfigGroup& g) {
    if (auto n = g.find_child("rad")) return n->as_value().as_real();
    return g.child_real("deg") / 180 * kPi;
}

Affine basic_transform3(const ConfigGroup& g) {
    const std::string type = g.child_str("type");
    if (ends_with(type, "//")) return identity_affine();
    if (type == "translate") {
        Vec3 o = g.child_vec3("offset");
        float m[12] = {1, 0, 0, o.x, 0, 1, 0, o.y, 0, 0, 1, o.z};
        return make_affine(m);
    }
    if (type == "rotate") return rotation(g.child_vec3("axis"), read_angle(g));
    if (type == "rotate_x") return rotation(Vec3(1, 0, 0), read_angle(g));
    if (type == "rotate_y") return rotation(Vec3(0, 1, 0), read_angle(g));
    if (type == "rotate_z") return rotation(Vec3(0, 0, 1), read_angle(g));
    if (type == "scale") {
        const ConfigNode* r = g.find_child("ratio");
        if (!r) throw ConfigError("scale: missing 'ratio'");
        Vec3 s = r->is_array() ? node_to_vec3(*r) : Vec3(r->as_value().as_real());
        float m[12] = {s.x, 0, 0, 0, 0, s.y, 0, 0, 0, 0, s.z, 0};
        return make_affine(m);
    }
    if (type == "mat3") {
        // config.cpp:261-292
        if (const ConfigArray* a = g.find_child_array("row_major")) {
            if (a->size() != 9) throw ConfigError("invalid mat3 elem count");
            float m[12] = {a->at_real(0), a->at_real(1), a->at_real(2), 0,
                           a->at_real(3), a->at_real(4), a->at_real(5), 0,
                           a->at_real(6), a->at_real(7), a->at_real(8), 0};
            return make_affine(m);
        }
        if (const ConfigArray* a = g.find_child_array("col_major")) {
            if (a->size() != 9) throw ConfigError("invalid mat3 elem count");
            float m[12] = {a->at_real(0), a->at_real(3), a->at_real(6), 0,
                           a->at_real(1), a->at_real(4), a->at_real(7), 0,
                           a->at_real(2), a->at_real(5), a->at_real(8), 0};
            return make_affine(m);
        }
        throw ConfigError("row_major/col_major expected");
    }
    throw ConfigError("unknown transform3 type (type = " + type + ")");
}

Affine2 affine2_identity() {
    Affine2 a;
    a.m[0] = 1; a.m[1] = 0; a.m[2] = 0; a.m[3] = 0; a.m[4] = 1; a.m[5] = 0;
    return a;
}

Affine2 affine2_mul(const Affine2& a, const Affine2& b) {
    Affine2 r;
    r.m[0] = a.m[0] * b.m[0] + a.m[1] * b.m[3];
    r.m[1] = a.m[0] * b.m[1] + a.m[1] * b.m[4];
    r.m[2] = a.m[0] * b.m[2] + a.m[1] * b.m[5] + a.m[2];
    r.m[3] = a.m[3] * b.m[0] + a.m[4] * b.m[3];
    r.m[4] = a.m[3] * b.m[1] + a.m[4] * b.m[4];
    r.m[5] = a.m[3] * b.m[2] + a.m[4] * b.m[5] + a.m[5];
    return r;
}

Affine2 basic_transform2(const ConfigGroup& g) {
    const std::string type = g.child_str("type");
    if (ends_with(type, "//")) return affine2_identity();
    Affine2 r = affine2_identity();
    if (type == "translate") {
        Vec2 o = g.child_vec2("offset");
        r.m[2] = o.x; r.m[5] = o.y;
        return r;
    }
    if (type == "rotate") {
        float a = read_angle(g);
        r.m[0] = std::cos(a); r.m[1] = -std::sin(a);
        r.m[3] = std::sin(a); r.m[4] = std::cos(a);
        return r;
    }
    if (type == "scale") {
        const ConfigNode* n = g.find_child("ratio");
        if (!n) throw ConfigError("scale: missing 'ratio'");
        Vec2 s = n->is_array() ? node_to_vec2(*n) : Vec2(n->as_value().as_real());
        r.m[0] = s.x; r.m[4] = s.y;
        return r;
    }
    throw ConfigError("unknown transform2 type (type = " + type + ")");
}

}  // namespace

// ------------------------------------------------------------------- nodes
const ConfigGroup& ConfigNode::as_group() const {
    if (!is_group()) throw ConfigError(std::string("expected a group, found a ") + kind());
    return static_cast<const ConfigGroup&>(*this);
}
const ConfigArray& ConfigNode::as_array() const {
    if (!is_array()) throw ConfigError(std::string("expected an array, found a ") + kind());
    return static_cast<const ConfigArray&>(*this);
}
const ConfigValue& ConfigNode::as_value() const {
    if (!is_value()) throw ConfigError(std::string("expected a value, found a ") + kind());
    return static_cast<const ConfigValue&>(*this);
}

int ConfigValue::as_int() const {
    try {
        size_t idx = 0;
        int v = std::stoi(str_, &idx);
        return v;
    } catch (...) {
        throw ConfigError("cannot convert '" + str_ + "' to int");
    }
}

float ConfigValue::as_real() const {
    try {
        return std::stof(str_);
    } catch (...) {
        throw ConfigError("cannot convert '" + str_ + "' to real");
    }
}

const ConfigNode& ConfigArray::at(size_t i) const {
    if (i >= elems_.size()) throw ConfigError("array index out of range");
    return *elems_[i];
}

const ConfigNode* ConfigGroup::find_child(const std::string& name) const {
    auto it = children_.find(name);
    return it == children_.end() ? nullptr : it->second.get();
}
const ConfigGroup* ConfigGroup::find_child_group(const std::string& name) const {
    auto n = find_child(name);
    return n ? &n->as_group() : nullptr;
}
const ConfigArray* ConfigGroup::find_child_array(const std::string& name) const {
    auto n = find_child(name);
    return n ? &n->as_array() : nullptr;
}
const ConfigNode& ConfigGroup::child(const std::string& name) const {
    auto n = find_child(name);
    if (!n) throw ConfigError("missing field '" + name + "'");
    return *n;
}
const ConfigGroup& ConfigGroup::child_group(const std::string& name) const { return child(name).as_group(); }
const ConfigArray& ConfigGroup::child_array(const std::string& name) const { return child(name).as_array(); }
std::string ConfigGroup::child_str(const std::string& name) const { return child(name).as_value().as_str(); }
std::string ConfigGroup::child_str_or(const std::string& name, const std::string& d) const {
    auto n = find_child(name);
    return n ? n->as_value().as_str() : d;
}
int ConfigGroup::child_int(const std::string& name) const { return child(name).as_value().as_int(); }
int ConfigGroup::child_int_or(const std::string& name, int d) const {
    auto n = find_child(name);
    return n ? n->as_value().as_int() : d;
}
float ConfigGroup::child_real(const std::string& name) const { return child(name).as_value().as_real(); }
float ConfigGroup::child_real_or(const std::string& name, float d) const {
    auto n = find_child(name);
    return n ? n->as_value().as_real() : d;
}
Vec2 ConfigGroup::child_vec2(const std::string& name) const { return node_to_vec2(child(name)); }
Vec2 ConfigGroup::child_vec2_or(const std::string& name, Vec2 d) const {
    auto n = find_child(name);
    return n ? node_to_vec2(*n) : d;
}
Vec3 ConfigGroup::child_vec3(const std::string& name) const { return node_to_vec3(child(name)); }
Vec3 ConfigGroup::child_vec3_or(const std::string& name, Vec3 d) const {
    auto n = find_child(name);
    return n ? node_to_vec3(*n) : d;
}
int ConfigGroup::child_vec3i_perm(const std::string& name, int out[3]) const {
    auto n = find_child(name);
    if (!n) { out[0] = 0; out[1] = 1; out[2] = 2; return 0; }
    const ConfigArray& a = n->as_array();
    if (a.size() == 1) { out[0] = out[1] = out[2] = a.at_int(0); return 1; }
    if (a.size() != 3) throw ConfigError("invalid Vec3i size");
    for (int i = 0; i < 3; ++i) out[i] = a.at_int(i);
    return 1;
}
Affine ConfigGroup::child_transform3(const std::string& name) const { return node_to_transform3(child(name)); }
Affine ConfigGroup::child_transform3_or_identity(const std::string& name) const {
    auto n = find_child(name);
    return n ? node_to_transform3(*n) : identity_affine();
}
Affine2 ConfigGroup::child_transform2_or_identity(const std::string& name) const {
    auto n = find_child(name);
    return n ? node_to_transform2(*n) : affine2_identity();
}

Vec2 node_to_vec2(const ConfigNode& n) {
    const ConfigArray& a = n.as_array();
    if (a.size() == 1) return Vec2(a.at_real(0));
    if (a.size() == 2) return Vec2(a.at_real(0), a.at_real(1));
    throw ConfigError("invalid array size (actual = " + std::to_string(a.size()) + ")");
}
Vec3 node_to_vec3(const ConfigNode& n) {
    const ConfigArray& a = n.as_array();
    if (a.size() == 1) return Vec3(a.at_real(0));
    if (a.size() == 3) return Vec3(a.at_real(0), a.at_real(1), a.at_real(2));
    throw ConfigError("invalid array size (actual = " + std::to_string(a.size()) + ")");
}
Affine node_to_transform3(const ConfigNode& n) {
    if (n.is_group()) return basic_transform3(n.as_group());
    const ConfigArray& a = n.as_array();
    Affine r = identity_affine();
    for (size_t i = 0; i < a.size(); ++i) r = compose(r, basic_transform3(a.at(i).as_group()));
    return r;
}
Affine2 node_to_transform2(const ConfigNode& n) {
    if (n.is_group()) return basic_transform2(n.as_group());
    const ConfigArray& a = n.as_array();
    Affine2 r = affine2_identity();
    for (size_t i = 0; i < a.size(); ++i) r = affine2_mul(r, basic_transform2(a.at(i).as_group()));
    return r;
}

bool ends_with(const std::string& s, const std::string& suffix) {
    return s.size() >= suffix.size() && s.compare(s.size() - suffix.size(), suffix.size(), suffix) == 0;
}

std::shared_ptr<ConfigGroup> parse_json_config(const std::string& text) {
    JsonParser p(text);
    auto root = p.parse_root();
    if (!root->is_group()) throw ConfigError("the top-level JSON value must be an object");
    return std::static_pointer_cast<ConfigGroup>(root);
}

}  // namespace atrc
