// agz-utils compatibility shim (test infrastructure).
//
// Atrc's tracer and factory include agz-utils (https://github.com/AirGuanZ/
// agz-utils), a git submodule whose checkout is empty in the reference, with
// no pinned commit.  This header restates the subset that the tracer and the
// factory call -- vectors, colours, frames, transforms, matrices, sampling
// distributions, texture containers and filters, the object arena, a thread
// group, image and mesh loading, string helpers -- written from the
// mathematics and from the way the reference calls it, so that the
// reference's own sources compile and render here as a second oracle for the
// pt_cuda renderer.  Where agz-utils fixes a convention the reference does not
// show (luminance weights, the cosine-hemisphere and triangle mappings,
// frames from a normal, texel centres, alias tables), the shim uses the same
// convention as this project's CPU oracle and device code: parity at that
// boundary is by construction, not pinned by agz-utils itself.
#pragma once

#include <algorithm>
#include <array>
#include <atomic>
#include <cassert>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <exception>
#include <filesystem>
#include <fstream>
#include <functional>
#include <limits>
#include <memory>
#include <mutex>
#include <span>
#include <sstream>
#include <stdexcept>
#include <string>
#include <thread>
#include <tuple>
#include <type_traits>
#include <utility>
#include <variant>
#include <vector>

// ----------------------------------------------------------------- macros

#define AGZ_SHIM_CAT2(a, b) a##b
#define AGZ_SHIM_CAT(a, b) AGZ_SHIM_CAT2(a, b)
// AGZ_SCOPE_EXIT{ ... }; runs the block when the enclosing scope ends: the
// guard is a named local (a temporary would run it at once)
#define AGZ_SCOPE_EXIT auto AGZ_SHIM_CAT(agz_scope_exit_, __COUNTER__) = ::agz::misc::scope_exit_maker_t{} + [&]() -> void
#define AGZ_UNACCESSED(x) ((void)(x))
#define AGZ_HIERARCHY_TRY try {
#define AGZ_HIERARCHY_WRAP(MSG)                                         \
    }                                                                   \
    catch (...) {                                                       \
        std::throw_with_nested(::agz::misc::hierarchy_exception_t(MSG)); \
    }

namespace agz {

struct uninitialized_t {};
inline constexpr uninitialized_t UNINIT{};

template <class T, size_t N>
constexpr size_t array_size(const T (&)[N]) noexcept { return N; }

// ------------------------------------------------------------------- misc
namespace misc {

class uncopyable_t {
public:
    uncopyable_t() = default;
    uncopyable_t(const uncopyable_t&) = delete;
    uncopyable_t& operator=(const uncopyable_t&) = delete;
};

struct hierarchy_exception_t : std::runtime_error {
    using std::runtime_error::runtime_error;
};

template <class F>
struct scope_exit_t {
    F f;
    ~scope_exit_t() { f(); }
};
struct scope_exit_maker_t {
    template <class F>
    scope_exit_t<F> operator+(F&& f) const { return scope_exit_t<F>{std::forward<F>(f)}; }
};

template <class T>
using span = std::span<T>;

template <class... Fs>
struct overloaded_t : Fs... {
    using Fs::operator()...;
};
template <class... Fs>
overloaded_t(Fs...) -> overloaded_t<Fs...>;

template <class... Ts>
class variant_t : public std::variant<Ts...> {
public:
    using std::variant<Ts...>::variant;
    using std::variant<Ts...>::operator=;
    template <class T> bool is() const noexcept { return std::holds_alternative<T>(*this); }
    template <class T> T& as() { return std::get<T>(*this); }
    template <class T> const T& as() const { return std::get<T>(*this); }
    template <class T> T* as_if() noexcept { return std::get_if<T>(this); }
    template <class T> const T* as_if() const noexcept { return std::get_if<T>(this); }
    template <class... Fs> decltype(auto) match(Fs&&... fs) { return std::visit(overloaded_t<std::decay_t<Fs>...>{std::forward<Fs>(fs)...}, static_cast<std::variant<Ts...>&>(*this)); }
    template <class... Fs> decltype(auto) match(Fs&&... fs) const { return std::visit(overloaded_t<std::decay_t<Fs>...>{std::forward<Fs>(fs)...}, static_cast<const std::variant<Ts...>&>(*this)); }
};


template <class V, class... Fs>
decltype(auto) match_variant(V&& v, Fs&&... fs) {
    return std::visit(overloaded_t{std::forward<Fs>(fs)...}, std::forward<V>(v));
}

// Restores a variable's value when the scope ends.
template <class T>
class scope_assignment_t {
    T* dst_ = nullptr;
    T old_{};

    void restore() noexcept {
        if (dst_) *dst_ = old_;
        dst_ = nullptr;
    }

public:
    scope_assignment_t() = default;
    scope_assignment_t(T* dst, const T& v) : dst_(dst), old_(*dst) { *dst_ = v; }
    scope_assignment_t(const scope_assignment_t&) = delete;
    scope_assignment_t& operator=(const scope_assignment_t&) = delete;
    scope_assignment_t(scope_assignment_t&& o) noexcept : dst_(o.dst_), old_(o.old_) { o.dst_ = nullptr; }
    // the assignment held before is undone first
    scope_assignment_t& operator=(scope_assignment_t&& o) noexcept {
        if (this != &o) {
            restore();
            dst_ = o.dst_;
            old_ = o.old_;
            o.dst_ = nullptr;
        }
        return *this;
    }
    ~scope_assignment_t() { restore(); }
};

// Hash combination (boost-style golden-ratio mixing).
inline size_t hash_combine(size_t seed, size_t h) { return seed ^ (h + 0x9e3779b97f4a7c15ull + (seed << 6) + (seed >> 2)); }
template <class... Ts>
size_t hash(const Ts&... xs) {
    size_t s = 0;
    ((s = hash_combine(s, std::hash<Ts>{}(xs))), ...);
    return s;
}

[[noreturn]] inline void unreachable() {
    std::fprintf(stderr, "agz shim: unreachable code reached\n");
    std::abort();
}

}  // namespace misc

// ------------------------------------------------------------------- math
namespace math {

template <class T>
constexpr T PI = T(3.14159265358979323846264338327950288);
template <class T>
constexpr T invPI = T(1) / PI<T>;

template <class T>
constexpr T sqr(T x) noexcept { return x * x; }
template <class T>
constexpr T clamp(T x, T lo, T hi) noexcept { return x < lo ? lo : (x > hi ? hi : x); }
template <class T>
constexpr T saturate(T x) noexcept { return clamp<T>(x, T(0), T(1)); }
template <class T, class F>
constexpr T lerp(T a, T b, F t) noexcept { return a * (F(1) - t) + b * t; }
template <class T, class F>
constexpr T mix(T a, T b, F t) noexcept { return a * (F(1) - t) + b * t; }
template <class T>
std::pair<T, T> minmax(T a, T b) noexcept { return a < b ? std::make_pair(a, b) : std::make_pair(b, a); }
template <class T>
constexpr T deg2rad(T d) noexcept { return d * (PI<T> / T(180)); }
template <class T>
constexpr T rad2deg(T r) noexcept { return r * (T(180) / PI<T>); }
inline bool is_finite(float x) noexcept { return std::isfinite(x); }
inline bool is_finite(double x) noexcept { return std::isfinite(x); }
template <class T>
T atomic_add(std::atomic<T>& a, T v) {
    T old = a.load();
    while (!a.compare_exchange_weak(old, old + v)) {
    }
    return old;
}

// ---------------------------------------------------------------- tvec2
template <class T>
struct tvec2 {
    T x, y;
    constexpr tvec2() noexcept : x(0), y(0) {}
    constexpr explicit tvec2(T v) noexcept : x(v), y(v) {}
    constexpr tvec2(T x_, T y_) noexcept : x(x_), y(y_) {}
    explicit tvec2(uninitialized_t) noexcept {}
    template <class U>
    constexpr explicit tvec2(const tvec2<U>& o) noexcept : x(T(o.x)), y(T(o.y)) {}
    T& operator[](size_t i) noexcept { return i == 0 ? x : y; }
    const T& operator[](size_t i) const noexcept { return i == 0 ? x : y; }
    T length_square() const noexcept { return x * x + y * y; }
    T length() const noexcept { return std::sqrt(length_square()); }
    tvec2 normalize() const noexcept { return *this / length(); }
    T product() const noexcept { return x * y; }
    T sum() const noexcept { return x + y; }
    T min_elem() const noexcept { return (std::min)(x, y); }
    T max_elem() const noexcept { return (std::max)(x, y); }
    bool is_zero() const noexcept { return x == T(0) && y == T(0); }
    bool operator!() const noexcept { return is_zero(); }
    template <class F>
    auto map(F&& f) const { return tvec2<decltype(f(x))>(f(x), f(y)); }
    tvec2 clamp(T lo, T hi) const noexcept { return tvec2(math::clamp(x, lo, hi), math::clamp(y, lo, hi)); }
    tvec2 saturate() const noexcept { return clamp(T(0), T(1)); }
    tvec2 abs() const noexcept { return tvec2(std::abs(x), std::abs(y)); }
    tvec2 operator-() const noexcept { return tvec2(-x, -y); }
    tvec2& operator+=(const tvec2& o) noexcept { x += o.x; y += o.y; return *this; }
    tvec2& operator-=(const tvec2& o) noexcept { x -= o.x; y -= o.y; return *this; }
    tvec2& operator*=(const tvec2& o) noexcept { x *= o.x; y *= o.y; return *this; }
    tvec2& operator/=(const tvec2& o) noexcept { x /= o.x; y /= o.y; return *this; }
    tvec2& operator*=(T s) noexcept { x *= s; y *= s; return *this; }
    tvec2& operator/=(T s) noexcept { x /= s; y /= s; return *this; }
    bool operator==(const tvec2& o) const noexcept { return x == o.x && y == o.y; }
    bool operator!=(const tvec2& o) const noexcept { return !(*this == o); }
};
template <class T> tvec2<T> operator+(const tvec2<T>& a, const tvec2<T>& b) noexcept { return {a.x + b.x, a.y + b.y}; }
template <class T> tvec2<T> operator-(const tvec2<T>& a, const tvec2<T>& b) noexcept { return {a.x - b.x, a.y - b.y}; }
template <class T> tvec2<T> operator*(const tvec2<T>& a, const tvec2<T>& b) noexcept { return {a.x * b.x, a.y * b.y}; }
template <class T> tvec2<T> operator/(const tvec2<T>& a, const tvec2<T>& b) noexcept { return {a.x / b.x, a.y / b.y}; }
template <class T> tvec2<T> operator*(const tvec2<T>& a, T s) noexcept { return {a.x * s, a.y * s}; }
template <class T> tvec2<T> operator*(T s, const tvec2<T>& a) noexcept { return {s * a.x, s * a.y}; }
template <class T> tvec2<T> operator/(const tvec2<T>& a, T s) noexcept { return {a.x / s, a.y / s}; }
template <class T> tvec2<T> operator+(const tvec2<T>& a, T s) noexcept { return {a.x + s, a.y + s}; }
template <class T> tvec2<T> operator-(const tvec2<T>& a, T s) noexcept { return {a.x - s, a.y - s}; }
template <class T> T dot(const tvec2<T>& a, const tvec2<T>& b) noexcept { return a.x * b.x + a.y * b.y; }
template <class T> tvec2<T> elem_min(const tvec2<T>& a, const tvec2<T>& b) noexcept { return {(std::min)(a.x, b.x), (std::min)(a.y, b.y)}; }
template <class T> tvec2<T> elem_max(const tvec2<T>& a, const tvec2<T>& b) noexcept { return {(std::max)(a.x, b.x), (std::max)(a.y, b.y)}; }
template <class T> T length(const tvec2<T>& a) noexcept { return a.length(); }
template <class T> T distance(const tvec2<T>& a, const tvec2<T>& b) noexcept { return (a - b).length(); }
template <class T> T distance2(const tvec2<T>& a, const tvec2<T>& b) noexcept { return (a - b).length_square(); }
template <class T> tvec2<T> normalize(const tvec2<T>& a) noexcept { return a.normalize(); }

// ---------------------------------------------------------------- tvec3
template <class T>
struct tvec3 {
    T x, y, z;
    constexpr tvec3() noexcept : x(0), y(0), z(0) {}
    constexpr explicit tvec3(T v) noexcept : x(v), y(v), z(v) {}
    constexpr tvec3(T x_, T y_, T z_) noexcept : x(x_), y(y_), z(z_) {}
    constexpr tvec3(const tvec2<T>& xy, T z_) noexcept : x(xy.x), y(xy.y), z(z_) {}
    explicit tvec3(uninitialized_t) noexcept {}
    template <class U>
    constexpr explicit tvec3(const tvec3<U>& o) noexcept : x(T(o.x)), y(T(o.y)), z(T(o.z)) {}
    T& operator[](size_t i) noexcept { return i == 0 ? x : (i == 1 ? y : z); }
    const T& operator[](size_t i) const noexcept { return i == 0 ? x : (i == 1 ? y : z); }
    T length_square() const noexcept { return x * x + y * y + z * z; }
    T length() const noexcept { return std::sqrt(length_square()); }
    tvec3 normalize() const noexcept { return *this / length(); }
    T product() const noexcept { return x * y * z; }
    T sum() const noexcept { return x + y + z; }
    T min_elem() const noexcept { return (std::min)((std::min)(x, y), z); }
    T max_elem() const noexcept { return (std::max)((std::max)(x, y), z); }
    bool is_zero() const noexcept { return x == T(0) && y == T(0) && z == T(0); }
    bool operator!() const noexcept { return is_zero(); }
    bool is_finite() const noexcept { return std::isfinite(x) && std::isfinite(y) && std::isfinite(z); }
    template <class F>
    auto map(F&& f) const { return tvec3<decltype(f(x))>(f(x), f(y), f(z)); }
    tvec3 clamp(T lo, T hi) const noexcept { return tvec3(math::clamp(x, lo, hi), math::clamp(y, lo, hi), math::clamp(z, lo, hi)); }
    tvec3 saturate() const noexcept { return clamp(T(0), T(1)); }
    tvec3 abs() const noexcept { return tvec3(std::abs(x), std::abs(y), std::abs(z)); }
    tvec2<T> xy() const noexcept { return {x, y}; }
    tvec3 operator-() const noexcept { return tvec3(-x, -y, -z); }
    tvec3& operator+=(const tvec3& o) noexcept { x += o.x; y += o.y; z += o.z; return *this; }
    tvec3& operator-=(const tvec3& o) noexcept { x -= o.x; y -= o.y; z -= o.z; return *this; }
    tvec3& operator*=(const tvec3& o) noexcept { x *= o.x; y *= o.y; z *= o.z; return *this; }
    tvec3& operator/=(const tvec3& o) noexcept { x /= o.x; y /= o.y; z /= o.z; return *this; }
    tvec3& operator*=(T s) noexcept { x *= s; y *= s; z *= s; return *this; }
    tvec3& operator/=(T s) noexcept { x /= s; y /= s; z /= s; return *this; }
    bool operator==(const tvec3& o) const noexcept { return x == o.x && y == o.y && z == o.z; }
    bool operator!=(const tvec3& o) const noexcept { return !(*this == o); }
};
template <class T> tvec3<T> operator+(const tvec3<T>& a, const tvec3<T>& b) noexcept { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class T> tvec3<T> operator-(const tvec3<T>& a, const tvec3<T>& b) noexcept { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class T> tvec3<T> operator*(const tvec3<T>& a, const tvec3<T>& b) noexcept { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
template <class T> tvec3<T> operator/(const tvec3<T>& a, const tvec3<T>& b) noexcept { return {a.x / b.x, a.y / b.y, a.z / b.z}; }
template <class T> tvec3<T> operator*(const tvec3<T>& a, T s) noexcept { return {a.x * s, a.y * s, a.z * s}; }
template <class T> tvec3<T> operator*(T s, const tvec3<T>& a) noexcept { return {s * a.x, s * a.y, s * a.z}; }
template <class T> tvec3<T> operator/(const tvec3<T>& a, T s) noexcept { return {a.x / s, a.y / s, a.z / s}; }
template <class T> tvec3<T> operator/(T s, const tvec3<T>& a) noexcept { return {s / a.x, s / a.y, s / a.z}; }
template <class T> tvec3<T> operator+(const tvec3<T>& a, T s) noexcept { return {a.x + s, a.y + s, a.z + s}; }
template <class T> tvec3<T> operator-(const tvec3<T>& a, T s) noexcept { return {a.x - s, a.y - s, a.z - s}; }
template <class T> tvec3<T> operator-(T s, const tvec3<T>& a) noexcept { return {s - a.x, s - a.y, s - a.z}; }
template <class T> T dot(const tvec3<T>& a, const tvec3<T>& b) noexcept { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class T> tvec3<T> cross(const tvec3<T>& a, const tvec3<T>& b) noexcept {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <class T> T cos(const tvec3<T>& a, const tvec3<T>& b) noexcept { return dot(a, b) / (a.length() * b.length()); }
template <class T> tvec3<T> elem_min(const tvec3<T>& a, const tvec3<T>& b) noexcept {
    return {(std::min)(a.x, b.x), (std::min)(a.y, b.y), (std::min)(a.z, b.z)};
}
template <class T> tvec3<T> elem_max(const tvec3<T>& a, const tvec3<T>& b) noexcept {
    return {(std::max)(a.x, b.x), (std::max)(a.y, b.y), (std::max)(a.z, b.z)};
}
template <class T> T distance(const tvec3<T>& a, const tvec3<T>& b) noexcept { return (a - b).length(); }
template <class T> T distance2(const tvec3<T>& a, const tvec3<T>& b) noexcept { return (a - b).length_square(); }
template <class T> T length(const tvec3<T>& a) noexcept { return a.length(); }
template <class T> T length_square(const tvec3<T>& a) noexcept { return a.length_square(); }
template <class T> tvec3<T> normalize(const tvec3<T>& a) noexcept { return a.normalize(); }

// ---------------------------------------------------------------- tvec4
template <class T>
struct tvec4 {
    T x, y, z, w;
    constexpr tvec4() noexcept : x(0), y(0), z(0), w(0) {}
    constexpr explicit tvec4(T v) noexcept : x(v), y(v), z(v), w(v) {}
    constexpr tvec4(T x_, T y_, T z_, T w_) noexcept : x(x_), y(y_), z(z_), w(w_) {}
    constexpr tvec4(const tvec3<T>& v, T w_) noexcept : x(v.x), y(v.y), z(v.z), w(w_) {}
    explicit tvec4(uninitialized_t) noexcept {}
    T& operator[](size_t i) noexcept { return i == 0 ? x : (i == 1 ? y : (i == 2 ? z : w)); }
    const T& operator[](size_t i) const noexcept { return i == 0 ? x : (i == 1 ? y : (i == 2 ? z : w)); }
    tvec3<T> xyz() const noexcept { return {x, y, z}; }
};
template <class T> tvec4<T> operator*(const tvec4<T>& a, T s) noexcept { return {a.x * s, a.y * s, a.z * s, a.w * s}; }
template <class T> tvec4<T> operator+(const tvec4<T>& a, const tvec4<T>& b) noexcept { return {a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w}; }
template <class T> T dot(const tvec4<T>& a, const tvec4<T>& b) noexcept { return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w; }

using vec2 = tvec2<float>;
using vec3 = tvec3<float>;
using vec4 = tvec4<float>;
using vec2i = tvec2<int>;
using vec3i = tvec3<int>;
using vec4i = tvec4<int>;
using float2 = tvec2<float>;
using float3 = tvec3<float>;
using float4 = tvec4<float>;

// ----------------------------------------------------------------- aabb
template <class V>
struct taabb {
    V low, high;
    taabb() noexcept = default;
    taabb(const V& lo, const V& hi) noexcept : low(lo), high(hi) {}
    explicit taabb(uninitialized_t) noexcept : low(UNINIT), high(UNINIT) {}
    bool contains(const V& p) const noexcept {
        for (size_t i = 0; i < sizeof(V) / sizeof(p.x); ++i)
            if (p[i] < low[i] || p[i] > high[i]) return false;
        return true;
    }
};
template <class T>
using taabb2 = taabb<tvec2<T>>;
template <class T>
using taabb3 = taabb<tvec3<T>>;
using aabb2i = taabb2<int>;
using aabb3i = taabb3<int>;

// --------------------------------------------------------------- tcolor3
template <class T>
struct tcolor3 {
    T r, g, b;
    constexpr tcolor3() noexcept : r(0), g(0), b(0) {}
    constexpr explicit tcolor3(T v) noexcept : r(v), g(v), b(v) {}
    constexpr tcolor3(T r_, T g_, T b_) noexcept : r(r_), g(g_), b(b_) {}
    explicit tcolor3(uninitialized_t) noexcept {}
    constexpr explicit tcolor3(const tvec3<T>& v) noexcept : r(v.x), g(v.y), b(v.z) {}
    template <class U>
    constexpr explicit tcolor3(const tcolor3<U>& o) noexcept : r(T(o.r)), g(T(o.g)), b(T(o.b)) {}
    T& operator[](size_t i) noexcept { return i == 0 ? r : (i == 1 ? g : b); }
    const T& operator[](size_t i) const noexcept { return i == 0 ? r : (i == 1 ? g : b); }
    // ITU-R BT.709 relative luminance
    T lum() const noexcept { return T(0.2126) * r + T(0.7152) * g + T(0.0722) * b; }
    bool is_black() const noexcept { return r == T(0) && g == T(0) && b == T(0); }
    bool operator!() const noexcept { return is_black(); }
    bool is_finite() const noexcept { return std::isfinite(float(r)) && std::isfinite(float(g)) && std::isfinite(float(b)); }
    T min_elem() const noexcept { return (std::min)((std::min)(r, g), b); }
    T max_elem() const noexcept { return (std::max)((std::max)(r, g), b); }
    template <class F>
    auto map(F&& f) const { return tcolor3<std::decay_t<decltype(f(r))>>(f(r), f(g), f(b)); }
    tcolor3 clamp(T lo, T hi) const noexcept { return tcolor3(math::clamp(r, lo, hi), math::clamp(g, lo, hi), math::clamp(b, lo, hi)); }
    tcolor3 saturate() const noexcept { return clamp(T(0), T(1)); }
    tvec3<T> to_vec3() const noexcept { return {r, g, b}; }
    tcolor3 operator-() const noexcept { return tcolor3(-r, -g, -b); }
    tcolor3& operator+=(const tcolor3& o) noexcept { r += o.r; g += o.g; b += o.b; return *this; }
    tcolor3& operator-=(const tcolor3& o) noexcept { r -= o.r; g -= o.g; b -= o.b; return *this; }
    tcolor3& operator*=(const tcolor3& o) noexcept { r *= o.r; g *= o.g; b *= o.b; return *this; }
    tcolor3& operator/=(const tcolor3& o) noexcept { r /= o.r; g /= o.g; b /= o.b; return *this; }
    tcolor3& operator*=(T s) noexcept { r *= s; g *= s; b *= s; return *this; }
    tcolor3& operator/=(T s) noexcept { r /= s; g /= s; b /= s; return *this; }
    bool operator==(const tcolor3& o) const noexcept { return r == o.r && g == o.g && b == o.b; }
    bool operator!=(const tcolor3& o) const noexcept { return !(*this == o); }
};
template <class T> tcolor3<T> operator+(const tcolor3<T>& a, const tcolor3<T>& b) noexcept { return {a.r + b.r, a.g + b.g, a.b + b.b}; }
template <class T> tcolor3<T> operator-(const tcolor3<T>& a, const tcolor3<T>& b) noexcept { return {a.r - b.r, a.g - b.g, a.b - b.b}; }
template <class T> tcolor3<T> operator*(const tcolor3<T>& a, const tcolor3<T>& b) noexcept { return {a.r * b.r, a.g * b.g, a.b * b.b}; }
template <class T> tcolor3<T> operator/(const tcolor3<T>& a, const tcolor3<T>& b) noexcept { return {a.r / b.r, a.g / b.g, a.b / b.b}; }
template <class T> tcolor3<T> operator*(const tcolor3<T>& a, T s) noexcept { return {a.r * s, a.g * s, a.b * s}; }
template <class T> tcolor3<T> operator*(T s, const tcolor3<T>& a) noexcept { return {s * a.r, s * a.g, s * a.b}; }
template <class T> tcolor3<T> operator/(const tcolor3<T>& a, T s) noexcept { return {a.r / s, a.g / s, a.b / s}; }
template <class T> tcolor3<T> operator/(T s, const tcolor3<T>& a) noexcept { return {s / a.r, s / a.g, s / a.b}; }
template <class T> tcolor3<T> operator+(const tcolor3<T>& a, T s) noexcept { return {a.r + s, a.g + s, a.b + s}; }
template <class T> tcolor3<T> operator+(T s, const tcolor3<T>& a) noexcept { return {s + a.r, s + a.g, s + a.b}; }
template <class T> tcolor3<T> operator-(const tcolor3<T>& a, T s) noexcept { return {a.r - s, a.g - s, a.b - s}; }
template <class T> tcolor3<T> operator-(T s, const tcolor3<T>& a) noexcept { return {s - a.r, s - a.g, s - a.b}; }
template <class T> tcolor3<T> exp(const tcolor3<T>& c) noexcept { return {std::exp(c.r), std::exp(c.g), std::exp(c.b)}; }
template <class T> tcolor3<T> sqrt(const tcolor3<T>& c) noexcept { return {std::sqrt(c.r), std::sqrt(c.g), std::sqrt(c.b)}; }
template <class T> tcolor3<T> log(const tcolor3<T>& c) noexcept { return {std::log(c.r), std::log(c.g), std::log(c.b)}; }
template <class T> tcolor3<T> abs(const tcolor3<T>& c) noexcept { return {std::abs(c.r), std::abs(c.g), std::abs(c.b)}; }
template <class T, class U> tcolor3<T> pow(const tcolor3<T>& c, U e) noexcept {
    return {T(std::pow(c.r, e)), T(std::pow(c.g, e)), T(std::pow(c.b, e))};
}
template <class T> tcolor3<T> elem_min(const tcolor3<T>& a, const tcolor3<T>& b) noexcept {
    return {(std::min)(a.r, b.r), (std::min)(a.g, b.g), (std::min)(a.b, b.b)};
}
template <class T> tcolor3<T> elem_max(const tcolor3<T>& a, const tcolor3<T>& b) noexcept {
    return {(std::max)(a.r, b.r), (std::max)(a.g, b.g), (std::max)(a.b, b.b)};
}
template <class T> bool is_finite(const tcolor3<T>& c) noexcept { return c.is_finite(); }
template <class T> bool is_black(const tcolor3<T>& c) noexcept { return c.is_black(); }
template <class T, class F> tcolor3<T> lerp(const tcolor3<T>& a, const tcolor3<T>& b, F t) noexcept { return a * (T(1) - T(t)) + b * T(t); }
template <class T, class F> tcolor3<T> mix(const tcolor3<T>& a, const tcolor3<T>& b, F t) noexcept { return a * (T(1) - T(t)) + b * T(t); }
template <class T> tcolor3<T> clamp(const tcolor3<T>& c, T lo, T hi) noexcept { return c.clamp(lo, hi); }
template <class T> tcolor3<T> saturate(const tcolor3<T>& c) noexcept { return c.saturate(); }

using color3f = tcolor3<float>;
using color3b = tcolor3<uint8_t>;

template <class T = float>
tcolor3<T> from_color3b(const color3b& c) noexcept { return {T(c.r) / T(255), T(c.g) / T(255), T(c.b) / T(255)}; }
template <class T>
color3b to_color3b(const tcolor3<T>& c) noexcept {
    auto q = [](T v) { return uint8_t(math::clamp<T>(v, T(0), T(1)) * T(255)); };
    return {q(c.r), q(c.g), q(c.b)};
}

// The SIMD spectrum of agz-utils, a float colour that is a type of its own
// (the reference overloads on it beside tcolor3<float>).
struct _simd_float3_t : tcolor3<float> {
    using tcolor3<float>::tcolor3;
    constexpr _simd_float3_t() noexcept : tcolor3<float>() {}
    constexpr _simd_float3_t(const tcolor3<float>& c) noexcept : tcolor3<float>(c) {}
    constexpr explicit _simd_float3_t(const tvec3<float>& v) noexcept : tcolor3<float>(v.x, v.y, v.z) {}
};

// ---------------------------------------------------------------- tcoord3
// An orthonormal frame (x, y, z).
template <class T>
struct tcoord3 {
    tvec3<T> x, y, z;
    tcoord3() noexcept : x(1, 0, 0), y(0, 1, 0), z(0, 0, 1) {}
    tcoord3(const tvec3<T>& x_, const tvec3<T>& y_, const tvec3<T>& z_) noexcept : x(x_), y(y_), z(z_) {}
    explicit tcoord3(uninitialized_t) noexcept : x(UNINIT), y(UNINIT), z(UNINIT) {}
    // x from the world axis least aligned with z, y = z cross x
    static tcoord3 from_z(const tvec3<T>& zz) noexcept {
        const tvec3<T> nz = zz.normalize();
        const tvec3<T> t = std::abs(nz.x) > T(0.9) ? tvec3<T>(0, 1, 0) : tvec3<T>(1, 0, 0);
        const tvec3<T> ny = cross(nz, t).normalize();
        const tvec3<T> nx = cross(ny, nz);
        return tcoord3(nx, ny, nz);
    }
    tvec3<T> local_to_global(const tvec3<T>& v) const noexcept { return x * v.x + y * v.y + z * v.z; }
    tvec3<T> global_to_local(const tvec3<T>& v) const noexcept { return {dot(v, x), dot(v, y), dot(v, z)}; }
    bool in_positive_z_hemisphere(const tvec3<T>& v) const noexcept { return dot(v, z) > 0; }
    // the frame turned so that its z is new_z (Gram-Schmidt of the old x)
    tcoord3 rotate_to_new_z(const tvec3<T>& new_z) const noexcept {
        const tvec3<T> nz = new_z.normalize();
        tvec3<T> nx = x - nz * dot(x, nz);
        const T l = nx.length();
        if (!(l > T(1e-6))) return from_z(nz);
        nx = nx / l;
        return tcoord3(nx, cross(nz, nx), nz);
    }
    tcoord3 operator-() const noexcept { return tcoord3(-x, -y, -z); }
};
using float3_coord = tcoord3<float>;

// --------------------------------------------------------------- matrices
// Column-major 3x3 / 4x4 matrices (agz-utils' *_c); m[c][r].
template <class T>
struct tmat3_c {
    T m[3][3];
    tmat3_c() noexcept { set_identity(); }
    explicit tmat3_c(uninitialized_t) noexcept {}
    // the nine elements row by row
    tmat3_c(T m00, T m01, T m02, T m10, T m11, T m12, T m20, T m21, T m22) noexcept {
        const T v[9] = {m00, m01, m02, m10, m11, m12, m20, m21, m22};
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) m[c][r] = v[3 * r + c];
    }
    T* operator[](int c) noexcept { return m[c]; }  // column c
    const T* operator[](int c) const noexcept { return m[c]; }
    void set_identity() noexcept {
        for (int c = 0; c < 3; ++c)
            for (int r = 0; r < 3; ++r) m[c][r] = c == r ? T(1) : T(0);
    }
    static tmat3_c from_rows(const tvec3<T>& r0, const tvec3<T>& r1, const tvec3<T>& r2) noexcept {
        tmat3_c a(UNINIT);
        const tvec3<T> rows[3] = {r0, r1, r2};
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) a.m[c][r] = rows[r][c];
        return a;
    }
    static tmat3_c from_cols(const tvec3<T>& c0, const tvec3<T>& c1, const tvec3<T>& c2) noexcept {
        tmat3_c a(UNINIT);
        const tvec3<T> cols[3] = {c0, c1, c2};
        for (int c = 0; c < 3; ++c)
            for (int r = 0; r < 3; ++r) a.m[c][r] = cols[c][r];
        return a;
    }
    static tmat3_c all(T v) noexcept {
        tmat3_c a(UNINIT);
        for (int c = 0; c < 3; ++c)
            for (int r = 0; r < 3; ++r) a.m[c][r] = v;
        return a;
    }
    T& operator()(int r, int c) noexcept { return m[c][r]; }
    const T& operator()(int r, int c) const noexcept { return m[c][r]; }
    tvec3<T> get_row(int r) const noexcept { return {m[0][r], m[1][r], m[2][r]}; }
    tvec3<T> get_col(int c) const noexcept { return {m[c][0], m[c][1], m[c][2]}; }
    tvec3<T> operator*(const tvec3<T>& v) const noexcept {
        return {m[0][0] * v.x + m[1][0] * v.y + m[2][0] * v.z, m[0][1] * v.x + m[1][1] * v.y + m[2][1] * v.z,
                m[0][2] * v.x + m[1][2] * v.y + m[2][2] * v.z};
    }
    tmat3_c operator*(const tmat3_c& b) const noexcept {
        tmat3_c o(UNINIT);
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) o.m[c][r] = m[0][r] * b.m[c][0] + m[1][r] * b.m[c][1] + m[2][r] * b.m[c][2];
        return o;
    }
    tmat3_c transpose() const noexcept {
        tmat3_c o(UNINIT);
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) o.m[c][r] = m[r][c];
        return o;
    }
    T det() const noexcept {
        const auto& a = *this;
        return a(0, 0) * (a(1, 1) * a(2, 2) - a(1, 2) * a(2, 1)) - a(0, 1) * (a(1, 0) * a(2, 2) - a(1, 2) * a(2, 0)) +
               a(0, 2) * (a(1, 0) * a(2, 1) - a(1, 1) * a(2, 0));
    }
    tmat3_c inv() const noexcept {
        const auto& a = *this;
        const T id = T(1) / det();
        tmat3_c o(UNINIT);
        o(0, 0) = (a(1, 1) * a(2, 2) - a(1, 2) * a(2, 1)) * id;
        o(0, 1) = (a(0, 2) * a(2, 1) - a(0, 1) * a(2, 2)) * id;
        o(0, 2) = (a(0, 1) * a(1, 2) - a(0, 2) * a(1, 1)) * id;
        o(1, 0) = (a(1, 2) * a(2, 0) - a(1, 0) * a(2, 2)) * id;
        o(1, 1) = (a(0, 0) * a(2, 2) - a(0, 2) * a(2, 0)) * id;
        o(1, 2) = (a(0, 2) * a(1, 0) - a(0, 0) * a(1, 2)) * id;
        o(2, 0) = (a(1, 0) * a(2, 1) - a(1, 1) * a(2, 0)) * id;
        o(2, 1) = (a(0, 1) * a(2, 0) - a(0, 0) * a(2, 1)) * id;
        o(2, 2) = (a(0, 0) * a(1, 1) - a(0, 1) * a(1, 0)) * id;
        return o;
    }
    static tmat3_c diag(T a, T b, T c) noexcept {
        tmat3_c o;
        o.m[0][0] = a; o.m[1][1] = b; o.m[2][2] = c;
        return o;
    }
    static tmat3_c rotate(const tvec3<T>& axis, T rad) noexcept {
        const tvec3<T> a = axis.normalize();
        const T s = std::sin(rad), c = std::cos(rad), t = T(1) - c;
        return from_rows({t * a.x * a.x + c, t * a.x * a.y - s * a.z, t * a.x * a.z + s * a.y},
                         {t * a.x * a.y + s * a.z, t * a.y * a.y + c, t * a.y * a.z - s * a.x},
                         {t * a.x * a.z - s * a.y, t * a.y * a.z + s * a.x, t * a.z * a.z + c});
    }
};

template <class T>
struct tmat4_c {
    T m[4][4];
    tmat4_c() noexcept { set_identity(); }
    explicit tmat4_c(uninitialized_t) noexcept {}
    T* operator[](int c) noexcept { return m[c]; }  // column c: m[c][r]
    const T* operator[](int c) const noexcept { return m[c]; }
    void set_identity() noexcept {
        for (int c = 0; c < 4; ++c)
            for (int r = 0; r < 4; ++r) m[c][r] = c == r ? T(1) : T(0);
    }
    static tmat4_c from_rows(T m00, T m01, T m02, T m03, T m10, T m11, T m12, T m13, T m20, T m21, T m22, T m23,
                             T m30, T m31, T m32, T m33) noexcept {
        tmat4_c a(UNINIT);
        const T v[16] = {m00, m01, m02, m03, m10, m11, m12, m13, m20, m21, m22, m23, m30, m31, m32, m33};
        for (int r = 0; r < 4; ++r)
            for (int c = 0; c < 4; ++c) a.m[c][r] = v[4 * r + c];
        return a;
    }
    static tmat4_c from_rows(const tvec4<T>& r0, const tvec4<T>& r1, const tvec4<T>& r2, const tvec4<T>& r3) noexcept {
        return from_rows(r0.x, r0.y, r0.z, r0.w, r1.x, r1.y, r1.z, r1.w, r2.x, r2.y, r2.z, r2.w, r3.x, r3.y, r3.z, r3.w);
    }
    T& operator()(int r, int c) noexcept { return m[c][r]; }
    const T& operator()(int r, int c) const noexcept { return m[c][r]; }
    tmat4_c operator*(const tmat4_c& b) const noexcept {
        tmat4_c o(UNINIT);
        for (int r = 0; r < 4; ++r)
            for (int c = 0; c < 4; ++c)
                o.m[c][r] = m[0][r] * b.m[c][0] + m[1][r] * b.m[c][1] + m[2][r] * b.m[c][2] + m[3][r] * b.m[c][3];
        return o;
    }
    tvec4<T> operator*(const tvec4<T>& v) const noexcept {
        tvec4<T> o;
        for (int r = 0; r < 4; ++r) o[r] = m[0][r] * v.x + m[1][r] * v.y + m[2][r] * v.z + m[3][r] * v.w;
        return o;
    }
    tmat4_c transpose() const noexcept {
        tmat4_c o(UNINIT);
        for (int r = 0; r < 4; ++r)
            for (int c = 0; c < 4; ++c) o.m[c][r] = m[r][c];
        return o;
    }
    // general inverse by Gauss-Jordan elimination with partial pivoting
    tmat4_c inv() const noexcept {
        double a[4][8];
        for (int r = 0; r < 4; ++r)
            for (int c = 0; c < 8; ++c) a[r][c] = c < 4 ? double(m[c][r]) : (c - 4 == r ? 1.0 : 0.0);
        for (int col = 0; col < 4; ++col) {
            int piv = col;
            for (int r = col + 1; r < 4; ++r)
                if (std::abs(a[r][col]) > std::abs(a[piv][col])) piv = r;
            for (int c = 0; c < 8; ++c) std::swap(a[col][c], a[piv][c]);
            const double d = a[col][col];
            for (int c = 0; c < 8; ++c) a[col][c] /= d;
            for (int r = 0; r < 4; ++r)
                if (r != col) {
                    const double f = a[r][col];
                    for (int c = 0; c < 8; ++c) a[r][c] -= f * a[col][c];
                }
        }
        tmat4_c o(UNINIT);
        for (int r = 0; r < 4; ++r)
            for (int c = 0; c < 4; ++c) o.m[c][r] = T(a[r][c + 4]);
        return o;
    }

    // Transforms acting on column vectors (p' = M p).
    struct left_transform {
        static tmat4_c translate(const tvec3<T>& o) noexcept {
            return tmat4_c::from_rows(1, 0, 0, o.x, 0, 1, 0, o.y, 0, 0, 1, o.z, 0, 0, 0, 1);
        }
        static tmat4_c translate(T x, T y, T z) noexcept { return translate(tvec3<T>(x, y, z)); }
        static tmat4_c scale(const tvec3<T>& s) noexcept {
            return tmat4_c::from_rows(s.x, 0, 0, 0, 0, s.y, 0, 0, 0, 0, s.z, 0, 0, 0, 0, 1);
        }
        static tmat4_c scale(T x, T y, T z) noexcept { return scale(tvec3<T>(x, y, z)); }
        static tmat4_c rotate(const tvec3<T>& axis, T rad) noexcept {
            const tmat3_c<T> r = tmat3_c<T>::rotate(axis, rad);
            return tmat4_c::from_rows(r(0, 0), r(0, 1), r(0, 2), 0, r(1, 0), r(1, 1), r(1, 2), 0, r(2, 0), r(2, 1),
                                      r(2, 2), 0, 0, 0, 0, 1);
        }
        static tmat4_c rotate_x(T rad) noexcept { return rotate({1, 0, 0}, rad); }
        static tmat4_c rotate_y(T rad) noexcept { return rotate({0, 1, 0}, rad); }
        static tmat4_c rotate_z(T rad) noexcept { return rotate({0, 0, 1}, rad); }
        // world-to-view matrix of a camera at eye looking at dst (the tracer takes its inverse)
        static tmat4_c look_at(const tvec3<T>& eye, const tvec3<T>& dst, const tvec3<T>& up) noexcept {
            const tvec3<T> d = (dst - eye).normalize();
            const tvec3<T> x = cross(up, d).normalize();
            const tvec3<T> y = cross(d, x);
            // world -> view: the view frame has z = forward, x = up x z, y = z x x
            return tmat4_c::from_rows(x.x, x.y, x.z, -dot(x, eye), y.x, y.y, y.z, -dot(y, eye),
                                      d.x, d.y, d.z, -dot(d, eye), 0, 0, 0, 1);
        }
    };
};
using float4x4 = tmat4_c<float>;

// ------------------------------------------------------------- transforms
// Affine 3D transform with its inverse kept beside it.
template <class T>
class ttransform3 {
public:
    tmat4_c<T> mat, inv_mat;
    ttransform3() noexcept = default;
    explicit ttransform3(const tmat4_c<T>& m) noexcept : mat(m), inv_mat(m.inv()) {}
    ttransform3(const tmat4_c<T>& m, const tmat4_c<T>& im) noexcept : mat(m), inv_mat(im) {}
    template <class U>
    explicit ttransform3(const ttransform3<U>& o) noexcept {
        for (int c = 0; c < 4; ++c)
            for (int r = 0; r < 4; ++r) { mat.m[c][r] = T(o.mat.m[c][r]); inv_mat.m[c][r] = T(o.inv_mat.m[c][r]); }
    }
    static ttransform3 translate(const tvec3<T>& o) noexcept { return ttransform3(tmat4_c<T>::left_transform::translate(o)); }
    static ttransform3 translate(T x, T y, T z) noexcept { return translate(tvec3<T>(x, y, z)); }
    static ttransform3 scale(const tvec3<T>& s) noexcept { return ttransform3(tmat4_c<T>::left_transform::scale(s)); }
    static ttransform3 scale(T x, T y, T z) noexcept { return scale(tvec3<T>(x, y, z)); }
    static ttransform3 rotate(const tvec3<T>& axis, T rad) noexcept { return ttransform3(tmat4_c<T>::left_transform::rotate(axis, rad)); }
    static ttransform3 rotate_x(T rad) noexcept { return rotate({1, 0, 0}, rad); }
    static ttransform3 rotate_y(T rad) noexcept { return rotate({0, 1, 0}, rad); }
    static ttransform3 rotate_z(T rad) noexcept { return rotate({0, 0, 1}, rad); }
    ttransform3 operator*(const ttransform3& b) const noexcept { return ttransform3(mat * b.mat, b.inv_mat * inv_mat); }
    ttransform3& operator*=(const ttransform3& b) noexcept { return *this = *this * b; }
    ttransform3 inv() const noexcept { return ttransform3(inv_mat, mat); }
    static tvec3<T> point(const tmat4_c<T>& m, const tvec3<T>& p) noexcept {
        return {m.m[0][0] * p.x + m.m[1][0] * p.y + m.m[2][0] * p.z + m.m[3][0],
                m.m[0][1] * p.x + m.m[1][1] * p.y + m.m[2][1] * p.z + m.m[3][1],
                m.m[0][2] * p.x + m.m[1][2] * p.y + m.m[2][2] * p.z + m.m[3][2]};
    }
    static tvec3<T> vector(const tmat4_c<T>& m, const tvec3<T>& v) noexcept {
        return {m.m[0][0] * v.x + m.m[1][0] * v.y + m.m[2][0] * v.z, m.m[0][1] * v.x + m.m[1][1] * v.y + m.m[2][1] * v.z,
                m.m[0][2] * v.x + m.m[1][2] * v.y + m.m[2][2] * v.z};
    }
    tvec3<T> apply_to_point(const tvec3<T>& p) const noexcept { return point(mat, p); }
    tvec3<T> apply_to_vector(const tvec3<T>& v) const noexcept { return vector(mat, v); }
    // normals: the inverse transpose
    tvec3<T> apply_to_normal(const tvec3<T>& n) const noexcept {
        return {inv_mat.m[0][0] * n.x + inv_mat.m[0][1] * n.y + inv_mat.m[0][2] * n.z,
                inv_mat.m[1][0] * n.x + inv_mat.m[1][1] * n.y + inv_mat.m[1][2] * n.z,
                inv_mat.m[2][0] * n.x + inv_mat.m[2][1] * n.y + inv_mat.m[2][2] * n.z};
    }
    tcoord3<T> apply_to_coord(const tcoord3<T>& c) const noexcept {
        return tcoord3<T>(apply_to_vector(c.x).normalize(), apply_to_vector(c.y).normalize(), apply_to_vector(c.z).normalize());
    }
    tvec3<T> apply_inverse_to_point(const tvec3<T>& p) const noexcept { return point(inv_mat, p); }
    tvec3<T> apply_inverse_to_vector(const tvec3<T>& v) const noexcept { return vector(inv_mat, v); }
    tcoord3<T> apply_inverse_to_coord(const tcoord3<T>& c) const noexcept { return inv().apply_to_coord(c); }
};
using float3_transform = ttransform3<float>;

// Affine 2D transform (3x3 homogeneous, column vectors).
template <class T>
class ttransform2 {
public:
    tmat3_c<T> mat, inv_mat;
    ttransform2() noexcept = default;
    explicit ttransform2(const tmat3_c<T>& m) noexcept : mat(m), inv_mat(m.inv()) {}
    ttransform2(const tmat3_c<T>& m, const tmat3_c<T>& im) noexcept : mat(m), inv_mat(im) {}
    static ttransform2 translate(const tvec2<T>& o) noexcept {
        return ttransform2(tmat3_c<T>::from_rows({1, 0, o.x}, {0, 1, o.y}, {0, 0, 1}));
    }
    static ttransform2 translate(T x, T y) noexcept { return translate(tvec2<T>(x, y)); }
    static ttransform2 scale(const tvec2<T>& s) noexcept {
        return ttransform2(tmat3_c<T>::from_rows({s.x, 0, 0}, {0, s.y, 0}, {0, 0, 1}));
    }
    static ttransform2 scale(T x, T y) noexcept { return scale(tvec2<T>(x, y)); }
    static ttransform2 rotate(T rad) noexcept {
        const T s = std::sin(rad), c = std::cos(rad);
        return ttransform2(tmat3_c<T>::from_rows({c, -s, 0}, {s, c, 0}, {0, 0, 1}));
    }
    ttransform2 operator*(const ttransform2& b) const noexcept { return ttransform2(mat * b.mat, b.inv_mat * inv_mat); }
    ttransform2& operator*=(const ttransform2& b) noexcept { return *this = *this * b; }
    ttransform2 inv() const noexcept { return ttransform2(inv_mat, mat); }
    tvec2<T> apply_to_point(const tvec2<T>& p) const noexcept {
        return {mat.m[0][0] * p.x + mat.m[1][0] * p.y + mat.m[2][0], mat.m[0][1] * p.x + mat.m[1][1] * p.y + mat.m[2][1]};
    }
    tvec2<T> apply_to_vector(const tvec2<T>& v) const noexcept {
        return {mat.m[0][0] * v.x + mat.m[1][0] * v.y, mat.m[0][1] * v.x + mat.m[1][1] * v.y};
    }
};

// ----------------------------------------------------------- distribution
namespace distribution {

// Concentric disk of Shirley and Chiu (1997).
template <class T>
tvec2<T> uniform_on_unit_disk(T u, T v) noexcept {
    const T a = 2 * u - 1, b = 2 * v - 1;
    if (a == 0 && b == 0) return {0, 0};
    T r, phi;
    if (std::abs(a) > std::abs(b)) {
        r = a;
        phi = (PI<T> / 4) * (b / a);
    } else {
        r = b;
        phi = PI<T> / 2 - (PI<T> / 4) * (a / b);
    }
    return {r * std::cos(phi), r * std::sin(phi)};
}

// Malley's method: the concentric disk lifted to the hemisphere.
template <class T>
std::pair<tvec3<T>, T> zweighted_on_hemisphere(T u, T v) noexcept {
    const tvec2<T> d = uniform_on_unit_disk(u, v);
    const T z = std::sqrt((std::max)(T(0), 1 - d.x * d.x - d.y * d.y));
    return {tvec3<T>(d.x, d.y, z), z * invPI<T>};
}
template <class T>
T zweighted_on_hemisphere_pdf(T cos_theta) noexcept { return cos_theta > 0 ? cos_theta * invPI<T> : 0; }

template <class T>
std::pair<tvec3<T>, T> uniform_on_hemisphere(T u, T v) noexcept {
    const T z = u;
    const T r = std::sqrt((std::max)(T(0), 1 - z * z));
    const T phi = 2 * PI<T> * v;
    return {tvec3<T>(r * std::cos(phi), r * std::sin(phi), z), 1 / (2 * PI<T>)};
}

template <class T>
std::pair<tvec3<T>, T> uniform_on_sphere(T u, T v) noexcept {
    const T z = 1 - 2 * u;
    const T r = std::sqrt((std::max)(T(0), 1 - z * z));
    const T phi = 2 * PI<T> * v;
    return {tvec3<T>(r * std::cos(phi), r * std::sin(phi), z), 1 / (4 * PI<T>)};
}
template <class T>
constexpr T uniform_on_sphere_pdf = 1 / (4 * PI<T>);

template <class T>
T uniform_on_cone_pdf(T max_cos_theta) noexcept { return 1 / (2 * PI<T> * (1 - max_cos_theta)); }
template <class T>
std::pair<tvec3<T>, T> uniform_on_cone(T max_cos_theta, T u, T v) noexcept {
    const T cos_t = (1 - u) + u * max_cos_theta;
    const T sin_t = std::sqrt((std::max)(T(0), 1 - cos_t * cos_t));
    const T phi = 2 * PI<T> * v;
    return {tvec3<T>(std::cos(phi) * sin_t, std::sin(phi) * sin_t, cos_t), uniform_on_cone_pdf(max_cos_theta)};
}

// Barycentric coordinates (weights of B and C) uniform on a triangle:
// b0 = 1 - sqrt(u) on A, sqrt(u) v on C.
template <class T>
tvec2<T> uniform_on_triangle(T u, T v) noexcept {
    const T t = std::sqrt(u);
    return {1 - t, t * v};
}
template <class T>
tvec3<T> uniform_on_triangle(const tvec3<T>& a, const tvec3<T>& b, const tvec3<T>& c, T u, T v) noexcept {
    const tvec2<T> bc = uniform_on_triangle(u, v);
    return a * (1 - bc.x - bc.y) + b * bc.x + c * bc.y;
}

template <class T, class I>
std::pair<I, T> extract_uniform_int(T u, I lo, I hi) noexcept {
    // an integer of the half-open [lo, hi) (the callers pass the count as
    // hi) and u's remaining fraction, reusable as a fresh uniform
    const I n = hi - lo;
    const I k = (std::min)(I(u * T(n)), n - 1);
    return {lo + k, u * T(n) - T(k)};
}

template <class I, class T>
I uniform_integer(I lo, I hi, T u) noexcept {
    const I n = hi - lo;
    return lo + (std::min)(I(u * T(n)), n - 1);
}

// Walker's alias table (Vose's construction).
template <class F, class I = int32_t>
class alias_sampler_t {
    std::vector<F> prob_;
    std::vector<I> alias_;

public:
    alias_sampler_t() = default;
    alias_sampler_t(const F* w, I n) { initialize(w, n); }
    void initialize(const F* w, I n) {
        prob_.assign(size_t(n), F(0));
        alias_.assign(size_t(n), I(0));
        double sum = 0;
        for (I i = 0; i < n; ++i) sum += w[i];
        std::vector<double> p(static_cast<size_t>(n));
        std::vector<I> small, large;
        for (I i = 0; i < n; ++i) {
            p[i] = sum > 0 ? double(w[i]) * n / sum : 1.0;
            (p[i] < 1 ? small : large).push_back(i);
        }
        while (!small.empty() && !large.empty()) {
            const I s = small.back();
            small.pop_back();
            const I l = large.back();
            large.pop_back();
            prob_[s] = F(p[s]);
            alias_[s] = l;
            p[l] = (p[l] + p[s]) - 1;
            (p[l] < 1 ? small : large).push_back(l);
        }
        for (I i : large) prob_[i] = F(1);
        for (I i : small) prob_[i] = F(1);
    }
    bool available() const noexcept { return !prob_.empty(); }
    void destroy() {
        prob_.clear();
        alias_.clear();
    }
    I sample(F u) const noexcept {
        const I n = I(prob_.size());
        const F x = u * F(n);
        const I k = (std::min)(I(x), n - 1);
        return (x - F(k)) < prob_[k] ? k : alias_[k];
    }
    I sample(F u1, F u2) const noexcept {
        const I n = I(prob_.size());
        const I k = (std::min)(I(u1 * F(n)), n - 1);
        return u2 < prob_[k] ? k : alias_[k];
    }
};

// Inverse-CDF table lookup with linear interpolation between entries.
template <class T>
T sample_inv_cdf_table(T u, const T* table, size_t n) noexcept {
    const T x = u * T(n - 1);
    const size_t i = (std::min)(size_t(x), n - 2);
    const T t = x - T(i);
    return table[i] * (1 - t) + table[i + 1] * t;
}

}  // namespace distribution
}  // namespace math

// ---------------------------------------------------------------- texture
namespace texture {

// A 2D array of texels, row-major, height rows of width texels.
template <class T>
class texture2d_t {
    int w_ = 0, h_ = 0;
    std::vector<T> d_;

public:
    texture2d_t() = default;
    texture2d_t(int height, int width) { initialize(height, width); }
    texture2d_t(int height, int width, const T& init) { initialize(height, width, init); }
    texture2d_t(int height, int width, const T* data) : w_(width), h_(height), d_(data, data + size_t(width) * height) {}
    void initialize(int height, int width) {
        w_ = width;
        h_ = height;
        std::vector<T>(size_t(width) * height).swap(d_);
    }
    void initialize(int height, int width, const T& init) {
        w_ = width;
        h_ = height;
        d_.assign(size_t(width) * height, init);
    }
    void destroy() {
        w_ = h_ = 0;
        std::vector<T>().swap(d_);
    }
    void clear(const T& v) {
        for (auto& t : d_) t = v;
    }
    std::array<int, 2> shape() const noexcept { return {h_, w_}; }
    T& operator()(const math::vec2i& p) noexcept { return (*this)(p.y, p.x); }
    const T& operator()(const math::vec2i& p) const noexcept { return (*this)(p.y, p.x); }
    bool is_available() const noexcept { return !d_.empty(); }
    int width() const noexcept { return w_; }
    int height() const noexcept { return h_; }
    math::vec2i size() const noexcept { return {w_, h_}; }
    T& operator()(int y, int x) noexcept { return d_[size_t(y) * w_ + x]; }
    const T& operator()(int y, int x) const noexcept { return d_[size_t(y) * w_ + x]; }
    T& at(int y, int x) noexcept { return d_[size_t(y) * w_ + x]; }
    const T& at(int y, int x) const noexcept { return d_[size_t(y) * w_ + x]; }
    T* raw_data() noexcept { return d_.data(); }
    const T* raw_data() const noexcept { return d_.data(); }
    T* data() noexcept { return d_.data(); }
    const T* data() const noexcept { return d_.data(); }
    void swap(texture2d_t& o) noexcept {
        std::swap(w_, o.w_);
        std::swap(h_, o.h_);
        d_.swap(o.d_);
    }
    texture2d_t flip_vertically() const {
        texture2d_t o(h_, w_);
        for (int y = 0; y < h_; ++y)
            for (int x = 0; x < w_; ++x) o(h_ - 1 - y, x) = (*this)(y, x);
        return o;
    }
    template <class F>
    auto map(F&& f) const {
        texture2d_t<std::decay_t<decltype(f(std::declval<const T&>()))>> o(h_, w_);
        for (size_t i = 0; i < d_.size(); ++i) o.raw_data()[i] = f(d_[i]);
        return o;
    }
    texture2d_t& get_data() noexcept { return *this; }
    const texture2d_t& get_data() const noexcept { return *this; }
    texture2d_t subtex(int y0, int y1, int x0, int x1) const {
        texture2d_t o(y1 - y0, x1 - x0);
        for (int y = y0; y < y1; ++y)
            for (int x = x0; x < x1; ++x) o(y - y0, x - x0) = (*this)(y, x);
        return o;
    }
};

template <class A, class B>
auto operator+(const texture2d_t<A>& a, const texture2d_t<B>& b) {
    texture2d_t<std::decay_t<decltype(std::declval<const A&>() + std::declval<const B&>())>> o(a.height(), a.width());
    for (int y = 0; y < a.height(); ++y)
        for (int x = 0; x < a.width(); ++x) o(y, x) = a(y, x) + b(y, x);
    return o;
}
template <class A, class B>
auto operator*(const texture2d_t<A>& a, const texture2d_t<B>& b) {
    texture2d_t<std::decay_t<decltype(std::declval<const A&>() * std::declval<const B&>())>> o(a.height(), a.width());
    for (int y = 0; y < a.height(); ++y)
        for (int x = 0; x < a.width(); ++x) o(y, x) = a(y, x) * b(y, x);
    return o;
}
template <class A, class S, class = std::enable_if_t<std::is_arithmetic_v<S>>>
auto operator*(const texture2d_t<A>& a, S s) {
    return a.map([s](const A& v) { return v * s; });
}
template <class A, class S, class = std::enable_if_t<std::is_arithmetic_v<S>>>
auto operator*(S s, const texture2d_t<A>& a) {
    return a.map([s](const A& v) { return s * v; });
}
template <class A, class B>
texture2d_t<A>& operator+=(texture2d_t<A>& a, const texture2d_t<B>& b) {
    for (int y = 0; y < a.height(); ++y)
        for (int x = 0; x < a.width(); ++x) a(y, x) += b(y, x);
    return a;
}
template <class A, class S, class = std::enable_if_t<std::is_arithmetic_v<S>>>
auto operator/(const texture2d_t<A>& a, S s) {
    return a.map([s](const A& v) { return v / s; });
}

// A 3D array of texels (depth slices of height rows of width texels).
template <class T>
class texture3d_t {
    int w_ = 0, h_ = 0, d_ = 0;
    std::vector<T> t_;

public:
    texture3d_t() = default;
    texture3d_t(int depth, int height, int width) { initialize(depth, height, width); }
    texture3d_t(int depth, int height, int width, const T& init) { initialize(depth, height, width, init); }
    texture3d_t(int depth, int height, int width, const T* data)
        : w_(width), h_(height), d_(depth), t_(data, data + size_t(width) * height * depth) {}
    void initialize(int depth, int height, int width) {
        w_ = width;
        h_ = height;
        d_ = depth;
        std::vector<T>(size_t(width) * height * depth).swap(t_);
    }
    void initialize(int depth, int height, int width, const T& init) {
        w_ = width;
        h_ = height;
        d_ = depth;
        t_.assign(size_t(width) * height * depth, init);
    }
    bool is_available() const noexcept { return !t_.empty(); }
    int width() const noexcept { return w_; }
    int height() const noexcept { return h_; }
    int depth() const noexcept { return d_; }
    math::vec3i size() const noexcept { return {w_, h_, d_}; }
    T& operator()(int z, int y, int x) noexcept { return t_[(size_t(z) * h_ + y) * w_ + x]; }
    const T& operator()(int z, int y, int x) const noexcept { return t_[(size_t(z) * h_ + y) * w_ + x]; }
    T& at(int z, int y, int x) noexcept { return (*this)(z, y, x); }
    const T& at(int z, int y, int x) const noexcept { return (*this)(z, y, x); }
    T* raw_data() noexcept { return t_.data(); }
    const T* raw_data() const noexcept { return t_.data(); }
    T* data() noexcept { return t_.data(); }
    const T* data() const noexcept { return t_.data(); }
    template <class F>
    auto map(F&& f) const {
        texture3d_t<std::decay_t<decltype(f(std::declval<const T&>()))>> o(d_, h_, w_);
        for (size_t i = 0; i < t_.size(); ++i) o.raw_data()[i] = f(t_[i]);
        return o;
    }
};

// Filters over a texel accessor tex(x, y) / tex(x, y, z) (the reference's
// accessors take the column first); uv in [0, 1] maps texel centres to
// (i + 0.5) / n, clamped to the edge texels.
template <class T, class F>
auto nearest_sample2d(const math::tvec2<T>& uv, F&& tex, int width, int height) {
    const int x = math::clamp(int(uv.x * T(width)), 0, width - 1);
    const int y = math::clamp(int(uv.y * T(height)), 0, height - 1);
    return tex(x, y);
}
template <class T, class F>
auto linear_sample2d(const math::tvec2<T>& uv, F&& tex, int width, int height) {
    const T fx = uv.x * T(width) - T(0.5), fy = uv.y * T(height) - T(0.5);
    const T flx = std::floor(fx), fly = std::floor(fy);
    const T ax = fx - flx, ay = fy - fly;
    const int x0 = math::clamp(int(flx), 0, width - 1), x1 = math::clamp(int(flx) + 1, 0, width - 1);
    const int y0 = math::clamp(int(fly), 0, height - 1), y1 = math::clamp(int(fly) + 1, 0, height - 1);
    const auto a = tex(x0, y0) * (T(1) - ax) + tex(x1, y0) * ax;
    const auto b = tex(x0, y1) * (T(1) - ax) + tex(x1, y1) * ax;
    return a * (T(1) - ay) + b * ay;
}
template <class T, class F>
auto nearest_sample3d(const math::tvec3<T>& uvw, F&& tex, int width, int height, int depth) {
    const int x = math::clamp(int(uvw.x * T(width)), 0, width - 1);
    const int y = math::clamp(int(uvw.y * T(height)), 0, height - 1);
    const int z = math::clamp(int(uvw.z * T(depth)), 0, depth - 1);
    return tex(x, y, z);
}
template <class T, class F>
auto linear_sample3d(const math::tvec3<T>& uvw, F&& tex, int width, int height, int depth) {
    const T f[3] = {uvw.x * T(width) - T(0.5), uvw.y * T(height) - T(0.5), uvw.z * T(depth) - T(0.5)};
    const int n[3] = {width, height, depth};
    int i0[3], i1[3];
    T a[3];
    for (int k = 0; k < 3; ++k) {
        const T fl = std::floor(f[k]);
        a[k] = f[k] - fl;
        i0[k] = math::clamp(int(fl), 0, n[k] - 1);
        i1[k] = math::clamp(int(fl) + 1, 0, n[k] - 1);
    }
    auto lx = [&](int z, int y) { return tex(i0[0], y, z) * (T(1) - a[0]) + tex(i1[0], y, z) * a[0]; };
    auto ly = [&](int z) { return lx(z, i0[1]) * (T(1) - a[1]) + lx(z, i1[1]) * a[1]; };
    return ly(i0[2]) * (T(1) - a[2]) + ly(i1[2]) * a[2];
}

}  // namespace texture

// ------------------------------------------------------------------ alloc
namespace alloc {

inline void* aligned_alloc(size_t bytes, size_t align) {
    void* p = nullptr;
    if (posix_memalign(&p, (std::max)(align, sizeof(void*)), (std::max<size_t>)(bytes, 1)) != 0) throw std::bad_alloc();
    return p;
}
inline void aligned_free(void* p) noexcept { std::free(p); }
template <class T>
void call_destructor(T& x) noexcept { x.~T(); }
template <class T>
void call_destructor(T* arr, size_t n) noexcept {
    for (size_t i = 0; i < n; ++i) arr[i].~T();
}

// Bump allocator of objects; release() destroys what create() made.
class obj_arena_t : public misc::uncopyable_t {
    struct Block {
        std::unique_ptr<unsigned char[]> mem;
        size_t size = 0, used = 0;
    };
    struct Dtor {
        void* obj;
        void (*fn)(void*);
    };
    std::vector<Block> blocks_;
    std::vector<Dtor> dtors_;
    size_t used_ = 0;

    void* raw(size_t bytes, size_t align) {
        if (blocks_.empty() || !fits(blocks_.back(), bytes, align)) {
            Block b;
            b.size = (std::max)(size_t(64 * 1024), bytes + align);
            b.mem.reset(new unsigned char[b.size]);
            blocks_.push_back(std::move(b));
        }
        Block& b = blocks_.back();
        size_t off = (reinterpret_cast<uintptr_t>(b.mem.get()) + b.used + align - 1) / align * align -
                     reinterpret_cast<uintptr_t>(b.mem.get());
        b.used = off + bytes;
        used_ += bytes;
        return b.mem.get() + off;
    }
    static bool fits(const Block& b, size_t bytes, size_t align) {
        const size_t off = (reinterpret_cast<uintptr_t>(b.mem.get()) + b.used + align - 1) / align * align -
                           reinterpret_cast<uintptr_t>(b.mem.get());
        return off + bytes <= b.size;
    }

public:
    obj_arena_t() = default;
    obj_arena_t(obj_arena_t&&) noexcept = default;
    ~obj_arena_t() { release(); }
    template <class T, class... Args>
    T* create(Args&&... args) {
        T* p = new (raw(sizeof(T), alignof(T))) T(std::forward<Args>(args)...);
        dtors_.push_back({p, [](void* o) { static_cast<T*>(o)->~T(); }});
        return p;
    }
    template <class T, class... Args>
    T* create_nodestruct(Args&&... args) {
        return new (raw(sizeof(T), alignof(T))) T(std::forward<Args>(args)...);
    }
    void release() {
        for (auto it = dtors_.rbegin(); it != dtors_.rend(); ++it) it->fn(it->obj);
        dtors_.clear();
        if (blocks_.size() > 1) blocks_.erase(blocks_.begin(), blocks_.end() - 1);
        if (!blocks_.empty()) blocks_.back().used = 0;
        used_ = 0;
    }
    size_t used_bytes() const noexcept { return used_; }
};

}  // namespace alloc

// ----------------------------------------------------------------- thread
namespace thread {

// worker_count <= 0: all hardware threads plus worker_count (at least 1)
inline int actual_worker_count(int worker_count) noexcept {
    if (worker_count > 0) return worker_count;
    const int hw = (std::max)(1, int(std::thread::hardware_concurrency()));
    return (std::max)(1, hw + worker_count);
}

// A group of threads: run(count, f) calls f(i) for i in [0, count) on
// count threads and returns when all have finished (the reference's
// parallel grids read their results right after run returns).
class thread_group_t : public misc::uncopyable_t {
public:
    thread_group_t() = default;
    explicit thread_group_t(int) {}
    template <class F>
    void run(int count, F&& f) {
        std::vector<std::thread> ts;
        for (int i = 1; i < count; ++i) ts.emplace_back([&f, i] { f(i); });
        if (count > 0) f(0);
        for (auto& t : ts) t.join();
    }
};

// func(thread_index, i) for i in [begin, end) over worker_count threads.
template <class I, class F>
void parallel_forrange(I begin, I end, F&& func, int worker_count = 0) {
    const int n = actual_worker_count(worker_count);
    std::atomic<I> next{begin};
    std::vector<std::thread> ts;
    for (int k = 0; k < n; ++k)
        ts.emplace_back([&, k] {
            for (;;) {
                const I i = next++;
                if (i >= end) break;
                func(k, i);
            }
        });
    for (auto& t : ts) t.join();
}
template <class I, class F>
void parallel_forrange(I begin, I end, F&& func, thread_group_t&, int worker_count) {
    parallel_forrange(begin, end, std::forward<F>(func), worker_count);
}

}  // namespace thread

// ----------------------------------------------------------------- stdstr
namespace stdstr {

template <class... Ts>
std::string cat(const Ts&... xs) {
    std::ostringstream os;
    (os << ... << xs);
    return os.str();
}
inline bool ends_with(const std::string& s, const std::string& suffix) {
    return s.size() >= suffix.size() && s.compare(s.size() - suffix.size(), suffix.size(), suffix) == 0;
}
inline bool starts_with(const std::string& s, const std::string& prefix) { return s.rfind(prefix, 0) == 0; }
template <class T>
T from_string(const std::string& s) {
    if constexpr (std::is_same_v<T, float>) return std::stof(s);
    else if constexpr (std::is_same_v<T, double>) return std::stod(s);
    else if constexpr (std::is_integral_v<T>) return T(std::stoll(s));
    else return T(s);
}
// Replaces every occurrence in place; returns how many were replaced.
inline size_t replace_(std::string& s, const std::string& from, const std::string& to) {
    if (from.empty()) return 0;
    size_t n = 0;
    for (size_t i = s.find(from); i != std::string::npos; i = s.find(from, i + to.size())) {
        s.replace(i, from.size(), to);
        ++n;
    }
    return n;
}
inline std::string replace(std::string s, const std::string& from, const std::string& to) {
    replace_(s, from, to);
    return s;
}

}  // namespace stdstr

// ------------------------------------------------------------------- file
namespace file {
inline void create_directory_for_file(const std::string& filename) {
    const auto dir = std::filesystem::path(filename).parent_path();
    if (!dir.empty()) std::filesystem::create_directories(dir);
}
inline std::vector<unsigned char> read_binary_file(const std::string& filename) {
    std::ifstream f(filename, std::ios::binary);
    if (!f) throw std::runtime_error("failed to open file: " + filename);
    return std::vector<unsigned char>(std::istreambuf_iterator<char>(f), {});
}
}  // namespace file

namespace sys {
inline void open_with_default_app(const std::string&) {}
}  // namespace sys

// ---------------------------------------------------------------- console
namespace console {
class progress_bar_f_t {
public:
    progress_bar_f_t(int, char) {}
    void set_percent(double) {}
    void display() {}
    void done() {}
    void reset_time() {}
};
}  // namespace console

// ------------------------------------------------------------------- mesh
namespace mesh {

struct vertex_t {
    math::vec3 position;
    math::vec3 normal;
    math::vec2 tex_coord;
};
struct triangle_t {
    vertex_t vertices[3];
};
static_assert(sizeof(triangle_t) == 96, "the .bm layout is 96 bytes per triangle");

std::vector<triangle_t> load_from_file(const std::string& filename);  // _shim_io.cpp

}  // namespace mesh

// -------------------------------------------------------------------- img
namespace img {

// _shim_io.cpp: Radiance .hdr (RLE RGBE), .pfm and 8-bit PNG / PPM readers;
// writers used by post processors (PNG, HDR)
texture::texture2d_t<math::color3f> load_rgb_from_hdr_file(const std::string& filename);
texture::texture2d_t<math::color3b> load_rgb_from_file(const std::string& filename);
texture::texture2d_t<uint8_t> load_gray_from_file(const std::string& filename);
void save_rgb_to_png_file(const std::string& filename, const texture::texture2d_t<math::color3b>& img);
void save_rgb_to_jpg_file(const std::string& filename, const texture::texture2d_t<math::color3b>& img);
void save_rgb_to_hdr_file(const std::string& filename, const texture::texture2d_t<math::color3f>& img);

}  // namespace img

}  // namespace agz
