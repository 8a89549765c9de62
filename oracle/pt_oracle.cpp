// CPU oracle for the `pt` hot path of AirGuanZ/Atrc.
//
// TEST INFRASTRUCTURE ONLY: used by tests/, __graft_entry__.smoke() and the
// CPU-baseline leg of bench.py as the checker / the timed CPU baseline.  The
// product never calls it.  Parity status: pinned to the reference's own
// code built from its sources (see oracle.h).
//
// Every function restates the reference algorithm it names (file:line inside
// the reference checkout, src/tracer/... unless noted).  The small vector
// library is the oracle's own; it uses the conventions documented for the
// missing agz-utils submodule: dot = (x*x' + y*y') + z*z', cross in the usual
// component order, affine rows as ((m0*x + m1*y) + m2*z) + m3, compiled without
// fused multiply-add so that every float operation rounds once, in order.
#include "oracle.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <functional>
#include <memory>
#include <mutex>
#include <queue>
#include <stack>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

namespace {

thread_local std::string g_err;

const float PI = 3.14159265358979323846f;
const float INV_PI = 1.0f / PI;
const float REAL_INF = INFINITY;
const float REAL_MAX = 3.402823466e38f;

// ======================================================================= math
struct V2 {
    float x = 0, y = 0;
    V2() = default;
    V2(float a, float b) : x(a), y(b) {}
};
V2 operator+(V2 a, V2 b) { return {a.x + b.x, a.y + b.y}; }
V2 operator-(V2 a, V2 b) { return {a.x - b.x, a.y - b.y}; }
V2 operator*(float s, V2 a) { return {s * a.x, s * a.y}; }

struct V3 {
    float x = 0, y = 0, z = 0;
    V3() = default;
    explicit V3(float v) : x(v), y(v), z(v) {}
    V3(float a, float b, float c) : x(a), y(b), z(c) {}
    explicit V3(const float* p) : x(p[0]), y(p[1]), z(p[2]) {}
    float operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
    float& operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
    bool black() const { return x == 0 && y == 0 && z == 0; }
};
V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
V3 operator-(V3 a) { return {-a.x, -a.y, -a.z}; }
V3 operator*(V3 a, V3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
V3 operator/(V3 a, V3 b) { return {a.x / b.x, a.y / b.y, a.z / b.z}; }
V3 operator*(float s, V3 a) { return {s * a.x, s * a.y, s * a.z}; }
V3 operator*(V3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
V3 operator/(V3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }
V3& operator+=(V3& a, V3 b) { a = a + b; return a; }
V3& operator*=(V3& a, V3 b) { a = a * b; return a; }
V3& operator*=(V3& a, float s) { a = a * s; return a; }
V3& operator/=(V3& a, float s) { a = a / s; return a; }
float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
V3 cross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
float len2(V3 a) { return dot(a, a); }
float len(V3 a) { return std::sqrt(dot(a, a)); }
V3 normalize(V3 a) { return a * (1.0f / len(a)); }
float cosv(V3 a, V3 b) { return dot(a, b) / (len(a) * len(b)); }
V3 vsqrt(V3 a) { return {std::sqrt(a.x), std::sqrt(a.y), std::sqrt(a.z)}; }
V3 mix(V3 a, V3 b, float t) { return a * (1 - t) + b * t; }
float mixf(float a, float b, float t) { return a * (1 - t) + b * t; }
float sqr(float x) { return x * x; }
float clampf(float x, float lo, float hi) { return std::min(std::max(x, lo), hi); }
// ITU-R BT.709 luminance (agz-utils tcolor3::lum, coefficients documented)
float lum(V3 c) { return 0.2126f * c.x + 0.7152f * c.y + 0.0722f * c.z; }
bool finite3(V3 c) { return std::isfinite(c.x) && std::isfinite(c.y) && std::isfinite(c.z); }

struct Xform {  // row-major 3x4 + inverse
    float m[12], inv[12];
};
V3 xpoint(const float* m, V3 p) {
    return {m[0] * p.x + m[1] * p.y + m[2] * p.z + m[3],
            m[4] * p.x + m[5] * p.y + m[6] * p.z + m[7],
            m[8] * p.x + m[9] * p.y + m[10] * p.z + m[11]};
}
V3 xvec(const float* m, V3 v) {
    return {m[0] * v.x + m[1] * v.y + m[2] * v.z,
            m[4] * v.x + m[5] * v.y + m[6] * v.z,
            m[8] * v.x + m[9] * v.y + m[10] * v.z};
}
Xform to_xform(const AtrcTransform& t) {
    Xform x;
    std::memcpy(x.m, t.m, sizeof(x.m));
    std::memcpy(x.inv, t.inv, sizeof(x.inv));
    return x;
}

// Orthonormal frame (agz-utils tcoord3).
struct Coord {
    V3 x, y, z;
    Coord() : x(1, 0, 0), y(0, 1, 0), z(0, 0, 1) {}
    Coord(V3 a, V3 b, V3 c) : x(a), y(b), z(c) {}
    V3 local_to_global(V3 v) const { return x * v.x + y * v.y + z * v.z; }
    V3 global_to_local(V3 v) const { return {dot(v, x), dot(v, y), dot(v, z)}; }
    bool in_positive_z_hemisphere(V3 v) const { return dot(v, z) > 0; }
    Coord operator-() const { return Coord(-x, -y, -z); }
    // from_z: x from the world axis least aligned with z
    static Coord from_z(V3 zz) {
        V3 z_ = normalize(zz);
        V3 t = std::abs(z_.x) > 0.9f ? V3(0, 1, 0) : V3(1, 0, 0);
        V3 y_ = normalize(cross(z_, t));
        V3 x_ = cross(y_, z_);
        return Coord(x_, y_, z_);
    }
    // rotate_to_new_z: Gram-Schmidt of the old x against the new z
    Coord rotate_to_new_z(V3 nz_) const {
        V3 nz = normalize(nz_);
        V3 nx = x - nz * dot(x, nz);
        float l = len(nx);
        if (!(l > 1e-6f)) return from_z(nz);
        nx = nx / l;
        return Coord(nx, cross(nz, nx), nz);
    }
};
Coord xcoord(const float* m, const Coord& c) {
    return Coord(normalize(xvec(m, c.x)), normalize(xvec(m, c.y)), normalize(xvec(m, c.z)));
}

struct Ray {
    V3 o, d;
    float t_min = 0, t_max = REAL_INF;
    Ray() = default;
    Ray(V3 o_, V3 d_, float a = 0, float b = REAL_INF) : o(o_), d(d_), t_min(a), t_max(b) {}
    V3 at(float t) const { return o + t * d; }
    bool between(float t) const { return t_min <= t && t <= t_max; }  // common.h:320-323
};

// The ray-primitive test of the calling thread's current query batch:
// ATRC_ISECT_EXACT (the reference's) or ATRC_ISECT_WATERTIGHT (not in the
// reference).  In watertight mode the box tests also accept a box whose entry
// distance exceeds its exit distance by a relative 5e-7 (the device's slack):
// the reference's exact box test culls a leaf whose corner the ray passes
// through, so its traversal misses hits that the watertight test finds.
thread_local int g_isect = ATRC_ISECT_EXACT;

inline bool box_overlap(float lo, float hi) {
    return g_isect == ATRC_ISECT_WATERTIGHT ? lo <= hi * 1.0000005f + 1e-30f : lo <= hi;
}

struct AABB {
    V3 low{REAL_MAX}, high{-REAL_MAX};
    void add(V3 p) {
        low = V3(std::min(low.x, p.x), std::min(low.y, p.y), std::min(low.z, p.z));
        high = V3(std::max(high.x, p.x), std::max(high.y, p.y), std::max(high.z, p.z));
    }
    void add(const AABB& b) { add(b.low); add(b.high); }
    // AABB::intersect (common.h:384-395)
    bool intersect(V3 ori, V3 inv_dir, float t_min, float t_max) const {
        V3 n = inv_dir * (low - ori), f = inv_dir * (high - ori);
        float lo = t_min, hi = t_max;
        for (int i = 0; i < 3; ++i) {
            lo = std::max(lo, std::min(n[i], f[i]));
            hi = std::min(hi, std::max(n[i], f[i]));
        }
        return box_overlap(lo, hi);
    }
};

// degenerate-axis widening used by world_bound() (triangle_bvh.cpp:594-599,
// quad.cpp:67-71)
void widen_degenerate(AABB& b) {
    for (int i = 0; i < 3; ++i)
        if (b.low[i] >= b.high[i]) b.low[i] = b.high[i] - 0.1f * std::abs(b.high[i]);
}

// ============================================================ distributions
// agz-utils math::distribution (absent); published mappings:
// concentric disk of Shirley & Chiu (1997), Malley's cosine-weighted
// hemisphere, sqrt-parameterised uniform triangle, uniform sphere / cone.
V2 concentric_disk(float u, float v) {
    float a = 2 * u - 1, b = 2 * v - 1;
    if (a == 0 && b == 0) return {0, 0};
    float r, phi;
    if (std::abs(a) > std::abs(b)) { r = a; phi = (PI / 4) * (b / a); }
    else { r = b; phi = PI / 2 - (PI / 4) * (a / b); }
    return {r * std::cos(phi), r * std::sin(phi)};
}
float zweighted_pdf(float z) { return z > 0 ? z * INV_PI : 0; }
V3 zweighted_on_hemisphere(float u, float v, float* pdf) {
    V2 d = concentric_disk(u, v);
    float z = std::sqrt(std::max(0.0f, 1 - d.x * d.x - d.y * d.y));
    *pdf = z * INV_PI;
    return {d.x, d.y, z};
}
V2 uniform_on_triangle(float u, float v) {
    float t = std::sqrt(u);
    return {1 - t, t * v};
}
V3 uniform_on_sphere(float u, float v, float* pdf) {
    float z = 1 - 2 * u;
    float r = std::sqrt(std::max(0.0f, 1 - z * z));
    float phi = 2 * PI * v;
    *pdf = 1 / (4 * PI);
    return {r * std::cos(phi), r * std::sin(phi), z};
}
float uniform_on_cone_pdf(float cos_max) { return 1 / (2 * PI * (1 - cos_max)); }
V3 uniform_on_cone(float cos_max, float u, float v, float* pdf) {
    float cos_t = (1 - u) + u * cos_max;
    float sin_t = std::sqrt(std::max(0.0f, 1 - cos_t * cos_t));
    float phi = 2 * PI * v;
    *pdf = uniform_on_cone_pdf(cos_max);
    return {std::cos(phi) * sin_t, std::sin(phi) * sin_t, cos_t};
}

// Walker's alias method, Vose's construction.
struct Alias {
    std::vector<float> prob;
    std::vector<int> alias;
    void init(const float* w, int n) {
        prob.assign(n, 0);
        alias.assign(n, 0);
        double sum = 0;
        for (int i = 0; i < n; ++i) sum += w[i];
        std::vector<double> p(n);
        std::vector<int> small, large;
        for (int i = 0; i < n; ++i) {
            p[i] = sum > 0 ? w[i] * n / sum : 1.0;
            (p[i] < 1 ? small : large).push_back(i);
        }
        while (!small.empty() && !large.empty()) {
            int s = small.back(); small.pop_back();
            int l = large.back(); large.pop_back();
            prob[s] = float(p[s]);
            alias[s] = l;
            p[l] = (p[l] + p[s]) - 1;
            (p[l] < 1 ? small : large).push_back(l);
        }
        for (int i : large) { prob[i] = 1; alias[i] = i; }
        for (int i : small) { prob[i] = 1; alias[i] = i; }
    }
    bool available() const { return !prob.empty(); }
    int sample(float u) const {
        int n = int(prob.size());
        float nu = u * n;
        int i = std::min(int(nu), n - 1);
        float frac = nu - float(i);
        return frac < prob[i] ? i : alias[i];
    }
};

// ================================================================== sampler
// pcg32 (O'Neill, PCG-XSH-RR 64/32) + uniform floats in [0, 1)
// (NativeSampler, core/sampler.h:25-121).
struct Sampler {
    uint64_t state = 0, inc = 1;
    Sampler(uint64_t seed, uint64_t stream) {
        inc = (stream << 1u) | 1u;
        state = 0;
        next();
        state += seed;
        next();
    }
    uint32_t next() {
        uint64_t old = state;
        state = old * 6364136223846793005ULL + inc;
        uint32_t xs = uint32_t(((old >> 18u) ^ old) >> 27u);
        uint32_t rot = uint32_t(old >> 59u);
        return (xs >> rot) | (xs << ((-rot) & 31));
    }
    float u() { return float(next() >> 8) * (1.0f / 16777216.0f); }
};

uint64_t mix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

// ============================================================== textures
float wrap_apply(int mode, float x) {  // texture2d.h:62-77
    if (mode == ATRC_WRAP_REPEAT) return clampf(x - std::floor(x), 0, 1);
    if (mode == ATRC_WRAP_MIRROR) {
        const int intp = int(x >= 0 ? x : std::floor(x));
        return clampf((intp & 1) ? 1 - x + intp : x - intp, 0, 1);
    }
    return clampf(x, 0, 1);
}

struct Tex2D {
    AtrcTexture2DDesc d;
    V3 texel(int x, int y) const {
        const float* p = d.data + (size_t(y) * d.width + x) * 3;
        return {p[0], p[1], p[2]};
    }
    // agz-utils linear_sample2d / nearest_sample2d: texel centres at
    // (i + 0.5) / size, edge texels clamped.
    V3 sample_impl(V2 uv) const {
        float u = clampf(uv.x, 0, 1), v = clampf(uv.y, 0, 1);
        if (d.type == ATRC_TEX_CHECKER) {  // CheckerBoard::sample_spectrum_impl (checker_board.cpp:15-22)
            float gs = 1.0f / float(d.grid_count);
            int ui = int(u / gs), vi = int(v / gs);
            return ((ui + vi) & 1) ? V3(d.texel) : V3(d.texel2);
        }
        if (d.nearest) {
            int x = std::min(int(u * d.width), d.width - 1);
            int y = std::min(int(v * d.height), d.height - 1);
            return texel(x, y);
        }
        float fx = u * d.width - 0.5f, fy = v * d.height - 0.5f;
        float flx = std::floor(fx), fly = std::floor(fy);
        int x0 = int(flx), y0 = int(fly);
        float tx = fx - flx, ty = fy - fly;
        int x1 = std::min(x0 + 1, d.width - 1), y1 = std::min(y0 + 1, d.height - 1);
        x0 = std::max(x0, 0); y0 = std::max(y0, 0);
        x1 = std::max(x1, 0); y1 = std::max(y1, 0);
        V3 a = texel(x0, y0) * (1 - tx) + texel(x1, y0) * tx;
        V3 b = texel(x0, y1) * (1 - tx) + texel(x1, y1) * tx;
        return a * (1 - ty) + b * ty;
    }
    // Texture2D::sample_spectrum (texture2d.h:133-145); Constant2D ignores uv
    V3 sample(V2 uv) const {
        if (d.type == ATRC_TEX_CONSTANT) return V3(d.texel);
        const float* m = d.uv_transform;
        V2 t(m[0] * uv.x + m[1] * uv.y + m[2], m[3] * uv.x + m[4] * uv.y + m[5]);
        V2 w(wrap_apply(d.wrap_u, t.x), wrap_apply(d.wrap_v, t.y));
        if (d.type == ATRC_TEX_SOLID) return solid_sample(V3(w.x, w.y, 0));  // solid_image.cpp:12-15
        V3 r = sample_impl(w);
        if (d.inv_gamma != 1) r = V3(std::pow(r.x, d.inv_gamma), std::pow(r.y, d.inv_gamma), std::pow(r.z, d.inv_gamma));
        return r;
    }
    float sample_real(V2 uv) const { return sample(uv).x; }
    // Texture2D::sample_spectrum(inct): a solid image at the world position
    // (solid_image.cpp:25-33), every other texture at uv
    V3 sample_at(V2 uv, V3 pos) const { return d.type == ATRC_TEX_SOLID ? solid_sample(pos) : sample(uv); }
    const struct Tex3D* solid = nullptr;  // the 3D texture of a solid image
    V3 solid_sample(V3 p) const;
};

struct Tex3D {
    AtrcTexture3DDesc d;
    float at(int x, int y, int z, int c) const {
        return d.data[((size_t(z) * d.height + y) * d.width + x) * d.channels + (d.channels == 3 ? c : 0)];
    }
    V3 texel(int x, int y, int z) const { return {at(x, y, z, 0), at(x, y, z, 1), at(x, y, z, 2)}; }
    V3 sample_impl(V3 uvw) const {  // agz-utils linear_sample3d / nearest_sample3d
        float u = clampf(uvw.x, 0, 1), v = clampf(uvw.y, 0, 1), w = clampf(uvw.z, 0, 1);
        if (d.nearest) {
            int x = std::min(int(u * d.width), d.width - 1);
            int y = std::min(int(v * d.height), d.height - 1);
            int z = std::min(int(w * d.depth), d.depth - 1);
            return texel(x, y, z);
        }
        float f[3] = {u * d.width - 0.5f, v * d.height - 0.5f, w * d.depth - 0.5f};
        int size[3] = {d.width, d.height, d.depth};
        int i0[3], i1[3];
        float t[3];
        for (int k = 0; k < 3; ++k) {
            float fl = std::floor(f[k]);
            t[k] = f[k] - fl;
            i0[k] = std::max(int(fl), 0);
            i1[k] = std::max(std::min(int(fl) + 1, size[k] - 1), 0);
            i0[k] = std::min(i0[k], size[k] - 1);
        }
        V3 c00 = texel(i0[0], i0[1], i0[2]) * (1 - t[0]) + texel(i1[0], i0[1], i0[2]) * t[0];
        V3 c10 = texel(i0[0], i1[1], i0[2]) * (1 - t[0]) + texel(i1[0], i1[1], i0[2]) * t[0];
        V3 c01 = texel(i0[0], i0[1], i1[2]) * (1 - t[0]) + texel(i1[0], i0[1], i1[2]) * t[0];
        V3 c11 = texel(i0[0], i1[1], i1[2]) * (1 - t[0]) + texel(i1[0], i1[1], i1[2]) * t[0];
        V3 c0 = c00 * (1 - t[1]) + c10 * t[1];
        V3 c1 = c01 * (1 - t[1]) + c11 * t[1];
        return c0 * (1 - t[2]) + c1 * t[2];
    }
    V3 sample(V3 uvw) const {  // Texture3D::sample_spectrum (texture3d.h)
        if (d.type == ATRC_TEX_CONSTANT) return V3(d.texel);
        V3 p = xpoint(d.uvw_transform, uvw);
        V3 r = sample_impl(V3(wrap_apply(d.wrap[0], p.x), wrap_apply(d.wrap[1], p.y), wrap_apply(d.wrap[2], p.z)));
        if (d.inv_gamma != 1) r = V3(std::pow(r.x, d.inv_gamma), std::pow(r.y, d.inv_gamma), std::pow(r.z, d.inv_gamma));
        return r;
    }
    float sample_real(V3 uvw) const { return sample(uvw).x; }
};
V3 Tex2D::solid_sample(V3 p) const { return solid->sample(p); }

// ============================================================ intersections
struct SurfacePoint {
    V3 pos;
    V2 uv;
    Coord geo, user;
};
struct GeoInct : SurfacePoint {
    float t = -1;
    V3 wr;
    int prim = 0;  // original primitive index (for ray parity reports)
};

float g_eps = 3e-4f;  // common.cpp:7 (EPS(), set_eps)
int g_disney_fixed = 0;  // render option of pt_cuda (not in the reference): sample the Disney diffuse lobe

// triangle_aux.h:9-30
bool has_tri(const Ray& r, V3 A, V3 B_A, V3 C_A) {
    V3 s1 = cross(r.d, C_A);
    float div = dot(s1, B_A);
    if (!div) return false;
    float inv_div = 1 / div;
    V3 o_A = r.o - A;
    float alpha = dot(o_A, s1) * inv_div;
    if (alpha < 0 || alpha > 1) return false;
    V3 s2 = cross(o_A, B_A);
    float beta = dot(r.d, s2) * inv_div;
    if (beta < 0 || alpha + beta > 1) return false;
    float t = dot(C_A, s2) * inv_div;
    return r.between(t);
}
// triangle_aux.h:38-69
bool closest_tri(const Ray& r, V3 A, V3 B_A, V3 C_A, float* t_out, V2* uv) {
    V3 s1 = cross(r.d, C_A);
    float div = dot(s1, B_A);
    if (!div) return false;
    float inv_div = 1 / div;
    V3 o_A = r.o - A;
    float alpha = dot(o_A, s1) * inv_div;
    if (alpha < 0) return false;
    V3 s2 = cross(o_A, B_A);
    float beta = dot(r.d, s2) * inv_div;
    if (beta < 0 || alpha + beta > 1) return false;
    float t = dot(C_A, s2) * inv_div;
    if (!r.between(t)) return false;
    *t_out = t;
    *uv = V2(alpha, beta);
    return true;
}
float triangle_area(V3 B_A, V3 C_A) { return len(cross(B_A, C_A)) / 2; }

// Ray-primitive tests: ATRC_ISECT_EXACT runs the reference's
// Moller-Trumbore above; ATRC_ISECT_WATERTIGHT (g_isect, set per query batch)
// the watertight triangle test of Woop, Benthin and Wald (JCGT 2(1), 2013) on
// the exact vertices and the cancellation-free sphere roots of Haines et al.
// (Ray Tracing Gems, 2019), with the same float operations in the same order
// as the device's watertight mode.

float wt_comp(V3 v, int k) { return k == 0 ? v.x : (k == 1 ? v.y : v.z); }

// Shear the ray onto +z: kz = axis of the largest |d| component, kx, ky
// cyclic after it and swapped when d[kz] < 0 (keeps the winding); then the
// signs of the 2D edge functions of the sheared vertices decide the hit.
// Edge functions that round to 0 are evaluated again in double precision.
bool wt_tri(const Ray& r, V3 pa, V3 pb, V3 pc, float* t_out, V2* uv) {
    const float ax = std::fabs(r.d.x), ay = std::fabs(r.d.y), az = std::fabs(r.d.z);
    const int kz = ax > ay ? (ax > az ? 0 : 2) : (ay > az ? 1 : 2);
    int kx = kz == 2 ? 0 : kz + 1;
    int ky = kx == 2 ? 0 : kx + 1;
    const float dz = wt_comp(r.d, kz);
    if (dz < 0) std::swap(kx, ky);
    const float sx = wt_comp(r.d, kx) / dz, sy = wt_comp(r.d, ky) / dz, sz = 1.0f / dz;
    const V3 A = pa - r.o, B = pb - r.o, C = pc - r.o;
    const float Az = wt_comp(A, kz), Bz = wt_comp(B, kz), Cz = wt_comp(C, kz);
    const float Ax = wt_comp(A, kx) - sx * Az, Ay = wt_comp(A, ky) - sy * Az;
    const float Bx = wt_comp(B, kx) - sx * Bz, By = wt_comp(B, ky) - sy * Bz;
    const float Cx = wt_comp(C, kx) - sx * Cz, Cy = wt_comp(C, ky) - sy * Cz;
    float U = Cx * By - Cy * Bx, V = Ax * Cy - Ay * Cx, W = Bx * Ay - By * Ax;
    if (U == 0.0f || V == 0.0f || W == 0.0f) {
        U = float(double(Cx) * double(By) - double(Cy) * double(Bx));
        V = float(double(Ax) * double(Cy) - double(Ay) * double(Cx));
        W = float(double(Bx) * double(Ay) - double(By) * double(Ax));
    }
    if ((U < 0 || V < 0 || W < 0) && (U > 0 || V > 0 || W > 0)) return false;
    const float det = (U + V) + W;
    if (det == 0.0f) return false;
    const float T = (U * (sz * Az) + V * (sz * Bz)) + W * (sz * Cz);
    const float rcp = 1.0f / det;
    const float t = T * rcp;
    if (!r.between(t)) return false;
    *t_out = t;
    *uv = V2(V * rcp, W * rcp);
    return true;
}

bool tri_has(const Ray& r, V3 A, V3 B_A, V3 C_A, V3 B, V3 C) {
    if (g_isect == ATRC_ISECT_WATERTIGHT) {
        float t;
        V2 uv;
        return wt_tri(r, A, B, C, &t, &uv);
    }
    return has_tri(r, A, B_A, C_A);
}
bool tri_closest(const Ray& r, V3 A, V3 B_A, V3 C_A, V3 B, V3 C, float* t, V2* uv) {
    return g_isect == ATRC_ISECT_WATERTIGHT ? wt_tri(r, A, B, C, t, uv) : closest_tri(r, A, B_A, C_A, t, uv);
}

// Sphere roots: the reference's (sphere_aux.h:53-86), or without
// cancellation in watertight mode.  Returns false when the quadratic has no
// real root.
bool sphere_roots(const Ray& lr, float radius, float* t0, float* t1) {
    if (g_isect == ATRC_ISECT_WATERTIGHT) {
        const float a = len2(lr.d);
        if (!(a > 0)) return false;
        const float b = dot(lr.o, lr.d);
        const V3 l = lr.o - (b / a) * lr.d;
        const float disc = a * (radius * radius - len2(l));
        if (disc < 0) return false;
        const float c = len2(lr.o) - radius * radius;
        const float q = -(b + std::copysign(std::sqrt(disc), b));
        float r0 = q / a, r1 = q != 0.0f ? c / q : r0;
        if (r0 > r1) std::swap(r0, r1);
        *t0 = r0;
        *t1 = r1;
        return true;
    }
    float A = len2(lr.d), B = 2 * dot(lr.d, lr.o), C = len2(lr.o) - radius * radius;
    float delta = B * B - 4 * A * C;
    if (delta < 0) return false;
    delta = std::sqrt(delta);
    float inv2A = 0.5f / A;
    *t0 = (-B - delta) * inv2A;
    *t1 = (-B + delta) * inv2A;
    return true;
}
// triangle_aux.h:76-88
V3 dpdu_as_ex(V3 B_A, V3 C_A, V2 b_a, V2 c_a, V3 nor) {
    float m00 = b_a.x, m01 = b_a.y, m10 = c_a.x, m11 = c_a.y;
    float det = m00 * m11 - m01 * m10;
    if (!det) return Coord::from_z(nor).x;
    float inv_det = 1 / det;
    return normalize(m11 * inv_det * B_A - m01 * inv_det * C_A);
}

// ------------------------------------------------------------ triangle bvh
// UntransformedTriangleBVH (triangle_bvh.cpp:122-529)
struct TriBVH {
    struct Node {
        float low[3], high[3];
        uint32_t start, end_or_right;
        bool is_leaf() const { return start < UINT32_MAX; }
        // Node::has_intersection (triangle_bvh.cpp:75-97)
        bool hit(const float* ori, const float* inv, float t_min, float t_max, float* t) const {
            const float nx = inv[0] * (low[0] - ori[0]), ny = inv[1] * (low[1] - ori[1]), nz = inv[2] * (low[2] - ori[2]);
            const float fx = inv[0] * (high[0] - ori[0]), fy = inv[1] * (high[1] - ori[1]), fz = inv[2] * (high[2] - ori[2]);
            t_min = std::max(t_min, std::min(nx, fx));
            t_min = std::max(t_min, std::min(ny, fy));
            t_min = std::max(t_min, std::min(nz, fz));
            t_max = std::min(t_max, std::max(nx, fx));
            t_max = std::min(t_max, std::max(ny, fy));
            t_max = std::min(t_max, std::max(nz, fz));
            *t = t_min;
            return box_overlap(t_min, t_max);
        }
    };
    struct Prim { V3 a, b_a, c_a, b, c; };  // b, c: exact vertices (watertight test)
    struct Info { V3 n_a, n_b_a, n_c_a; V2 t_a, t_b_a, t_c_a; V3 x, z; };

    std::vector<Node> nodes;
    std::vector<Prim> prims;
    std::vector<Info> info;
    std::vector<uint32_t> orig;  // compacted index -> original triangle index
    Alias sampler;
    float area = 0;
    AABB world_bound;

    struct BVtx { V3 p, n; V2 t; };
    struct BTri { const BVtx* v; V3 centroid; uint32_t index; };
    struct BNode { AABB bound; BNode *l = nullptr, *r = nullptr; uint32_t start = 0, end = 0; };

    void init(const float* verts, size_t count, const Xform& l2w) {
        // TriangleBVH::load (triangle_bvh.cpp:533-558): bake positions and
        // normals into world space
        std::vector<BVtx> vtx(count * 3);
        for (size_t i = 0; i < count * 3; ++i) {
            const float* s = verts + i * 8;
            vtx[i].p = xpoint(l2w.m, V3(s));
            vtx[i].n = xvec(l2w.m, V3(s + 3));
            vtx[i].t = V2(s[6], s[7]);
        }
        std::vector<BTri> tris(count);
        area = 0;
        for (size_t i = 0; i < count; ++i) {
            tris[i].v = &vtx[i * 3];
            tris[i].index = uint32_t(i);
            tris[i].centroid = (vtx[i * 3].p + vtx[i * 3 + 1].p + vtx[i * 3 + 2].p) / 3.0f;
            area += triangle_area(vtx[i * 3 + 1].p - vtx[i * 3].p, vtx[i * 3 + 2].p - vtx[i * 3].p);
        }
        // build_bvh (triangle_bvh.cpp:122-223): BFS, longest centroid axis,
        // midpoint split while depth < 64, median split afterwards, leaf <= 5
        std::vector<std::unique_ptr<BNode>> pool;
        BNode* root = nullptr;
        struct Task { BNode** fill; uint32_t start, end, depth; };
        std::queue<Task> q;
        q.push({&root, 0, uint32_t(count), 0});
        size_t node_count = 0;
        while (!q.empty()) {
            Task task = q.front();
            q.pop();
            AABB all, cen;
            for (uint32_t i = task.start; i < task.end; ++i) {
                all.add(tris[i].v[0].p); all.add(tris[i].v[1].p); all.add(tris[i].v[2].p);
                cen.add(tris[i].centroid);
            }
            const uint32_t n = task.end - task.start;
            pool.push_back(std::make_unique<BNode>());
            BNode* node = pool.back().get();
            node->bound = all;
            *task.fill = node;
            ++node_count;
            if (n <= 5) { node->start = task.start; node->end = task.end; continue; }
            V3 cd = cen.high - cen.low;
            int axis = cd[0] > cd[1] ? (cd[0] > cd[2] ? 0 : 2) : (cd[1] > cd[2] ? 1 : 2);
            uint32_t mid;
            if (task.depth < 64) {
                float split = 0.5f * (cen.high[axis] + cen.low[axis]);
                mid = task.start;
                for (uint32_t i = task.start; i < task.end; ++i)
                    if (tris[i].centroid[axis] < split) std::swap(tris[i], tris[mid++]);
                if (mid == task.start || mid == task.end) mid = task.start + n / 2;
            } else {
                std::sort(tris.begin() + task.start, tris.begin() + task.end,
                          [axis](const BTri& a, const BTri& b) { return a.centroid[axis] < b.centroid[axis]; });
                mid = task.start + n / 2;
            }
            q.push({&node->l, task.start, mid, task.depth + 1});
            q.push({&node->r, mid, task.end, task.depth + 1});
        }
        // compact_bvh (triangle_bvh.cpp:225-304): DFS, left child = idx + 1
        nodes.resize(node_count);
        prims.resize(count);
        info.resize(count);
        orig.resize(count);
        struct CT { const BNode* t; uint32_t* fill; };
        std::stack<CT> st;
        st.push({root, nullptr});
        uint32_t next_node = 0, next_prim = 0;
        while (!st.empty()) {
            CT task = st.top();
            st.pop();
            if (task.fill) *task.fill = next_node;
            const BNode* t = task.t;
            Node& nd = nodes[next_node++];
            for (int k = 0; k < 3; ++k) { nd.low[k] = t->bound.low[k]; nd.high[k] = t->bound.high[k]; }
            if (t->l && t->r) {
                nd.start = UINT32_MAX;
                nd.end_or_right = 0;
                st.push({t->r, &nd.end_or_right});
                st.push({t->l, nullptr});
            } else {
                const uint32_t s = next_prim, e = next_prim + (t->end - t->start);
                nd.start = s;
                nd.end_or_right = e;
                for (uint32_t i = s, j = t->start; i < e; ++i, ++j) {
                    const BTri& tri = tris[j];
                    Prim& p = prims[i];
                    Info& in = info[i];
                    orig[i] = tri.index;
                    p.a = tri.v[0].p;
                    p.b_a = tri.v[1].p - tri.v[0].p;
                    p.c_a = tri.v[2].p - tri.v[0].p;
                    p.b = tri.v[1].p;
                    p.c = tri.v[2].p;
                    V3 na = normalize(tri.v[0].n), nb = normalize(tri.v[1].n), nc = normalize(tri.v[2].n);
                    in.n_a = na; in.n_b_a = nb - na; in.n_c_a = nc - na;
                    in.t_a = tri.v[0].t; in.t_b_a = tri.v[1].t - tri.v[0].t; in.t_c_a = tri.v[2].t - tri.v[0].t;
                    in.z = normalize(cross(p.b_a, p.c_a));
                    if (dot(na + nb + nc, in.z) < 0) in.z = -in.z;
                    in.x = dpdu_as_ex(p.b_a, p.c_a, in.t_b_a, in.t_c_a, in.z);
                }
                next_prim = e;
            }
        }
        std::vector<float> areas(count);
        for (size_t i = 0; i < count; ++i) areas[i] = triangle_area(prims[i].b_a, prims[i].c_a);
        sampler.init(areas.data(), int(count));
        // TriangleBVH ctor world bound (triangle_bvh.cpp:587-599)
        world_bound = AABB();
        for (auto& p : prims) { world_bound.add(p.a); world_bound.add(p.a + p.b_a); world_bound.add(p.a + p.c_a); }
        widen_degenerate(world_bound);
    }

    // has_intersection (triangle_bvh.cpp:363-401)
    bool has(const Ray& r) const {
        const float ori[3] = {r.o.x, r.o.y, r.o.z};
        const float inv[3] = {1 / r.d.x, 1 / r.d.y, 1 / r.d.z};
        float t;
        if (!nodes[0].hit(ori, inv, r.t_min, r.t_max, &t)) return false;
        uint32_t stack[128];
        int top = 0;
        stack[top++] = 0;
        while (top) {
            const uint32_t idx = stack[--top];
            const Node& n = nodes[idx];
            if (n.is_leaf()) {
                for (uint32_t i = n.start; i < n.end_or_right; ++i)
                    if (tri_has(r, prims[i].a, prims[i].b_a, prims[i].c_a, prims[i].b, prims[i].c)) return true;
            } else {
                if (top + 2 > 128) return false;
                if (nodes[idx + 1].hit(ori, inv, r.t_min, r.t_max, &t)) stack[top++] = idx + 1;
                if (nodes[n.end_or_right].hit(ori, inv, r.t_min, r.t_max, &t)) stack[top++] = n.end_or_right;
            }
        }
        return false;
    }

    // closest_intersection (triangle_bvh.cpp:403-488)
    bool closest(Ray r, GeoInct* inct) const {
        const float ori[3] = {r.o.x, r.o.y, r.o.z};
        const float inv[3] = {1 / r.d.x, 1 / r.d.y, 1 / r.d.z};
        float tmp;
        if (!nodes[0].hit(ori, inv, r.t_min, r.t_max, &tmp)) return false;
        uint32_t stack[128];
        int top = 0;
        stack[top++] = 0;
        float best_t = REAL_INF;
        V2 best_uv;
        uint32_t best = 0;
        while (top) {
            const uint32_t idx = stack[--top];
            const Node& n = nodes[idx];
            if (n.is_leaf()) {
                for (uint32_t i = n.start; i < n.end_or_right; ++i) {
                    float t;
                    V2 uv;
                    if (tri_closest(r, prims[i].a, prims[i].b_a, prims[i].c_a, prims[i].b, prims[i].c, &t, &uv)) {
                        best_t = t; best_uv = uv; r.t_max = t; best = i;
                    }
                }
            } else {
                float tl, tr;
                const bool al = nodes[idx + 1].hit(ori, inv, r.t_min, r.t_max, &tl);
                const bool ar = nodes[n.end_or_right].hit(ori, inv, r.t_min, r.t_max, &tr);
                if (top + 2 > 128) break;
                if (al && ar) {
                    if (tl < tr) { stack[top++] = n.end_or_right; stack[top++] = idx + 1; }
                    else { stack[top++] = idx + 1; stack[top++] = n.end_or_right; }
                } else if (al) stack[top++] = idx + 1;
                else if (ar) stack[top++] = n.end_or_right;
            }
        }
        if (std::isinf(best_t)) return false;
        const Info& in = info[best];
        inct->pos = r.at(best_t);
        inct->geo = Coord(in.x, cross(in.z, in.x), in.z);
        inct->uv = in.t_a + best_uv.x * in.t_b_a + best_uv.y * in.t_c_a;
        inct->t = best_t;
        V3 user_z = in.n_a + best_uv.x * in.n_b_a + best_uv.y * in.n_c_a;
        inct->user = inct->geo.rotate_to_new_z(user_z);
        inct->wr = -r.d;
        inct->prim = int(orig[best]);
        return true;
    }

    // sample (triangle_bvh.cpp:497-525)
    SurfacePoint sample(float* pdf, float u, float v, float w) const {
        int idx = sampler.sample(u);
        const Prim& p = prims[idx];
        const Info& in = info[idx];
        V2 uv = uniform_on_triangle(v, w);
        SurfacePoint s;
        s.pos = p.a + uv.x * p.b_a + uv.y * p.c_a;
        s.geo = Coord(in.x, cross(in.z, in.x), in.z);
        s.uv = in.t_a + uv.x * in.t_b_a + uv.y * in.t_c_a;
        V3 user_z = in.n_a + uv.x * in.n_b_a + uv.y * in.n_c_a;
        s.user = s.geo.rotate_to_new_z(user_z);
        *pdf = 1 / area;
        return s;
    }
};

// ----------------------------------------------------------- leaf geometry
struct Leaf {
    int type = 0;
    Xform xf;              // geometry transform
    std::shared_ptr<TriBVH> bvh;
    // quad / triangle (quad.cpp:134-157, triangle.cpp)
    V3 a, b_a, c_a, d_a;
    V3 b, c, d;            // exact vertices (watertight test)
    V2 t_a, t_b_a, t_c_a, t_d_a;
    V3 x_abc, x_acd, z;
    float area = 1, abc_prob = 0;
    float local_to_world_ratio = 1;
    float radius = 1, radius2 = 1, world_radius = 1;
    AABB bound;

    Ray to_local(const Ray& r) const {  // transformed_geometry.h:46-52
        return Ray(xpoint(xf.inv, r.o), xvec(xf.inv, r.d), r.t_min, r.t_max);
    }
    void to_world(SurfacePoint* s) const {
        s->pos = xpoint(xf.m, s->pos);
        s->geo = xcoord(xf.m, s->geo);
        s->user = xcoord(xf.m, s->user);
    }
    void to_world(GeoInct* g) const {
        to_world(static_cast<SurfacePoint*>(g));
        g->wr = xvec(xf.m, g->wr);
    }

    void init(const AtrcGeometryDesc& g, const AtrcSceneDesc& sd) {
        type = g.type;
        xf = to_xform(g.transform);
        local_to_world_ratio = len(xvec(xf.m, V3(1, 0, 0)));
        if (type == ATRC_GEOM_TRIANGLE_BVH) {
            const AtrcMeshDesc& m = sd.meshes[g.mesh];
            bvh = std::make_shared<TriBVH>();
            bvh->init(m.vertices, m.triangle_count, xf);
            bound = bvh->world_bound;
            area = bvh->area;
        } else if (type == ATRC_GEOM_QUAD) {
            // Quad::init_from_params (quad.cpp:134-157): baked into world
            V3 A = xpoint(xf.m, V3(g.p[0])), B = xpoint(xf.m, V3(g.p[1]));
            V3 C = xpoint(xf.m, V3(g.p[2])), D = xpoint(xf.m, V3(g.p[3]));
            a = A; b_a = B - A; c_a = C - A; d_a = D - A;
            b = B; c = C; d = D;
            t_a = V2(g.uv[0][0], g.uv[0][1]);
            t_b_a = V2(g.uv[1][0], g.uv[1][1]) - t_a;
            t_c_a = V2(g.uv[2][0], g.uv[2][1]) - t_a;
            t_d_a = V2(g.uv[3][0], g.uv[3][1]) - t_a;
            z = normalize(cross(b_a, c_a));
            x_abc = dpdu_as_ex(b_a, c_a, t_b_a, t_c_a, z);
            x_acd = dpdu_as_ex(c_a, d_a, t_c_a, t_d_a, z);
            float aabc = triangle_area(b_a, c_a), aacd = triangle_area(c_a, d_a);
            area = aabc + aacd;
            abc_prob = aabc / area;
            bound = AABB();
            bound.add(a); bound.add(a + b_a); bound.add(a + c_a); bound.add(a + d_a);
            widen_degenerate(bound);
        } else if (type == ATRC_GEOM_TRIANGLE) {
            // Triangle (triangle.cpp): local vertices, ray moved to local space
            a = V3(g.p[0]); b_a = V3(g.p[1]) - a; c_a = V3(g.p[2]) - a;
            b = V3(g.p[1]); c = V3(g.p[2]);
            t_a = V2(g.uv[0][0], g.uv[0][1]);
            t_b_a = V2(g.uv[1][0], g.uv[1][1]) - t_a;
            t_c_a = V2(g.uv[2][0], g.uv[2][1]) - t_a;
            z = normalize(cross(b_a, c_a));
            x_abc = dpdu_as_ex(b_a, c_a, t_b_a, t_c_a, z);
            area = triangle_area(xvec(xf.m, b_a), xvec(xf.m, c_a));  // triangle.cpp:121-124
            bound = AABB();
            bound.add(xpoint(xf.m, a)); bound.add(xpoint(xf.m, a + b_a)); bound.add(xpoint(xf.m, a + c_a));
            widen_degenerate(bound);
        } else if (type == ATRC_GEOM_SPHERE) {
            radius = g.radius;
            world_radius = local_to_world_ratio * radius;
            V3 o = xpoint(xf.m, V3(0.0f));
            bound.low = o - V3(world_radius + g_eps);
            bound.high = o + V3(world_radius + g_eps);
            area = 4 * PI * world_radius * world_radius;
        } else if (type == ATRC_GEOM_DISK) {
            radius = g.radius;
            radius2 = radius * radius;
            float vs = std::min(0.1f * radius, 0.01f);
            V3 lo(-radius, -radius, -vs), hi(radius, radius, vs);
            bound = AABB();
            for (int i = 0; i < 8; ++i)
                bound.add(xpoint(xf.m, V3(i & 1 ? hi.x : lo.x, i & 2 ? hi.y : lo.y, i & 4 ? hi.z : lo.z)));
            area = local_to_world_ratio * local_to_world_ratio * PI * radius2;
        }
    }

    bool has(const Ray& r) const {
        switch (type) {
        case ATRC_GEOM_TRIANGLE_BVH: return bvh->has(r);
        case ATRC_GEOM_QUAD: return tri_has(r, a, b_a, c_a, b, c) || tri_has(r, a, c_a, d_a, c, d);
        case ATRC_GEOM_TRIANGLE: return tri_has(to_local(r), a, b_a, c_a, b, c);
        case ATRC_GEOM_SPHERE: {  // sphere_aux.h:53-66
            Ray lr = to_local(r);
            float t0, t1;
            if (!sphere_roots(lr, radius, &t0, &t1)) return false;
            return lr.between(t0) || lr.between(t1);
        }
        case ATRC_GEOM_DISK: {  // disk.cpp:43-55
            Ray lr = to_local(r);
            float t = -lr.o.z / lr.d.z;
            if (std::isinf(t) || !lr.between(t)) return false;
            V3 p = lr.at(t);
            return p.x * p.x + p.y * p.y <= radius2;
        }
        }
        return false;
    }

    static void sphere_uv_coord(V3 p, V2* uv, Coord* c, float radius) {  // sphere_aux.h:19-51
        float phi = (!p.x && !p.y) ? 0.0f : std::atan2(p.y, p.x);
        if (phi < 0) phi += 2 * PI;
        float sin_theta = clampf(p.z / radius, -1, 1);
        float theta = std::asin(sin_theta);
        *uv = V2(0.5f * INV_PI * phi, INV_PI * theta + 0.5f);
        V3 ex, ey, ez = normalize(p);
        if (std::abs(ez.z - 1) < g_eps) { ex = V3(1, 0, 0); ey = V3(0, 1, 0); ez = V3(0, 0, 1); }
        else if (std::abs(ez.z + 1) < g_eps) { ex = V3(0, 1, 0); ey = V3(1, 0, 0); ez = V3(0, 0, -1); }
        else { ex = cross(V3(0, 0, 1), ez); ey = cross(ez, ex); }
        *c = Coord(ex, ey, ez);
    }

    SurfacePoint disk_point(V3 pos, float rad) const {  // disk.cpp:13-30
        float phi = (!pos.y && !pos.x) ? 0.0f : std::atan2(pos.y, pos.x);
        if (phi < 0) phi += 2 * PI;
        SurfacePoint s;
        s.pos = pos;
        s.uv = V2(phi / (2 * PI), rad / radius);
        V3 cx = normalize(V3(pos.x, pos.y, 0)), cz(0, 0, 1);
        s.geo = Coord(cx, cross(cz, cx), cz);
        s.user = s.geo;
        return s;
    }

    bool closest(const Ray& r, GeoInct* inct) const {
        switch (type) {
        case ATRC_GEOM_TRIANGLE_BVH: return bvh->closest(r, inct);
        case ATRC_GEOM_QUAD: {  // quad.cpp:30-58
            float t;
            V2 uv;
            if (tri_closest(r, a, b_a, c_a, b, c, &t, &uv)) {
                inct->pos = r.at(t);
                inct->geo = Coord(x_abc, cross(z, x_abc), z);
                inct->uv = t_a + uv.x * t_b_a + uv.y * t_c_a;
                inct->user = inct->geo;
                inct->wr = -r.d;
                inct->t = t;
                inct->prim = 0;
                return true;
            }
            if (tri_closest(r, a, c_a, d_a, c, d, &t, &uv)) {
                inct->pos = r.at(t);
                inct->geo = Coord(x_acd, cross(z, x_acd), z);
                inct->uv = t_a + uv.x * t_c_a + uv.y * t_d_a;
                inct->user = inct->geo;
                inct->wr = -r.d;
                inct->t = t;
                inct->prim = 1;
                return true;
            }
            return false;
        }
        case ATRC_GEOM_TRIANGLE: {  // triangle.cpp:31-51
            Ray lr = to_local(r);
            float t;
            V2 uv;
            if (!tri_closest(lr, a, b_a, c_a, b, c, &t, &uv)) return false;
            inct->pos = lr.at(t);
            inct->geo = Coord(x_abc, cross(z, x_abc), z);
            inct->uv = t_a + uv.x * t_b_a + uv.y * t_c_a;
            inct->user = inct->geo;
            inct->wr = -lr.d;
            inct->t = t;
            inct->prim = 0;
            to_world(inct);
            return true;
        }
        case ATRC_GEOM_SPHERE: {  // sphere.cpp:35-60, sphere_aux.h:68-86
            Ray lr = to_local(r);
            float t0, t1;
            if (!sphere_roots(lr, radius, &t0, &t1)) return false;
            if (lr.t_max < t0 || t1 < lr.t_min) return false;
            bool not_t0 = t0 < lr.t_min;
            if (not_t0 && t1 > lr.t_max) return false;
            float t = not_t0 ? t1 : t0;
            V3 pos = lr.at(t);
            V2 uv;
            Coord c;
            sphere_uv_coord(pos, &uv, &c, radius);
            inct->pos = pos; inct->geo = c; inct->uv = uv; inct->user = c;
            inct->wr = -lr.d; inct->t = t; inct->prim = 0;
            to_world(inct);
            return true;
        }
        case ATRC_GEOM_DISK: {  // disk.cpp:57-74
            Ray lr = to_local(r);
            float t = -lr.o.z / lr.d.z;
            if (std::isinf(t) || !lr.between(t)) return false;
            V3 pos = lr.at(t);
            float rad = std::sqrt(pos.x * pos.x + pos.y * pos.y);
            if (rad > radius) return false;
            *static_cast<SurfacePoint*>(inct) = disk_point(pos, rad);
            inct->wr = -lr.d; inct->t = t; inct->prim = 0;
            to_world(inct);
            return true;
        }
        }
        return false;
    }

    float surface_area() const { return area; }

    // Geometry::sample(ref, pdf, sam)
    SurfacePoint sample_ref(V3 ref, float* pdf, float u, float v, float w) const {
        switch (type) {
        case ATRC_GEOM_TRIANGLE_BVH: return bvh->sample(pdf, u, v, w);
        case ATRC_GEOM_QUAD: {  // quad.cpp:79-103
            V2 bi = uniform_on_triangle(u, v);
            SurfacePoint s;
            if (w < abc_prob) {
                s.pos = a + bi.x * b_a + bi.y * c_a;
                s.geo = Coord(x_abc, cross(z, x_abc), z);
                s.uv = t_a + bi.x * t_b_a + bi.y * t_c_a;
            } else {
                s.pos = a + bi.x * c_a + bi.y * d_a;
                s.geo = Coord(x_acd, cross(z, x_acd), z);
                s.uv = t_a + bi.x * t_c_a + bi.y * t_d_a;
            }
            s.user = s.geo;
            *pdf = 1 / area;
            return s;
        }
        case ATRC_GEOM_TRIANGLE: {
            V2 bi = uniform_on_triangle(u, v);
            SurfacePoint s;
            s.pos = a + bi.x * b_a + bi.y * c_a;
            s.geo = Coord(x_abc, cross(z, x_abc), z);
            s.uv = t_a + bi.x * t_b_a + bi.y * t_c_a;
            s.user = s.geo;
            to_world(&s);
            *pdf = 1 / area;
            return s;
        }
        case ATRC_GEOM_SPHERE: {  // sphere.cpp:82-133
            V3 local_ref = xpoint(xf.inv, ref);
            float d = len(local_ref);
            SurfacePoint s;
            V2 uv;
            Coord c;
            if (d <= radius) {
                float upd;
                V3 unit = uniform_on_sphere(u, v, &upd);
                *pdf = upd / (world_radius * world_radius);
                V3 pos = radius * unit;
                sphere_uv_coord(pos, &uv, &c, radius);
                s.pos = pos; s.geo = c; s.uv = uv; s.user = c;
                to_world(&s);
                return s;
            }
            float cos_theta = std::min(radius / d, 1.0f);
            float lpdf;
            V3 dir = uniform_on_cone(cos_theta, u, v, &lpdf);
            V3 pos = radius * normalize(Coord::from_z(local_ref).local_to_global(dir));
            sphere_uv_coord(pos, &uv, &c, radius);
            s.pos = pos; s.geo = c; s.uv = uv; s.user = c;
            to_world(&s);
            *pdf = lpdf / (world_radius * world_radius);
            return s;
        }
        case ATRC_GEOM_DISK: {  // disk.cpp:84-95
            V2 dp = concentric_disk(u, v);
            V2 p2 = radius * dp;
            *pdf = 1 / area;
            SurfacePoint s = disk_point(V3(p2.x, p2.y, 0), std::sqrt(p2.x * p2.x + p2.y * p2.y));
            to_world(&s);
            return s;
        }
        }
        *pdf = 0;
        return SurfacePoint();
    }

    // Geometry::pdf(ref, pos)
    float pdf_ref(V3 ref, V3 /*pos*/) const {
        if (type == ATRC_GEOM_SPHERE) {  // sphere.cpp:135-147
            V3 local_ref = xpoint(xf.inv, ref);
            float d = len(local_ref);
            if (d <= radius) return 1 / area;
            float cos_theta = std::min(radius / d, 1.0f);
            return uniform_on_cone_pdf(cos_theta) / (world_radius * world_radius);
        }
        return 1 / area;
    }
};

// ================================================================ entities
struct Entity {
    int index = 0;
    const Leaf* leaf = nullptr;
    bool has_wrap = false;
    Xform wrap;
    float scale_ratio = 1;  // transform_wrapper.cpp:13
    bool double_sided = false;
    int material = 0, med_in = 0, med_out = 0;
    V3 emit;
    bool is_light = false;
    bool no_denoise = false;
    float power = -1;
    AABB bound;

    // chain: TransformWrapper(DoubleSided(leaf)) -- the flip is frame-level and
    // commutes with the wrapper's rigid-plus-uniform-scale transforms
    bool has(const Ray& r) const {
        if (!has_wrap) return leaf->has(r);
        Ray lr(xpoint(wrap.inv, r.o), xvec(wrap.inv, r.d), r.t_min, r.t_max);
        return leaf->has(lr);
    }
    bool closest(const Ray& r, GeoInct* g) const {
        if (!has_wrap) {
            if (!leaf->closest(r, g)) return false;
        } else {  // transform_wrapper.cpp:51-68
            Ray lr(xpoint(wrap.inv, r.o), xvec(wrap.inv, r.d), r.t_min, r.t_max);
            if (!leaf->closest(lr, g)) return false;
            g->pos = xpoint(wrap.m, g->pos);
            g->geo = xcoord(wrap.m, g->geo);
            g->user = xcoord(wrap.m, g->user);
            g->wr = -r.d;
        }
        if (double_sided && dot(g->geo.z, g->wr) < 0) {  // double_sided.cpp:22-36
            g->geo = -g->geo;
            g->user = -g->user;
        }
        return true;
    }
    float surface_area() const {
        float a = leaf->surface_area();
        if (has_wrap) a *= scale_ratio * scale_ratio;
        if (double_sided) a *= 2;
        return a;
    }
    SurfacePoint sample_ref(V3 ref, float* pdf, float u, float v, float w) const {
        bool back = false;
        if (double_sided) {  // double_sided.cpp:58-78
            back = u < 0.5f;
            u = back ? 2 * u : 2 * (u - 0.5f);
        }
        SurfacePoint s;
        if (has_wrap) {  // transform_wrapper.cpp:101-112
            s = leaf->sample_ref(xpoint(wrap.inv, ref), pdf, u, v, w);
            s.pos = xpoint(wrap.m, s.pos);
            s.geo = xcoord(wrap.m, s.geo);
            s.user = xcoord(wrap.m, s.user);
            *pdf /= scale_ratio * scale_ratio;
        } else {
            s = leaf->sample_ref(ref, pdf, u, v, w);
        }
        if (double_sided) {
            *pdf *= 0.5f;
            if (back) { s.geo = -s.geo; s.user = -s.user; }
        }
        return s;
    }
    float pdf_ref(V3 ref, V3 pos) const {
        float p;
        if (has_wrap) p = leaf->pdf_ref(xpoint(wrap.inv, ref), xpoint(wrap.inv, pos)) / (scale_ratio * scale_ratio);
        else p = leaf->pdf_ref(ref, pos);
        if (double_sided) p *= 0.5f;
        return p;
    }

    // GeometryToDiffuseLight (geometry_to_diffuse_light.cpp:14-90)
    bool light_sample(V3 ref, const float* sam, V3* pos, V3* nor, V3* rad, float* pdf) const {
        float pdf_area;
        SurfacePoint s = sample_ref(ref, &pdf_area, sam[0], sam[1], sam[3]);
        if (dot(s.geo.z, ref - s.pos) <= 0) return false;
        V3 to_ref = ref - s.pos;
        float d2 = len2(to_ref);
        *pdf = pdf_area * d2 / std::abs(cosv(s.geo.z, to_ref));
        *pos = s.pos;
        *nor = s.geo.z;
        *rad = emit;
        return true;
    }
    V3 light_radiance(V3 nor, V3 light_to_out) const { return dot(nor, light_to_out) > 0 ? emit : V3(); }
    float light_pdf(V3 ref, V3 pos, V3 nor) const {
        if (dot(nor, ref - pos) <= 0) return 0;
        float area_pdf = pdf_ref(ref, pos);
        V3 to_ref = ref - pos;
        float d2 = len2(to_ref);
        float abscos = std::abs(cosv(nor, to_ref));
        return area_pdf * (d2 / abscos);
    }
};

struct EntInct : GeoInct {
    const Entity* ent = nullptr;
    // intersection.h:52-65
    int wr_medium() const { return dot(wr, geo.z) >= 0 ? ent->med_out : ent->med_in; }
    int medium(V3 d) const { return dot(d, geo.z) >= 0 ? ent->med_out : ent->med_in; }
    V3 eps_offset(V3 d) const {  // intersection.h:17-22
        if (dot(d, geo.z) > 0) return pos + geo.z * g_eps;
        return pos - geo.z * g_eps;
    }
};

// ================================================================== BSDFs
struct BSDFSample {
    V3 dir, f;
    float pdf = 0;
    bool delta = false;
};

struct BSDF {
    int type = ATRC_MAT_IDEAL_BLACK;
    Coord geo, shd;
    V3 albedo_;
    // invisible surface
    V3 geometry_normal;
    // disney (disney.cpp:18-476)
    V3 C, Ctint, specular_scale;
    float metallic = 0, roughness = 0, specular_tint = 0, anisotropic = 0, sheen = 0, sheen_tint = 0;
    float clearcoat = 0, transmission = 0, IOR = 1.5f, transmission_roughness = 0;
    float trans_ax = 0, trans_ay = 0, ax = 0, ay = 0, clearcoat_roughness = 0;
    float w_diffuse = 0.25f, w_specular = 0.25f, w_clearcoat = 0.25f, w_transmission = 0.25f;
    // mirror / metal conductor Fresnel: eta^2, (eta k)^2 per channel, colour
    V3 eta2, etak2, rc;
    // glass (glass.cpp:180-206)
    float glass_ior = 1.5f;
    V3 refl_c, refr_c;
    // phong (phong.cpp:33-79): diffuse / specular colours, exponent, weights
    V3 pd, ps;
    float pns = 1, wd = 0.5f, wsp = 0.5f;
    // exit point of a subsurface walk (SeparableBSDF, separable.cpp:38-103):
    // eta in IOR, sep_ci = 1 - 2 FM1(1 / eta)
    float sep_ci = 1;
    static constexpr int kSeparable = 100;
    V3 separable_eval(V3 wi) const {  // separable.cpp:50-60, any wi
        float fr = dielectric_fresnel(IOR, 1, cosv(wi, geo.z));
        return V3((1 - fr) / (sep_ci * PI) * IOR * IOR);
    }

    // ------------------------------------------------- LocalBSDF helpers
    // core/bsdf.h:113-202
    bool black_fringes(V3 w) const { return shd.in_positive_z_hemisphere(w) != geo.in_positive_z_hemisphere(w); }
    bool black_fringes(V3 a, V3 b) const { return black_fringes(a) || black_fringes(b); }
    V3 eval_black_fringes(V3 in, V3 out) const {
        if (!geo.in_positive_z_hemisphere(in) || !geo.in_positive_z_hemisphere(out)) return V3();
        return albedo_ / PI;
    }
    float normal_corr(V3 wi) const {  // common.h local_angle::normal_corr_factor
        float dem = std::abs(cosv(geo.z, wi));
        return dem < g_eps ? 1 : std::abs(cosv(shd.z, wi) / dem);
    }
    BSDFSample sample_black_fringes(V3 out, const float* sam) const {
        BSDFSample r;
        if (!geo.in_positive_z_hemisphere(out)) return r;
        float pdf;
        V3 lwi = zweighted_on_hemisphere(sam[0], sam[1], &pdf);
        if (pdf < g_eps) return r;
        V3 wi = normalize(geo.local_to_global(lwi));
        r.dir = wi;
        r.f = albedo_ / PI * normal_corr(wi);
        r.pdf = pdf;
        return r;
    }
    float pdf_black_fringes(V3 in, V3 out) const {
        if (geo.in_positive_z_hemisphere(in) != geo.in_positive_z_hemisphere(out)) return 0;
        V3 li = normalize(geo.global_to_local(in));
        return zweighted_pdf(li.z);
    }

    // ------------------------------------------------- disney helpers
    static float one_minus_5(float x) { float t = 1 - x, t2 = t * t; return t2 * t2 * t; }
    static float phi_of(V3 w) {  // local_angle::phi
        if (!w.y && !w.x) return 0;
        float r = std::atan2(w.y, w.x);
        return r < 0 ? r + 2 * PI : r;
    }
    static float cos_2_sin(float c) { return std::sqrt(std::max(0.0f, 1 - c * c)); }
    static float tan_theta(V3 w) { float t = 1 - w.z * w.z; if (t <= 0) return 0; return std::sqrt(t) / w.z; }
    static float dielectric_fresnel(float eta_i, float eta_o, float cos_i) {  // reflection.h:54-72
        if (cos_i < 0) { std::swap(eta_i, eta_o); cos_i = -cos_i; }
        float sin_i = std::sqrt(std::max(0.0f, 1 - cos_i * cos_i));
        float sin_t = eta_o / eta_i * sin_i;
        if (sin_t >= 1) return 1;
        float cos_t = std::sqrt(std::max(0.0f, 1 - sin_t * sin_t));
        float para = (eta_i * cos_i - eta_o * cos_t) / (eta_i * cos_i + eta_o * cos_t);
        float perp = (eta_o * cos_i - eta_i * cos_t) / (eta_o * cos_i + eta_i * cos_t);
        return 0.5f * (para * para + perp * perp);
    }
    static bool refract(V3 w, V3 n, float eta, V3* out) {  // reflection.h:30-46
        float ci = dot(w, n);
        float s2t = sqr(eta) * (1 - sqr(ci));
        float c2t = 1 - s2t;
        if (c2t <= 0) return false;
        float ct = std::sqrt(c2t);
        *out = normalize((eta * ci - ct) * n - eta * w);
        return true;
    }
    // microfacet.cpp:18-128
    static float compute_a(float sp, float cp, float axx, float ayy) { return sqr(cp / axx) + sqr(sp / ayy); }
    static float smith_gtr2(float tan_t, float alpha) {
        if (!tan_t) return 1;
        float root = alpha * tan_t;
        return 2 / (1 + std::sqrt(1 + root * root));
    }
    static float aniso_gtr2(float sp, float cp, float st, float ct, float axx, float ayy) {
        float A = compute_a(sp, cp, axx, ayy);
        float RD = sqr(st) * A + sqr(ct);
        return 1 / (PI * axx * ayy * sqr(RD));
    }
    static float smith_aniso_gtr2(float cp, float sp, float axx, float ayy, float tan_t) {
        float t = sqr(axx * cp) + sqr(ayy * sp);
        float sv = 1 + t * sqr(tan_t);
        float lambda = -0.5f + 0.5f * std::sqrt(sv);
        return 1 / (1 + lambda);
    }
    static V3 sample_aniso_gtr2(float axx, float ayy, float u, float v) {
        float sp = ayy * std::sin(2 * PI * u), cp = axx * std::cos(2 * PI * u);
        float nor = 1 / std::sqrt(sqr(sp) + sqr(cp));
        sp *= nor; cp *= nor;
        float A = compute_a(sp, cp, axx, ayy);
        float ct = std::sqrt(A * (1 - v) / ((1 - A) * v + A));
        float st = std::sqrt(std::max(0.0f, 1 - sqr(ct)));
        return normalize(V3(st * cp, st * sp, ct));
    }
    static float gtr1(float st, float ct, float alpha) {
        float U = sqr(alpha) - 1;
        float LD = 2 * PI * std::log(alpha);
        float RD = sqr(alpha * ct) + sqr(st);
        return U / (LD * RD);
    }
    static V3 sample_gtr1(float alpha, float u, float v) {
        float phi = 2 * PI * u;
        float ct = std::sqrt((std::pow(alpha, 2 - 2 * v) - 1) / (sqr(alpha) - 1));
        float st = cos_2_sin(ct);
        return normalize(V3(st * std::cos(phi), st * std::sin(phi), ct));
    }
    static V3 sample_aniso_gtr2_vnor(V3 ve, float axx, float ayy, float u, float v) {
        V3 vh = normalize(V3(axx * ve.x, ayy * ve.y, ve.z));
        float lensq = vh.x * vh.x + vh.y * vh.y;
        V3 t1 = lensq > g_eps ? V3(-vh.y, vh.x, 0) / std::sqrt(lensq) : V3(1, 0, 0);
        V3 t2 = cross(vh, t1);
        float r = std::sqrt(u);
        float phi = 2 * PI * v;
        float t_1 = r * std::cos(phi), _t_2 = r * std::sin(phi);
        float s = 0.5f * (1 + vh.z);
        float t_2 = (1 - s) * std::sqrt(1 - t_1 * t_1) + s * _t_2;
        V3 nh = t_1 * t1 + t_2 * t2 + std::sqrt(std::max(0.0f, 1 - t_1 * t_1 - t_2 * t_2)) * vh;
        return normalize(V3(axx * nh.x, ayy * nh.y, std::max(0.0f, nh.z)));
    }

    // ConductorPoint::eval (fresnel_point.h:44-64), per channel
    V3 conductor_fresnel(float ci) const {
        if (ci <= 0) return V3();
        float cos2 = ci * ci, sin2 = std::max(0.0f, 1 - cos2);
        float e2[3] = {eta2.x, eta2.y, eta2.z}, k2[3] = {etak2.x, etak2.y, etak2.z}, out[3];
        for (int c = 0; c < 3; ++c) {
            float t0 = e2[c] - k2[c] - sin2;
            float a2b2 = std::sqrt(t0 * t0 + 4 * e2[c] * k2[c]);
            float t1 = a2b2 + cos2;
            float a = std::sqrt(0.5f * (a2b2 + t0));
            float t2 = 2 * ci * a;
            float rs = (t1 - t2) / (t1 + t2);
            float t3 = cos2 * a2b2 + sin2 * sin2;
            float t4 = t2 * sin2;
            float rp = rs * (t3 - t4) / (t3 + t4);
            out[c] = 0.5f * (rp + rs);
        }
        return V3(out[0], out[1], out[2]);
    }
    // GGXMicrofacetReflectionComponent::eval / pdf (microfacet_refl_comp.cpp:9-55)
    void ggx_refl(V3 lwi, V3 lwo, V3* f, float* p) const {
        if (lwi.z <= 0 || lwo.z <= 0) { if (f) *f = V3(); if (p) *p = 0; return; }
        V3 lwh = normalize(lwi + lwo);
        float cd = dot(lwi, lwh);
        float ph = phi_of(lwh), pi_ = phi_of(lwi), po = phi_of(lwo);
        float D = aniso_gtr2(std::sin(ph), std::cos(ph), cos_2_sin(lwh.z), lwh.z, ax, ay);
        float Gi = smith_aniso_gtr2(std::cos(pi_), std::sin(pi_), ax, ay, tan_theta(lwi));
        float Go = smith_aniso_gtr2(std::cos(po), std::sin(po), ax, ay, tan_theta(lwo));
        if (f) *f = rc * conductor_fresnel(cd) * (D * Gi * Go / std::abs(4 * lwi.z * lwo.z));
        if (p) *p = Go * D / (4 * lwo.z);
    }
    // PhongSpecularComponent (phong_specular_comp.cpp:7-96)
    static float pow_cos_pdf(float e, float c) { return (e + 1) / (2 * PI) * std::pow(c, e); }
    V3 phong_spec_eval(V3 lwi, V3 lwo) const {
        if (lwi.z <= 0 || lwo.z <= 0) return V3();
        V3 ideal(-lwo.x, -lwo.y, lwo.z);
        return ps * pow_cos_pdf(pns, cosv(ideal, lwi));
    }
    float phong_spec_pdf(V3 lwi, V3 lwo) const {
        if (lwi.z <= 0 || lwo.z <= 0) return 0;
        V3 ideal(-lwo.x, -lwo.y, lwo.z);
        V3 l = Coord::from_z(ideal).global_to_local(lwi);
        if (l.z <= 0) return 0;
        return pow_cos_pdf(pns, normalize(l).z);
    }
    V3 phong_diffuse(V3 lwi, V3 lwo) const { return (lwi.z <= 0 || lwo.z <= 0) ? V3() : pd / PI; }

    V3 f_diffuse(float ci, float co, float cd) const {
        V3 f_lambert = C / PI;
        float FL = one_minus_5(ci), FV = one_minus_5(co);
        float RR = 2 * roughness * cd * cd;
        V3 retro = C / PI * RR * (FL + FV + FL * FV * (RR - 1));
        return f_lambert * (1 - 0.5f * FL) * (1 - 0.5f * FV) + retro;
    }
    V3 f_sheen(float cd) const { return 4 * sheen * mix(V3(1.0f), Ctint, sheen_tint) * one_minus_5(cd); }
    V3 f_clearcoat(float ci, float co, float ti, float to, float sh, float ch, float cd) const {
        float D = gtr1(sh, ch, clearcoat_roughness);
        float F = 0.04f + (1 - 0.04f) * one_minus_5(cd);
        float G = smith_gtr2(ti, 0.25f) * smith_gtr2(to, 0.25f);
        return V3(clearcoat * D * F * G / std::abs(4 * ci * co));
    }
    V3 f_trans(V3 lwi, V3 lwo) const {
        float ci = lwi.z, co = lwo.z;
        float eta = co > 0 ? IOR : 1 / IOR;
        V3 lwh = normalize(lwo + eta * lwi);
        if (lwh.z < 0) lwh = -lwh;
        float cd = dot(lwo, lwh);
        float F = dielectric_fresnel(IOR, 1, cd);
        float ph = phi_of(lwh), sph = std::sin(ph), cph = std::cos(ph);
        float ch = lwh.z, sh = cos_2_sin(ch);
        float D = aniso_gtr2(sph, cph, sh, ch, trans_ax, trans_ay);
        float pi_ = phi_of(lwi), po = phi_of(lwo);
        float G = smith_aniso_gtr2(std::cos(pi_), std::sin(pi_), trans_ax, trans_ay, tan_theta(lwi))
                * smith_aniso_gtr2(std::cos(po), std::sin(po), trans_ax, trans_ay, tan_theta(lwo));
        float sdem = cd + eta * dot(lwi, lwh);
        float corr = 1 / eta;  // TransMode::Radiance
        float val = (1 - F) * D * G * eta * eta * dot(lwi, lwh) * dot(lwo, lwh) * corr * corr / (ci * co * sdem * sdem);
        float tf = co > 0 ? transmission : 1;
        return (1 - metallic) * tf * vsqrt(C) * std::abs(val);
    }
    V3 f_inner_refl(V3 lwi, V3 lwo) const {
        V3 lwh = -normalize(lwi + lwo);
        float cd = dot(lwo, lwh);
        float F = dielectric_fresnel(IOR, 1, cd);
        float ph = phi_of(lwh), sph = std::sin(ph), cph = std::cos(ph);
        float ch = lwh.z, sh = cos_2_sin(ch);
        float D = aniso_gtr2(sph, cph, sh, ch, trans_ax, trans_ay);
        float pi_ = phi_of(lwi), po = phi_of(lwo);
        float G = smith_aniso_gtr2(std::cos(pi_), std::sin(pi_), trans_ax, trans_ay, tan_theta(lwi))
                * smith_aniso_gtr2(std::cos(po), std::sin(po), trans_ax, trans_ay, tan_theta(lwo));
        return transmission * C * std::abs(F * D * G / (4 * lwi.z * lwo.z));
    }
    V3 f_specular(V3 lwi, V3 lwo) const {
        float ci = lwi.z, co = lwo.z;
        V3 lwh = normalize(lwi + lwo);
        float cd = dot(lwi, lwh);
        V3 Cspec = mix(mix(V3(1.0f), Ctint, specular_tint), C, metallic);
        V3 diel = Cspec * dielectric_fresnel(IOR, 1, cd);
        V3 cond = Cspec + (V3(1.0f) - Cspec) * one_minus_5(cd);
        V3 F = mix(specular_scale * diel, cond, metallic);
        float ph = phi_of(lwh), sph = std::sin(ph), cph = std::cos(ph);
        float ch = lwh.z, sh = cos_2_sin(ch);
        float D = aniso_gtr2(sph, cph, sh, ch, ax, ay);
        float pi_ = phi_of(lwi), po = phi_of(lwo);
        float G = smith_aniso_gtr2(std::cos(pi_), std::sin(pi_), ax, ay, tan_theta(lwi))
                * smith_aniso_gtr2(std::cos(po), std::sin(po), ax, ay, tan_theta(lwo));
        return F * D * G / std::abs(4 * ci * co);
    }
    V3 sample_specular(V3 lwo, float u, float v) const {
        V3 lwh = normalize(sample_aniso_gtr2_vnor(lwo, ax, ay, u, v));
        if (lwh.z <= 0) return V3();
        V3 lwi = normalize(2 * dot(lwo, lwh) * lwh - lwo);
        if (lwi.z <= 0) return V3();
        return lwi;
    }
    V3 sample_clearcoat(V3 lwo, float u, float v) const {
        V3 lwh = sample_gtr1(clearcoat_roughness, u, v);
        if (lwh.z <= 0) return V3();
        V3 lwi = normalize(2 * dot(lwo, lwh) * lwh - lwo);
        if (lwi.z <= 0) return V3();
        return lwi;
    }
    V3 sample_transmission(V3 lwo, float u, float v) const {
        V3 lwh = sample_aniso_gtr2(trans_ax, trans_ay, u, v);
        if (lwh.z <= 0) return V3();
        if ((lwo.z > 0) != (dot(lwh, lwo) > 0)) return V3();
        float eta = lwo.z > 0 ? 1 / IOR : IOR;
        V3 owh = dot(lwh, lwo) > 0 ? lwh : -lwh;
        V3 lwi;
        if (!refract(lwo, owh, eta, &lwi)) return V3();
        lwi = normalize(lwi);
        if (lwi.z * lwo.z > 0 || ((lwi.z > 0) != (dot(lwh, lwi) > 0))) return V3();
        return lwi;
    }
    V3 sample_inner_refl(V3 lwo, float u, float v) const {
        V3 lwh = sample_aniso_gtr2(trans_ax, trans_ay, u, v);
        if (lwh.z <= 0) return V3();
        V3 lwi = 2 * dot(lwo, lwh) * lwh - lwo;
        if (lwi.z > 0) return V3();
        return normalize(lwi);
    }
    void pdf_spec_cc(V3 lwi, V3 lwo, float* ps, float* pc) const {
        V3 lwh = normalize(lwi + lwo);
        float ph = phi_of(lwh), sph = std::sin(ph), cph = std::cos(ph);
        float ch = lwh.z, sh = cos_2_sin(ch);
        float cd = dot(lwi, lwh);
        float cpo = std::cos(phi_of(lwo));
        float spo = cos_2_sin(cpo);
        float to = tan_theta(lwo);
        float sD = aniso_gtr2(sph, cph, sh, ch, ax, ay);
        *ps = smith_aniso_gtr2(cpo, spo, ax, ay, to) * sD / (4 * lwo.z);
        float cD = gtr1(sh, ch, clearcoat_roughness);
        *pc = ch * cD / (4 * cd);
    }
    float pdf_transmission(V3 lwi, V3 lwo) const {
        float eta = lwo.z > 0 ? IOR : 1 / IOR;
        V3 lwh = normalize(lwo + eta * lwi);
        if (lwh.z < 0) lwh = -lwh;
        if (((lwo.z > 0) != (dot(lwh, lwo) > 0)) || ((lwi.z > 0) != (dot(lwh, lwi) > 0))) return 0;
        float sdem = dot(lwo, lwh) + eta * dot(lwi, lwh);
        float dwh_dwi = eta * eta * dot(lwi, lwh) / (sdem * sdem);
        float ph = phi_of(lwh), sph = std::sin(ph), cph = std::cos(ph);
        float ch = lwh.z, sh = cos_2_sin(ch);
        float D = aniso_gtr2(sph, cph, sh, ch, trans_ax, trans_ay);
        return std::abs(ch * D * dwh_dwi);
    }
    float pdf_inner_refl(V3 lwi, V3 lwo) const {
        V3 lwh = -normalize(lwi + lwo);
        float ph = phi_of(lwh), sph = std::sin(ph), cph = std::cos(ph);
        float ch = lwh.z, sh = cos_2_sin(ch);
        float cd = dot(lwi, lwh);
        float D = aniso_gtr2(sph, cph, sh, ch, trans_ax, trans_ay);
        return std::abs(ch * D / (4 * cd));
    }

    void init_disney(V3 base_color, float met, float rough, V3 spec_scale, float spec_tint, float aniso,
                     float sh, float sh_tint, float cc, float cc_gloss, float trans, float trans_rough, float ior) {
        // DisneyBSDF ctor (disney.cpp:404-459)
        C = base_color;
        float l = lum(base_color);
        Ctint = l > 0 ? base_color / l : V3(1.0f);
        metallic = met; roughness = rough; specular_scale = spec_scale; specular_tint = spec_tint;
        anisotropic = aniso; sheen = sh; sheen_tint = sh_tint;
        transmission = trans; transmission_roughness = trans_rough;
        IOR = std::max(1.01f, ior);
        float aspect = aniso > 0 ? std::sqrt(1 - 0.9f * aniso) : 1.0f;
        ax = std::max(0.001f, sqr(rough) / aspect);
        ay = std::max(0.001f, sqr(rough) * aspect);
        trans_ax = std::max(0.001f, sqr(trans_rough) / aspect);
        trans_ay = std::max(0.001f, sqr(trans_rough) * aspect);
        clearcoat = cc;
        clearcoat_roughness = mixf(0.1f, 0.0f, cc_gloss);
        clearcoat_roughness *= clearcoat_roughness;
        clearcoat_roughness = std::max(clearcoat_roughness, 0.0001f);
        float A = clampf(lum(base_color) * (1 - metallic), 0.3f, 0.7f);
        float B = 1 - A;
        w_diffuse = A * (1 - transmission);
        w_transmission = A * transmission;
        w_specular = B * 2 / (2 + clearcoat);
        w_clearcoat = B * clearcoat / (2 + clearcoat);
        albedo_ = C;
    }

    // ------------------------------------------------- interface
    V3 eval(V3 wi, V3 wo) const {
        if (type == kSeparable) return separable_eval(wi);
        switch (type) {
        case ATRC_MAT_IDEAL_DIFFUSE: {  // AggregateBSDF::eval (component/aggregate.h:40-62)
            if (black_fringes(wi, wo)) return eval_black_fringes(wi, wo);
            V3 lwi = normalize(shd.global_to_local(wi)), lwo = normalize(shd.global_to_local(wo));
            if (!lwi.z || !lwo.z) return V3();
            if (lwi.z <= 0 || lwo.z <= 0) return V3();  // DiffuseComponent::eval
            return albedo_ / PI;
        }
        case ATRC_MAT_DISNEY: {  // disney.cpp:461-544
            if (black_fringes(wi, wo)) return eval_black_fringes(wi, wo);
            V3 lwi = normalize(shd.global_to_local(wi)), lwo = normalize(shd.global_to_local(wo));
            if (std::abs(lwi.z) < g_eps || std::abs(lwo.z) < g_eps) return V3();
            if (lwi.z * lwo.z < 0) {
                if (!transmission) return V3();
                return f_trans(lwi, lwo) * normal_corr(wi);
            }
            if (lwi.z < 0 && lwo.z < 0) {
                if (!transmission) return V3();
                return f_inner_refl(lwi, lwo) * normal_corr(wi);
            }
            if (lwi.z <= 0 || lwo.z <= 0) return V3();
            float ci = lwi.z, co = lwo.z;
            V3 lwh = normalize(lwi + lwo);
            float cd = dot(lwi, lwh);
            V3 diffuse, sheen_v;
            if (metallic < 1) {
                diffuse = f_diffuse(ci, co, cd);
                if (sheen > 0) sheen_v = f_sheen(cd);
            }
            V3 specular = f_specular(lwi, lwo);
            V3 cc;
            if (clearcoat > 0) {
                float ti = tan_theta(lwi), to = tan_theta(lwo);
                float ch = lwh.z, sh = cos_2_sin(ch);
                cc = f_clearcoat(ci, co, ti, to, sh, ch, cd);
            }
            V3 value = (1 - metallic) * (1 - transmission) * (diffuse + sheen_v) + specular + cc;
            return value * normal_corr(wi);
        }
        case ATRC_MAT_METAL:
        case ATRC_MAT_PHONG: {  // AggregateBSDF::eval (component/aggregate.h:40-62)
            if (black_fringes(wi, wo)) return eval_black_fringes(wi, wo);
            V3 lwi = normalize(shd.global_to_local(wi)), lwo = normalize(shd.global_to_local(wo));
            if (!lwi.z || !lwo.z) return V3();
            if (type == ATRC_MAT_METAL) { V3 f; ggx_refl(lwi, lwo, &f, nullptr); return f; }
            return phong_diffuse(lwi, lwo) + phong_spec_eval(lwi, lwo);
        }
        default:  // mirror and glass are delta: eval is 0 (mirror.cpp:27-30, glass.cpp:47-50)
            return V3();
        }
    }

    float pdf(V3 wi, V3 wo) const {
        if (type == kSeparable) return zweighted_pdf(normalize(geo.global_to_local(wi)).z);
        switch (type) {
        case ATRC_MAT_IDEAL_DIFFUSE: {  // AggregateBSDF::pdf (component/aggregate.h:200-225)
            if (black_fringes(wi, wo)) return pdf_black_fringes(wi, wo);
            V3 lwi = normalize(shd.global_to_local(wi)), lwo = normalize(shd.global_to_local(wo));
            if (!lwi.z || !lwo.z) return 0;
            if (lwi.z <= 0 || lwo.z <= 0) return 0;
            return zweighted_pdf(lwi.z);
        }
        case ATRC_MAT_DISNEY: {  // disney.cpp:628-660
            if (black_fringes(wi, wo)) return pdf_black_fringes(wi, wo);
            V3 lwi = normalize(shd.global_to_local(wi)), lwo = normalize(shd.global_to_local(wo));
            if (std::abs(lwi.z) < g_eps || std::abs(lwo.z) < g_eps) return 0;
            if (lwo.z < 0) {
                if (!transmission) return 0;
                float mF = clampf(dielectric_fresnel(IOR, 1, lwo.z), 0.1f, 0.9f);
                if (lwi.z > 0) return (1 - mF) * pdf_transmission(lwi, lwo);
                if (!mF) return 0;
                return mF * pdf_inner_refl(lwi, lwo);
            }
            if (lwi.z < 0) return w_transmission * pdf_transmission(lwi, lwo);
            float d = zweighted_pdf(lwi.z);
            float sp, pc;
            pdf_spec_cc(lwi, lwo, &sp, &pc);
            return w_diffuse * d + w_specular * sp + w_clearcoat * pc;
        }
        case ATRC_MAT_METAL:
        case ATRC_MAT_PHONG: {  // AggregateBSDF::pdf (component/aggregate.h:200-225)
            if (black_fringes(wi, wo)) return pdf_black_fringes(wi, wo);
            V3 lwi = normalize(shd.global_to_local(wi)), lwo = normalize(shd.global_to_local(wo));
            if (!lwi.z || !lwo.z) return 0;
            if (type == ATRC_MAT_METAL) { float p; ggx_refl(lwi, lwo, nullptr, &p); return p; }
            float pdd = (lwi.z <= 0 || lwo.z <= 0) ? 0.0f : zweighted_pdf(lwi.z);
            float wsum = wd + wsp;
            return wsum > 0 ? (wd * pdd + wsp * phong_spec_pdf(lwi, lwo)) / wsum : 0.0f;
        }
        default:
            return 0;
        }
    }

    BSDFSample sample(V3 wo, const float* sam) const {
        BSDFSample r;
        if (type == kSeparable) {  // separable.cpp:62-69
            float p;
            V3 lwi = zweighted_on_hemisphere(sam[0], sam[1], &p);
            r.dir = geo.local_to_global(lwi);
            r.f = separable_eval(r.dir);
            r.pdf = p;
            return r;
        }
        switch (type) {
        case ATRC_MAT_IDEAL_DIFFUSE: {  // AggregateBSDF::sample (component/aggregate.h:64-139)
            if (black_fringes(wo)) return sample_black_fringes(wo, sam);
            V3 lwo = normalize(shd.global_to_local(wo));
            if (!lwo.z) return r;
            const float weight_sum = 1;
            float sel = (sam[0] - 0.001f) * weight_sum;
            if (!(sel <= 1)) return r;
            // DiffuseComponent::sample_bidir (diffuse_comp.cpp:28-45)
            if (lwo.z <= 0) return r;
            float pdf;
            V3 lwi = zweighted_on_hemisphere(sam[1], sam[2], &pdf);
            if (pdf < 0.001f) return r;
            lwi = normalize(lwi);
            V3 wi = shd.local_to_global(lwi);
            r.dir = wi;
            r.f = albedo_ / PI * normal_corr(wi);
            r.pdf = pdf * 1.0f;
            return r;
        }
        case ATRC_MAT_DISNEY: {  // disney.cpp:546-612
            if (black_fringes(wo)) return sample_black_fringes(wo, sam);
            V3 lwo = normalize(shd.global_to_local(wo));
            if (std::abs(lwo.z) < g_eps) return r;
            V3 lwi;
            if (lwo.z < 0) {
                if (!transmission) return r;
                float mF = clampf(dielectric_fresnel(IOR, 1, lwo.z), 0.1f, 0.9f);
                if (sam[0] >= mF) lwi = sample_transmission(lwo, sam[1], sam[2]);
                else lwi = sample_inner_refl(lwo, sam[1], sam[2]);
            } else {
                // sampling fall-through of disney.cpp:578-589: the diffuse
                // choice is always overwritten by a later branch
                float sel = sam[0];
                float unused_pdf;
                if (g_disney_fixed && sel < w_diffuse) {
                    // fixed sampling mode (not the reference): the diffuse lobe
                    lwi = zweighted_on_hemisphere(sam[1], sam[2], &unused_pdf);
                    if (lwi.z <= 0) lwi = V3();
                } else {
                    if (sel < w_diffuse) lwi = zweighted_on_hemisphere(sam[1], sam[2], &unused_pdf);
                    else sel -= w_diffuse;
                    if (sel < w_transmission) lwi = sample_transmission(lwo, sam[1], sam[2]);
                    else if (sel -= w_transmission, sel < w_specular) lwi = sample_specular(lwo, sam[1], sam[2]);
                    else lwi = sample_clearcoat(lwo, sam[1], sam[2]);
                }
            }
            if (lwi.black()) { r = BSDFSample(); return r; }
            V3 wi = shd.local_to_global(lwi);
            r.dir = wi;
            r.f = eval(wi, wo);
            r.pdf = pdf(wi, wo);
            r.delta = false;
            return r;
        }
        case ATRC_MAT_MIRROR: {  // MirrorBSDF::sample (mirror.cpp:32-50)
            V3 lo = shd.global_to_local(wo);
            if (lo.z <= 0) return r;
            V3 nwo = normalize(lo);
            V3 dir = shd.local_to_global(V3(0, 0, 2 * nwo.z) - nwo);
            r.dir = dir;
            r.f = conductor_fresnel(nwo.z) * rc / std::abs(nwo.z) * normal_corr(dir);
            r.pdf = 1;
            r.delta = true;
            return r;
        }
        case ATRC_MAT_GLASS: {  // GlassBSDF::sample (glass.cpp:52-91), TransMode::Radiance
            V3 nwo = normalize(shd.global_to_local(wo));
            V3 nor = nwo.z > 0 ? V3(0, 0, 1) : V3(0, 0, -1);
            float fr = dielectric_fresnel(glass_ior, 1, nwo.z);
            r.delta = true;
            if (sam[0] < fr) {
                V3 lwi(-nwo.x, -nwo.y, nwo.z);
                V3 wi = shd.local_to_global(lwi);
                r.dir = wi;
                r.f = refl_c * fr / std::abs(lwi.z) * normal_corr(wi);
                r.pdf = fr;
                return r;
            }
            float eta_i = nwo.z > 0 ? 1 : glass_ior, eta_t = nwo.z > 0 ? glass_ior : 1;
            float eta = eta_i / eta_t;
            float ci = std::abs(nwo.z);
            float st2 = eta * eta * std::max(0.0f, 1 - ci * ci);
            if (st2 >= 1) return BSDFSample();
            float ct = std::sqrt(1 - st2);
            V3 nwi = normalize((eta * ci - ct) * nor - eta * nwo);
            V3 dir = shd.local_to_global(nwi);
            r.dir = dir;
            r.f = eta * eta * refr_c * (1 - fr) / std::abs(nwi.z) * normal_corr(dir);
            r.pdf = 1 - fr;
            return r;
        }
        case ATRC_MAT_METAL:
        case ATRC_MAT_PHONG: {  // AggregateBSDF::sample (component/aggregate.h:64-139)
            if (black_fringes(wo)) return sample_black_fringes(wo, sam);
            V3 lwo = normalize(shd.global_to_local(wo));
            if (!lwo.z) return r;
            bool metal = type == ATRC_MAT_METAL;
            float w0 = metal ? 1.0f : wd, w1 = metal ? 0.0f : wsp;
            float sel = (sam[0] - 0.001f) * (w0 + w1);
            int comp = -1;
            if (sel <= w0) comp = 0;
            else if (!metal && (sel -= w0) <= w1) comp = 1;
            if (comp < 0) return r;
            if (lwo.z <= 0) return r;
            V3 lwi, f;
            float p = 0;
            if (metal) {  // GGXMicrofacetReflectionComponent::sample
                V3 lwh = normalize(sample_aniso_gtr2_vnor(lwo, ax, ay, sam[1], sam[2]));
                if (lwh.z <= 0) return r;
                lwi = normalize(2 * dot(lwo, lwh) * lwh - lwo);
                if (lwi.z <= 0) return r;
                ggx_refl(lwi, lwo, &f, &p);
            } else if (comp == 0) {  // DiffuseComponent::sample_bidir
                lwi = zweighted_on_hemisphere(sam[1], sam[2], &p);
                if (p < 0.001f) return r;
                f = pd / PI;
            } else {  // PhongSpecularComponent::sample
                V3 ideal(-lwo.x, -lwo.y, lwo.z);
                float ct = std::pow(sam[1], 1 / (pns + 1));
                float st = cos_2_sin(ct);
                float phi = 2 * PI * sam[2];
                V3 local = normalize(V3(st * std::cos(phi), st * std::sin(phi), ct));
                lwi = normalize(Coord::from_z(ideal).local_to_global(local));
                if (lwi.z <= 0) return r;
                p = pow_cos_pdf(pns, local.z);
                f = phong_spec_eval(lwi, lwo);
            }
            if (!(p > 0)) return r;
            lwi = normalize(lwi);
            p *= comp == 0 ? w0 : w1;
            if (!metal) {  // the other component's contribution
                if (comp == 0) { f += phong_spec_eval(lwi, lwo); p += phong_spec_pdf(lwi, lwo) * w1; }
                else {
                    f += phong_diffuse(lwi, lwo);
                    p += ((lwi.z <= 0 || lwo.z <= 0) ? 0.0f : zweighted_pdf(lwi.z)) * w0;
                }
            }
            V3 wi = shd.local_to_global(lwi);
            r.dir = wi;
            r.f = f * normal_corr(wi);
            r.pdf = p;
            return r;
        }
        case ATRC_MAT_INVISIBLE_SURFACE: {  // invisible_surface.cpp:22-28
            float c = std::abs(cosv(geometry_normal, wo));
            r.dir = -wo;
            r.f = V3(1.0f) / (c < g_eps ? 1 : c);
            r.pdf = 1;
            r.delta = true;
            return r;
        }
        default:
            return r;
        }
    }

    V3 albedo() const {
        if (type == ATRC_MAT_INVISIBLE_SURFACE) return V3(1.0f);
        if (type == ATRC_MAT_IDEAL_BLACK || type == kSeparable) return V3();
        return albedo_;
    }
};

// Henyey-Greenstein phase function (utility/phase_function.h:8-90)
struct Phase {
    float g = 0;
    V3 albedo;
    float func(float u) const {
        float g2 = g * g;
        float dem = 1 + g2 - 2 * g * u;
        return (1 - g2) / (4 * PI * dem * std::sqrt(dem));
    }
    V3 eval(V3 wi, V3 wo) const { return V3(func(-cosv(wi, wo))); }
    float pdf(V3 wi, V3 wo) const { return func(-cosv(wi, wo)); }
    BSDFSample sample(V3 wo, const float* sam) const {
        float s = 2 * sam[0] - 1;
        float u;
        if (std::abs(g) < 0.001f) u = s;
        else { float g2 = g * g; u = (1 + g2 - sqr((1 - g2) / (1 + g * s))) / (2 * g); }
        float ct = -u;
        float st = BSDF::cos_2_sin(ct);
        float phi = 2 * PI * sam[1];
        V3 lwi(st * std::sin(phi), st * std::cos(phi), ct);
        float pv = func(u);
        BSDFSample r;
        r.dir = Coord::from_z(wo).local_to_global(lwi);
        r.f = V3(pv);
        r.pdf = pv;
        return r;
    }
};

// ============================================================= environment
struct EnvSampler {  // envir_light/env_sampler.h:15-169
    int w = 0, h = 0;
    std::vector<float> probs;
    Alias alias;
    void init(const std::function<V3(V2)>& tex, int tw, int th) {
        w = std::min(tw, 200);
        h = std::min(th, 200);
        probs.assign(size_t(w) * h, 0);
        double lum_sum = 0;
        for (int y = 0; y < h; ++y) {
            float y0 = float(y) / h, y1 = float(y + 1) / h;
            int ys0 = std::max(0, int(std::floor(y0 * th) - 1));
            int ys1 = std::min(th - 1, int(std::floor(y1 * th) + 1));
            for (int x = 0; x < w; ++x) {
                float x0 = float(x) / w, x1 = float(x + 1) / w;
                int xs0 = std::max(0, int(std::floor(x0 * tw) - 1));
                int xs1 = std::min(tw - 1, int(std::floor(x1 * tw) + 1));
                float pl = 0;
                for (int ys = ys0; ys <= ys1; ++ys)
                    for (int xs = xs0; xs <= xs1; ++xs)
                        pl += lum(tex(V2((xs + 0.5f) / tw, (ys + 0.5f) / th)));
                float da = std::abs(2 * PI * (x1 - x0) * (std::cos(PI * y1) - std::cos(PI * y0)));
                probs[size_t(y) * w + x] = pl * da;
                lum_sum += pl * da;
            }
        }
        if (lum_sum > g_eps) {
            float ratio = float(1 / lum_sum);
            for (auto& p : probs) p *= ratio;
        }
        alias.init(probs.data(), int(probs.size()));
    }
    V3 sample(float u, float v, float ww, float* pdf) const {
        int idx = alias.sample(u);
        int py = idx / w, px = idx % w;
        float pp = probs[idx];
        float u0 = float(px) / w, u1 = float(px + 1) / w;
        float v0 = float(py) / h, v1 = float(py + 1) / h;
        float a = std::cos(PI * v1), b = std::cos(PI * v0);
        float cmin = std::min(a, b), cmax = std::max(a, b);
        float ct = cmin + ww * (cmax - cmin);
        float st = BSDF::cos_2_sin(ct);
        float uu = mixf(u0, u1, v);
        float phi = 2 * PI * uu;
        *pdf = pp * (1 / (2 * PI * ((u1 - u0) * (cmax - cmin))));
        return V3(st * std::cos(phi), st * std::sin(phi), ct);
    }
    float pdf(V3 d) const {
        V3 dir = normalize(d);
        float theta = std::acos(dir.z);
        float phi = BSDF::phi_of(dir);
        float u = phi / (2 * PI), v = theta / PI;
        int px = std::min(std::max(int(std::floor(u * w)), 0), w - 1);
        int py = std::min(std::max(int(std::floor(v * h)), 0), h - 1);
        float pp = probs[size_t(py) * w + px];
        float u0 = float(px) / w, u1 = float(px + 1) / w;
        float v0 = float(py) / h, v1 = float(py + 1) / h;
        float a = std::cos(PI * v1), b = std::cos(PI * v0);
        float cmin = std::min(a, b), cmax = std::max(a, b);
        return pp * (1 / (2 * PI * ((u1 - u0) * (cmax - cmin))));
    }
};

struct Env {
    int type = ATRC_ENV_NONE;
    const Tex2D* tex = nullptr;
    EnvSampler sampler;
    V3 top, bottom;
    V3 centre;
    float radius = 1;

    V3 radiance(V3 d) const {
        if (type == ATRC_ENV_NATIVE_SKY) {  // native_sky.cpp:13-19
            float ct = clampf(normalize(d).z, -1, 1);
            float s = (ct + 1) / 2;
            return s * top + (1 - s) * bottom;
        }
        V3 dir = normalize(d);  // ibl.cpp:146-155
        float phi = BSDF::phi_of(dir);
        float theta = std::acos(clampf(dir.z, -1, 1));
        float u = clampf(phi / (2 * PI), 0, 1), v = clampf(theta / PI, 0, 1);
        return tex->sample(V2(u, v));
    }
    float pdf(V3 d) const {
        if (type == ATRC_ENV_NATIVE_SKY) return 1 / (4 * PI);
        return sampler.pdf(d);
    }
    V3 sample_dir(const float* sam, float* pdf) const {
        if (type == ATRC_ENV_NATIVE_SKY) return uniform_on_sphere(sam[0], sam[1], pdf);
        return sampler.sample(sam[0], sam[1], sam[2], pdf);
    }
    // emit_pos (ibl.cpp:103-131): point on the plane tangent to the enlarged
    // world sphere that the ray ref + t*d meets
    V3 emit_pos(V3 ref, V3 ref_to_light) const {
        Coord c = Coord::from_z(ref_to_light);
        V3 a = radius * c.x, b = radius * c.y, cc = -c.z;
        V3 m = ref - centre - radius * c.z;
        float D0 = a[1] * b[2] - a[2] * b[1];
        float D1 = a[0] * b[2] - a[2] * b[0];
        float D2 = a[0] * b[1] - a[1] * b[0];
        float det = cc[0] * D0 - cc[1] * D1 + cc[2] * D2;
        float tdet = m[0] * D0 - m[1] * D1 + m[2] * D2;
        float t = tdet / det;
        return ref + t * c.z;
    }
};

// ================================================================== media
struct Medium {
    int type = ATRC_MED_VOID;
    V3 sa, ss, st;
    float g = 0;
    int max_scat = INT32_MAX;
    Xform xf;
    const Tex3D *density = nullptr, *albedo = nullptr, *gtex = nullptr;
    float max_density = 1, inv_max_density = 1;
    bool white_for_indirect = false;

    V3 tr(V3 a, V3 b, Sampler& s) const {
        if (type == ATRC_MED_HOMOGENEOUS) {  // homogeneous.cpp:44-53
            V3 e = -1.0f * st * len(a - b);
            return V3(std::exp(e.x), std::exp(e.y), std::exp(e.z));
        }
        if (type == ATRC_MED_HETEROGENEOUS) {  // heterogeneous.cpp:52-74 (ratio tracking)
            float result = 1, t = 0;
            const float t_max = len(a - b);
            for (int it = 0; it < 1 << 20; ++it) {
                float dt = -std::log(1 - s.u()) * inv_max_density;
                t += dt;
                if (t >= t_max) break;
                V3 pos = a + (b - a) * (t / t_max);
                float dens = density->sample_real(xpoint(xf.inv, pos));
                result *= 1 - dens / max_density;
            }
            return V3(result);
        }
        return V3(1.0f);
    }
    V3 ab(V3 a, V3 b, Sampler& s) const {
        if (type == ATRC_MED_HOMOGENEOUS) {
            V3 e = -1.0f * sa * len(a - b);
            return V3(std::exp(e.x), std::exp(e.y), std::exp(e.z));
        }
        return tr(a, b, s);  // heterogeneous.cpp:76-81
    }
    // returns true if a scattering event happened
    bool sample_scattering(V3 a, V3 b, Sampler& s, bool indirect, V3* throughput, V3* pos, V3* wr, Phase* ph) const {
        if (type == ATRC_MED_HOMOGENEOUS) {  // homogeneous.cpp:66-109
            const float u = s.u();
            if (ss.black()) { *throughput = tr(a, b, s); return false; }
            const float t_max = len(b - a);
            // extract_uniform_int(u, 0, 3): channel = floor(3u), remaining
            // uniform = 3u - channel
            int ch = std::min(int(u * 3), 2);
            float nu = u * 3 - ch;
            float sampled = -std::log(nu) / st[ch];
            bool in_medium = sampled < t_max;
            V3 trv;
            for (int i = 0; i < 3; ++i) trv[i] = std::exp(-st[i] * std::min(sampled, t_max));
            V3 dens = in_medium ? st * trv : trv;
            float pdf = (dens.x + dens.y + dens.z) / 3;
            pdf = std::max(pdf, g_eps);
            V3 tp = trv / pdf;
            if (in_medium) tp = tp * ss;
            *throughput = tp;
            if (in_medium) {
                *pos = a + (b - a) * (sampled / t_max);
                *wr = (a - b) / t_max;
                ph->g = g;
                ph->albedo = st.black() ? V3(1.0f) : ss / st;
                return true;
            }
            return false;
        }
        if (type == ATRC_MED_HETEROGENEOUS) {  // heterogeneous.cpp:83-123 (delta tracking)
            const float t_max = len(b - a);
            float t = 0;
            for (int it = 0; it < 1 << 20; ++it) {
                float dt = -std::log(1 - s.u()) * inv_max_density;
                t += dt;
                if (t >= t_max) break;
                V3 p = a + (b - a) * (t / t_max);
                V3 unit = xpoint(xf.inv, p);
                float dens = density->sample_real(unit);
                if (s.u() < dens / max_density) {
                    V3 alb = white_for_indirect && indirect ? V3(1.0f) : albedo->sample(unit);
                    float gg = gtex->sample_real(unit);
                    *pos = p;
                    *wr = (a - b) / t_max;
                    ph->g = gg;
                    ph->albedo = alb;
                    *throughput = alb;
                    return true;
                }
            }
            *throughput = V3(1.0f);
            return false;
        }
        *throughput = V3(1.0f);
        return false;
    }
};

// ==================================================================== scene
struct Light {
    bool is_env = false;
    const Entity* ent = nullptr;
};

struct EntityBVHNode {
    AABB bound;
    bool leaf = false;
    size_t a = 0, b = 0;  // leaf: [start, end); interior: left, right
};

}  // namespace

struct OracleScene {
    std::vector<Leaf> leaves;
    std::vector<Entity> entities;
    std::vector<Tex2D> tex2d;
    std::vector<Tex3D> tex3d;
    std::vector<AtrcMaterialDesc> materials;
    std::vector<Medium> media;
    Env env;
    std::vector<Light> lights;
    int aggregate = ATRC_AGG_NATIVE;
    int max_leaf = 5;
    std::vector<EntityBVHNode> nodes;
    std::vector<const Entity*> prims;
    float eps = 3e-4f;

    // EntityBVH::build_aux (entity_bvh.cpp:46-116)
    size_t build_aux(std::vector<std::pair<const Entity*, AABB>>& recs, size_t begin, size_t count) {
        if (count <= size_t(max_leaf) || count < 2) {
            size_t start = prims.size();
            AABB bound;
            for (size_t i = 0; i < count; ++i) { prims.push_back(recs[begin + i].first); bound.add(recs[begin + i].second); }
            nodes.push_back({bound, true, start, start + count});
            return nodes.size() - 1;
        }
        AABB all;
        for (size_t i = 0; i < count; ++i) all.add(recs[begin + i].second);
        float best = -1;
        int axis = 0;
        for (int i = 0; i < 3; ++i) {
            float l = all.high[i] - all.low[i];
            if (l > best) { best = l; axis = i; }
        }
        std::sort(recs.begin() + begin, recs.begin() + begin + count, [axis](const auto& l, const auto& r) {
            return l.second.low[axis] + l.second.high[axis] < r.second.low[axis] + r.second.high[axis];
        });
        size_t idx = nodes.size();
        nodes.push_back({});
        size_t split = count / 2;
        size_t l = build_aux(recs, begin, split);
        size_t r = build_aux(recs, begin + split, count - split);
        nodes[idx] = {all, false, l, r};
        return idx;
    }

    bool has_aux(V3 inv, const Ray& r, size_t ni) const {  // entity_bvh.cpp:118-139
        const EntityBVHNode& n = nodes[ni];
        if (!n.bound.intersect(r.o, inv, r.t_min, r.t_max)) return false;
        if (n.leaf) {
            for (size_t i = n.a; i < n.b; ++i) if (prims[i]->has(r)) return true;
            return false;
        }
        return has_aux(inv, r, n.a) || has_aux(inv, r, n.b);
    }
    bool closest_aux(V3 inv, Ray& r, size_t ni, EntInct* inct) const {  // entity_bvh.cpp:141-172
        const EntityBVHNode& n = nodes[ni];
        if (!n.bound.intersect(r.o, inv, r.t_min, r.t_max)) return false;
        if (n.leaf) {
            bool ret = false;
            for (size_t i = n.a; i < n.b; ++i) {
                if (prims[i]->closest(r, inct)) { inct->ent = prims[i]; r.t_max = inct->t; ret = true; }
            }
            return ret;
        }
        bool l = closest_aux(inv, r, n.a, inct);
        bool rr = closest_aux(inv, r, n.b, inct);
        return l || rr;
    }

    bool has(const Ray& r) const {
        if (aggregate == ATRC_AGG_BVH) {
            V3 inv(1 / r.d.x, 1 / r.d.y, 1 / r.d.z);
            return has_aux(inv, r, 0);
        }
        for (auto& e : entities) if (e.has(r)) return true;  // native_aggregate.cpp:20-28
        return false;
    }
    bool closest(const Ray& r0, EntInct* inct) const {
        Ray r = r0;
        if (aggregate == ATRC_AGG_BVH) {
            V3 inv(1 / r.d.x, 1 / r.d.y, 1 / r.d.z);
            return closest_aux(inv, r, 0, inct);
        }
        bool ret = false;  // native_aggregate.cpp:30-44
        for (auto& e : entities) {
            if (e.closest(r, inct)) { inct->ent = &e; r.t_max = inct->t; ret = true; }
        }
        return ret;
    }
    // DefaultScene::visible (scene_default.cpp:136-141)
    bool visible(V3 A, V3 B) const {
        float dis = len(A - B);
        Ray sr(A, normalize(B - A), eps, dis - eps);
        return !has(sr);
    }

    // Material::shade -> BSDF
    BSDF shade(const EntInct& in, V3* shading_normal) const {
        BSDF b;
        const AtrcMaterialDesc& m = materials[in.ent->material];
        b.type = m.type;
        b.geo = in.geo;
        Coord shd = in.user;
        if (m.normal_map >= 0 && (m.type == ATRC_MAT_IDEAL_DIFFUSE || m.type == ATRC_MAT_DISNEY ||
                                  m.type == ATRC_MAT_METAL || m.type == ATRC_MAT_PHONG)) {
            // NormalMapper::reorient (material.h:25-57)
            V3 s = tex2d[m.normal_map].sample(in.uv);
            V3 ln = normalize(V3(s.x * 2 - 1, s.y * 2 - 1, s.z * 2 - 1));
            shd = in.user.rotate_to_new_z(in.user.local_to_global(ln));
        }
        b.shd = shd;
        switch (m.type) {
        case ATRC_MAT_IDEAL_DIFFUSE:
            b.albedo_ = tex2d[m.tex[0]].sample_at(in.uv, in.pos);  // ideal_diffuse.cpp:27, by intersection
            *shading_normal = shd.z;
            break;
        case ATRC_MAT_DISNEY: {
            auto T = [&](int slot) { return tex2d[m.tex[slot]].sample(in.uv); };
            auto R = [&](int slot) { return tex2d[m.tex[slot]].sample_real(in.uv); };
            b.init_disney(T(ATRC_DISNEY_BASE_COLOR), R(ATRC_DISNEY_METALLIC), R(ATRC_DISNEY_ROUGHNESS),
                          T(ATRC_DISNEY_SPECULAR_SCALE), R(ATRC_DISNEY_SPECULAR_TINT), R(ATRC_DISNEY_ANISOTROPIC),
                          R(ATRC_DISNEY_SHEEN), R(ATRC_DISNEY_SHEEN_TINT), R(ATRC_DISNEY_CLEARCOAT),
                          R(ATRC_DISNEY_CLEARCOAT_GLOSS), R(ATRC_DISNEY_TRANSMISSION),
                          R(ATRC_DISNEY_TRANSMISSION_ROUGHNESS), R(ATRC_DISNEY_IOR));
            *shading_normal = shd.z;
            break;
        }
        case ATRC_MAT_MIRROR: {  // Mirror::shade (mirror.cpp:98-115): ConductorPoint(ior, 1, k)
            V3 c = tex2d[m.tex[0]].sample(in.uv), ior = tex2d[m.tex[1]].sample(in.uv), k = tex2d[m.tex[2]].sample(in.uv);
            b.rc = c;
            b.eta2 = V3(1 / sqr(ior.x), 1 / sqr(ior.y), 1 / sqr(ior.z));
            b.etak2 = V3(sqr(k.x / ior.x), sqr(k.y / ior.y), sqr(k.z / ior.z));
            b.albedo_ = c;
            *shading_normal = shd.z;
            break;
        }
        case ATRC_MAT_GLASS: {  // Glass::shade (glass.cpp:180-206)
            b.glass_ior = tex2d[m.tex[2]].sample_at(in.uv, in.pos).x;  // by intersection
            b.refl_c = tex2d[m.tex[0]].sample_at(in.uv, in.pos);
            V3 rr = tex2d[m.tex[1]].sample_at(in.uv, in.pos);
            b.refr_c = V3(std::sqrt(rr.x), std::sqrt(rr.y), std::sqrt(rr.z));
            b.albedo_ = 0.5f * (b.refl_c + b.refr_c);
            *shading_normal = shd.z;
            break;
        }
        case ATRC_MAT_METAL: {  // Metal::shade (metal.cpp:39-62)
            V3 c = tex2d[m.tex[0]].sample(in.uv), eta = tex2d[m.tex[1]].sample(in.uv), k = tex2d[m.tex[2]].sample(in.uv);
            float rough = tex2d[m.tex[3]].sample_real(in.uv), aniso = tex2d[m.tex[4]].sample_real(in.uv);
            b.rc = c;
            b.eta2 = V3(sqr(eta.x), sqr(eta.y), sqr(eta.z));
            b.etak2 = V3(sqr(k.x), sqr(k.y), sqr(k.z));
            float aspect = aniso > 0 ? std::sqrt(1 - 0.9f * aniso) : 1.0f;
            b.ax = std::max(0.001f, sqr(rough) / aspect);
            b.ay = std::max(0.001f, sqr(rough) * aspect);
            b.roughness = rough;
            b.albedo_ = c;
            *shading_normal = shd.z;
            break;
        }
        case ATRC_MAT_PHONG: {  // Phong::shade (phong.cpp:33-79)
            V3 d = tex2d[m.tex[0]].sample(in.uv), sp = tex2d[m.tex[1]].sample(in.uv);
            float ns = tex2d[m.tex[2]].sample_real(in.uv);
            float dem = std::max(1.0f, std::max(d.x + sp.x, std::max(d.y + sp.y, d.z + sp.z)));
            d = d / dem;
            sp = sp / dem;
            float dl = lum(d), sl = lum(sp);
            b.wd = dl + sl > g_eps ? dl / (dl + sl) : 0.5f;
            b.wsp = 1 - b.wd;
            b.pd = d;
            b.ps = sp;
            b.pns = ns;
            b.albedo_ = d + sp;
            *shading_normal = shd.z;
            break;
        }
        case ATRC_MAT_INVISIBLE_SURFACE:
            b.geometry_normal = in.geo.z;
            *shading_normal = in.user.z;
            break;
        default:
            *shading_normal = in.user.z;
            break;
        }
        return b;
    }
};

namespace {

// ============================================================ direct light
struct Sample5 { float v[5]; };
Sample5 s5(Sampler& s) { Sample5 r; for (int i = 0; i < 5; ++i) r.v[i] = s.u(); return r; }

// mis_sample_area_light (surface) direct_illum.cpp:11-42
V3 mis_area_surface(const OracleScene& sc, const Entity* light, const EntInct& in, const BSDF& b, Sampler& s) {
    Sample5 sam = s5(s);
    V3 lpos, lnor, lrad;
    float lpdf;
    if (!light->light_sample(in.pos, sam.v, &lpos, &lnor, &lrad, &lpdf)) return V3();
    if (lrad.black() || !lpdf) return V3();
    const float slen = len(lpos - in.pos) - sc.eps;
    if (slen <= sc.eps) return V3();
    V3 to_light = normalize(lpos - in.pos);
    if (sc.has(Ray(in.pos, to_light, sc.eps, slen))) return V3();
    int med = in.medium(to_light);
    V3 bf = b.eval(to_light, in.wr);
    if (bf.black()) return V3();
    V3 f = sc.media[med].tr(lpos, in.pos, s) * lrad * bf * std::abs(cosv(to_light, in.geo.z));
    float bpdf = b.pdf(to_light, in.wr);
    return f / (lpdf + bpdf);
}
// mis_sample_area_light (medium) direct_illum.cpp:44-70
V3 mis_area_medium(const OracleScene& sc, const Entity* light, V3 pos, V3 wr, int med, const Phase& ph, Sampler& s) {
    Sample5 sam = s5(s);
    V3 lpos, lnor, lrad;
    float lpdf;
    if (!light->light_sample(pos, sam.v, &lpos, &lnor, &lrad, &lpdf)) return V3();
    if (lrad.black() || !lpdf) return V3();
    if (!sc.visible(lpos, pos)) return V3();
    V3 to_light = normalize(lpos - pos);
    V3 bf = ph.eval(to_light, wr);
    if (bf.black()) return V3();
    V3 f = sc.media[med].tr(pos, lpos, s) * lrad * bf;
    float bpdf = ph.pdf(to_light, wr);
    return f / (lpdf + bpdf);
}
// mis_sample_envir_light (surface) direct_illum.cpp:72-99
V3 mis_env_surface(const OracleScene& sc, const EntInct& in, const BSDF& b, Sampler& s) {
    Sample5 sam = s5(s);
    float pdf;
    V3 dir = sc.env.sample_dir(sam.v, &pdf);
    V3 rad = sc.env.radiance(dir);
    if (rad.black()) return V3();
    V3 lpos = sc.env.emit_pos(in.pos, dir);
    if (!sc.visible(in.pos, lpos)) return V3();
    V3 to_light = normalize(lpos - in.pos);
    V3 bf = b.eval(to_light, in.wr);
    if (bf.black()) return V3();
    V3 f = rad * bf * std::abs(cosv(to_light, in.geo.z));
    float bpdf = b.pdf(to_light, in.wr);
    return f / (pdf + bpdf);
}

// mis_sample_bsdf (surface) direct_illum.cpp:130-192, with the sample kept
V3 mis_bsdf_surface(const OracleScene& sc, const EntInct& in, const BSDF& b, Sampler& s) {
    float sam[3] = {s.u(), s.u(), s.u()};
    BSDFSample bs = b.sample(in.wr, sam);
    if (bs.f.black()) return V3();
    bs.dir = normalize(bs.dir);
    Ray nr(in.eps_offset(bs.dir), bs.dir);
    EntInct hit;
    bool has = sc.closest(nr, &hit);
    int med = in.medium(bs.dir);
    if (!has) {
        if (sc.env.type == ATRC_ENV_NONE) return V3();
        V3 lr = sc.env.radiance(nr.d);
        if (lr.black()) return V3();
        V3 f = lr * bs.f * std::abs(dot(in.geo.z, nr.d));
        if (bs.delta) return f / bs.pdf;
        return f / (bs.pdf + sc.env.pdf(nr.d));
    }
    if (!hit.ent->is_light) return V3();
    V3 lr = hit.ent->light_radiance(hit.geo.z, hit.wr);
    if (lr.black()) return V3();
    V3 tr = sc.media[med].tr(nr.o, hit.pos, s);
    V3 f = tr * lr * bs.f * std::abs(dot(in.geo.z, nr.d));
    if (bs.delta) return f / bs.pdf;
    return f / (bs.pdf + hit.ent->light_pdf(nr.o, hit.pos, hit.geo.z));
}
// mis_sample_bsdf (medium) direct_illum.cpp:194-248
V3 mis_bsdf_medium(const OracleScene& sc, V3 pos, V3 wr, int med, const Phase& ph, Sampler& s) {
    float sam[3] = {s.u(), s.u(), s.u()};
    BSDFSample bs = ph.sample(wr, sam);
    if (bs.f.black()) return V3();
    bs.dir = normalize(bs.dir);
    Ray nr(pos, bs.dir);
    EntInct hit;
    bool has = sc.closest(nr, &hit);
    if (!has) {
        if (sc.env.type == ATRC_ENV_NONE) return V3();
        V3 lf = sc.env.radiance(nr.d);
        if (lf.black()) return V3();
        V3 f = lf * bs.f;
        if (bs.delta) return f / bs.pdf;
        return f / (bs.pdf + sc.env.pdf(nr.d));
    }
    if (!hit.ent->is_light) return V3();
    V3 lf = hit.ent->light_radiance(hit.geo.z, hit.wr);
    if (lf.black()) return V3();
    V3 tr = sc.media[med].tr(nr.o, hit.pos, s);
    V3 f = tr * lf * bs.f;
    if (bs.delta) return f / bs.pdf;
    return f / (bs.pdf + hit.ent->light_pdf(nr.o, hit.pos, hit.geo.z));
}

struct Pixel {
    V3 value, albedo, normal;
    float denoise = 1;
};

// ---------------------------------------------------------- subsurface
// Normalized diffusion profile (normalized_diffusion.cpp:357-397): radial
// pdf p(x) = (e^-x + e^-x/3) / 4 in x = r / d, eval_r(r) = A (e^-x +
// e^-x/3) / (8 pi d), d = dmfp / (3.5 + 100 (A - 0.33)^4).  The reference
// samples r from a tabulated inverse cdf (agz-utils sample_inv_cdf_table,
// not in this container); this inverts the cdf by Newton's method.
float nd_inv_cdf(float uf) {
    double u = std::min(std::max(double(uf), 0.0), 1.0 - 1e-7);
    double x = u < 0.5 ? 2.0 * u : 3.0 * std::log(0.75 / (1.0 - u));
    for (int k = 0; k < 24; ++k) {
        double e1 = std::exp(-x), e3 = std::exp(-x / 3.0);
        double step = (1.0 - 0.25 * e1 - 0.75 * e3 - u) / (0.25 * (e1 + e3));
        x = std::max(x - step, 0.0);
        if (std::abs(step) <= 1e-12 * std::max(x, 1e-12)) break;
    }
    return float(x);
}
float nd_pdf_r(float d, float r) { float x = r / d; return 0.25f * (std::exp(-x) + std::exp(-x / 3.0f)) / d; }
float nd_scale(float a) { float t = a - 0.33f; return 3.5f + 100.0f * t * t * t * t; }
// first Fresnel moment, the polynomial fits used by separable.cpp:12-35
float fresnel_moment1(float eta) {
    float e2 = eta * eta, e3 = e2 * eta, e4 = e2 * e2, e5 = e2 * e3;
    if (eta < 1) return 0.45966f - 1.73965f * eta + 3.37668f * e2 - 3.904945f * e3 + 2.49277f * e4 - 0.68441f * e5;
    return -4.61686f + 11.1136f * eta - 10.4646f * e2 + 5.11455f * e3 - 1.27198f * e4 + 0.12746f * e5;
}

// SeparableBSSRDF::sample_pi (separable.cpp:107-220) from entry `po`:
// exit point `pi` with its separable BSDF, and the weight coef / pdf.
bool subsurface_sample(const OracleScene& sc, const AtrcMaterialDesc& m, const EntInct& po, Sampler& s,
                       EntInct* pi, BSDF* bx, V3* w) {
    const V3 A = sc.tex2d[m.bssrdf[0]].sample(po.uv), dmfp = sc.tex2d[m.bssrdf[1]].sample(po.uv);
    const float eta = sc.tex2d[m.bssrdf[2]].sample_real(po.uv);
    const float d[3] = {dmfp.x / nd_scale(A.x), dmfp.y / nd_scale(A.y), dmfp.z / nd_scale(A.z)};
    float sam[3] = {s.u(), s.u(), s.u()};
    int ch = std::min(int(sam[0] * 3), 2);  // extract_uniform_int
    float su = sam[0] * 3 - float(ch);
    Coord proj;
    float sv;
    if (sam[1] < 0.5f) { proj = po.geo; sv = 2 * sam[1]; }
    else if (sam[1] < 0.75f) { proj = Coord(po.geo.y, po.geo.z, po.geo.x); sv = 4 * (sam[1] - 0.5f); }
    else { proj = Coord(po.geo.z, po.geo.x, po.geo.y); sv = 4 * (sam[1] - 0.75f); }
    float r = nd_inv_cdf(su) * d[ch];
    float r_max = nd_inv_cdf(0.996f) * d[ch];
    if (!(r > 0) || r > r_max) return false;
    float phi = 2 * PI * sv;
    float hl = std::sqrt(std::max(0.0f, r_max * r_max - r * r));
    Ray probe(po.pos + proj.local_to_global(V3(r * std::cos(phi), r * std::sin(phi), hl)), -proj.z, g_eps,
              std::max(g_eps, 2 * hl));
    // every crossing of the same entity along the probe, one kept uniformly
    int cnt = 0;
    GeoInct pick;
    for (int k = 0; k < 64; ++k) {
        if (probe.t_min >= probe.t_max) break;
        GeoInct g;
        if (!po.ent->closest(probe, &g)) break;
        ++cnt;
        if (s.u() * float(cnt) < 1) pick = g;
        probe.o = probe.at(g.t + g_eps);
        probe.t_max -= g.t + g_eps;
    }
    if (!cnt) return false;
    static_cast<GeoInct&>(*pi) = pick;
    pi->ent = po.ent;
    // pdf_pi (separable.cpp:222-248)
    V3 ld = po.geo.global_to_local(po.pos - pi->pos), ln = po.geo.global_to_local(pi->geo.z);
    float rp[3] = {std::sqrt(ld.y * ld.y + ld.z * ld.z), std::sqrt(ld.z * ld.z + ld.x * ld.x),
                   std::sqrt(ld.x * ld.x + ld.y * ld.y)};
    float lnc[3] = {ln.x, ln.y, ln.z}, axis_pdf[3] = {0.25f, 0.25f, 0.5f};
    float pr = 0;
    for (int a = 0; a < 3; ++a)
        for (int c = 0; c < 3; ++c) pr += std::abs(lnc[a]) * nd_pdf_r(d[c], rp[a]) * axis_pdf[a];
    pr /= 3;
    float pdf = pr / (2 * PI) / float(cnt);
    if (!(pdf > 0)) return false;
    float fro = 1 - BSDF::dielectric_fresnel(eta, 1, cosv(po.wr, po.geo.z));
    float dist = len(pi->pos - po.pos);
    V3 ev(A.x * (std::exp(-dist / d[0]) + std::exp(-dist / (3 * d[0]))) / (8 * PI * d[0]),
          A.y * (std::exp(-dist / d[1]) + std::exp(-dist / (3 * d[1]))) / (8 * PI * d[1]),
          A.z * (std::exp(-dist / d[2]) + std::exp(-dist / (3 * d[2]))) / (8 * PI * d[2]));
    *w = fro * ev / pdf;
    BSDF b;
    b.type = BSDF::kSeparable;
    b.geo = b.shd = pi->geo;
    b.IOR = eta;
    b.sep_ci = 1 - 2 * fresnel_moment1(1 / eta);
    *bx = b;
    return true;
}

// render::trace_std (path_tracing.cpp:15-225), direct_illum_sample_count = 1
Pixel trace_std(const OracleScene& sc, const AtrcRenderDesc& p, Ray r, Sampler& s) {
    V3 coef(1);
    Pixel px;
    int scattering_count = 0;
    for (int depth = 1, s_depth = 1; depth <= p.max_depth; ++depth) {
        if (depth > p.min_depth) {
            if (s.u() > p.cont_prob) return px;
            coef /= p.cont_prob;
        }
        EntInct in;
        if (!sc.closest(r, &in)) {
            if (depth == 1 && sc.env.type != ATRC_ENV_NONE) px.value += coef * sc.env.radiance(r.d);
            return px;
        }
        V3 shading_normal;
        BSDF b = sc.shade(in, &shading_normal);
        if (depth == 1) {
            px.normal = shading_normal;
            px.albedo = b.albedo();
            if (in.ent->no_denoise) px.denoise = 0;
        }
        const int med = in.wr_medium();
        const Medium& medium = sc.media[med];
        if (scattering_count < medium.max_scat) {
            V3 tp, spos, swr;
            Phase ph;
            bool scattered = medium.sample_scattering(r.o, in.pos, s, scattering_count > 0, &tp, &spos, &swr, &ph);
            coef *= tp;
            if (scattered) {
                ++scattering_count;
                V3 di;
                for (const Light& l : sc.lights) {
                    if (l.is_env) continue;  // direct_illum.cpp:101-108 returns 0
                    di += coef * mis_area_medium(sc, l.ent, spos, swr, med, ph, s);
                }
                di += coef * mis_bsdf_medium(sc, spos, swr, med, ph, s);
                px.value += di;
                float sam[3] = {s.u(), s.u(), s.u()};
                BSDFSample bs = ph.sample(in.wr, sam);
                if (bs.f.black() || bs.pdf < sc.eps) return px;
                r = Ray(spos, normalize(bs.dir));
                coef *= bs.f / bs.pdf;
                continue;
            }
        } else {
            coef *= medium.ab(r.o, in.pos, s);
        }
        scattering_count = 0;
        if (depth == 1 && in.ent->is_light)
            px.value += coef * in.ent->light_radiance(in.geo.z, in.wr);
        V3 di;
        for (const Light& l : sc.lights) {
            if (l.is_env) di += coef * mis_env_surface(sc, in, b, s);
            else di += coef * mis_area_surface(sc, l.ent, in, b, s);
        }
        di += coef * mis_bsdf_surface(sc, in, b, s);
        px.value += di;
        float sam[3] = {s.u(), s.u(), s.u()};
        BSDFSample bs = b.sample(in.wr, sam);
        if (bs.f.black() || bs.pdf < sc.eps) return px;
        bool delta = bs.delta;
        const float abscos = std::abs(cosv(in.geo.z, bs.dir));
        coef *= bs.f * abscos / bs.pdf;
        r = Ray(in.eps_offset(bs.dir), normalize(bs.dir));
        // bssrdf (path_tracing.cpp:173-221)
        const AtrcMaterialDesc& mat = sc.materials[in.ent->material];
        if (mat.type == ATRC_MAT_DISNEY && mat.bssrdf[1] >= 0 && !in.geo.in_positive_z_hemisphere(bs.dir) &&
            in.geo.in_positive_z_hemisphere(in.wr)) {
            EntInct x;
            BSDF bx;
            V3 w;
            if (!subsurface_sample(sc, mat, in, s, &x, &bx, &w)) return px;
            coef *= w;
            V3 di2;
            for (const Light& l : sc.lights) {
                if (l.is_env) di2 += coef * mis_env_surface(sc, x, bx, s);
                else di2 += coef * mis_area_surface(sc, l.ent, x, bx, s);
            }
            di2 += coef * mis_bsdf_surface(sc, x, bx, s);
            px.value += di2;
            float sam2[3] = {s.u(), s.u(), s.u()};
            BSDFSample bs2 = bx.sample(x.wr, sam2);
            if (bs2.f.black()) return px;
            coef *= bs2.f * std::abs(cosv(x.geo.z, bs2.dir)) / bs2.pdf;
            r = Ray(x.eps_offset(bs2.dir), normalize(bs2.dir));
            delta = false;
        }
        if (delta && depth >= 2 && s_depth <= p.specular_depth) { --depth; ++s_depth; }
    }
    return px;
}

// render::trace_nomis (path_tracing.cpp:227-381), the pt renderer's path
// with use_mis = 0: BSDF sampling only, the emission of every light hit and
// the environment on every miss added unweighted, no light sampling.
Pixel trace_nomis(const OracleScene& sc, const AtrcRenderDesc& p, Ray r, Sampler& s) {
    V3 coef(1);
    Pixel px;
    int scattering_count = 0;
    for (int depth = 1, s_depth = 1; depth <= p.max_depth; ++depth) {
        if (depth > p.min_depth) {
            if (s.u() > p.cont_prob) return px;
            coef /= p.cont_prob;
        }
        EntInct in;
        if (!sc.closest(r, &in)) {
            if (sc.env.type != ATRC_ENV_NONE) px.value += coef * sc.env.radiance(r.d);
            return px;
        }
        V3 shading_normal;
        BSDF b = sc.shade(in, &shading_normal);
        if (depth == 1) {
            px.normal = shading_normal;
            px.albedo = b.albedo();
            if (in.ent->no_denoise) px.denoise = 0;
        }
        const Medium& medium = sc.media[in.wr_medium()];
        if (scattering_count < medium.max_scat) {
            V3 tp, spos, swr;
            Phase ph;
            bool scattered = medium.sample_scattering(r.o, in.pos, s, scattering_count > 0, &tp, &spos, &swr, &ph);
            coef *= tp;
            if (scattered) {
                ++scattering_count;
                float sam[3] = {s.u(), s.u(), s.u()};
                BSDFSample bs = ph.sample(in.wr, sam);
                if (bs.f.black() || !(bs.pdf > 0)) return px;
                coef *= bs.f / bs.pdf;
                r = Ray(spos, normalize(bs.dir));
                continue;
            }
        } else {
            coef *= medium.ab(r.o, in.pos, s);
        }
        scattering_count = 0;
        if (in.ent->is_light) px.value += coef * in.ent->light_radiance(in.geo.z, in.wr);
        float sam[3] = {s.u(), s.u(), s.u()};
        BSDFSample bs = b.sample(in.wr, sam);
        if (bs.f.black() || !(bs.pdf > 0)) return px;
        bool delta = bs.delta;
        coef *= bs.f * std::abs(cosv(in.geo.z, bs.dir)) / bs.pdf;
        r = Ray(in.eps_offset(bs.dir), normalize(bs.dir));
        const AtrcMaterialDesc& mat = sc.materials[in.ent->material];
        if (mat.type == ATRC_MAT_DISNEY && mat.bssrdf[1] >= 0 && !in.geo.in_positive_z_hemisphere(bs.dir) &&
            in.geo.in_positive_z_hemisphere(in.wr)) {
            EntInct x;
            BSDF bx;
            V3 w;
            if (!subsurface_sample(sc, mat, in, s, &x, &bx, &w)) return px;
            coef *= w;
            float sam2[3] = {s.u(), s.u(), s.u()};
            BSDFSample bs2 = bx.sample(x.wr, sam2);
            if (bs2.f.black() || !(bs2.pdf > 0)) return px;
            coef *= bs2.f * std::abs(cosv(x.geo.z, bs2.dir)) / bs2.pdf;
            r = Ray(x.eps_offset(bs2.dir), normalize(bs2.dir));
            delta = bs2.delta;
        }
        if (delta && depth >= 2 && s_depth <= p.specular_depth) { --depth; ++s_depth; }
    }
    return px;
}

// render::trace_ao (path_tracing.cpp:383-415)
Pixel trace_ao(const OracleScene& sc, const AtrcRenderDesc& p, Ray r, Sampler& s) {
    Pixel px;
    EntInct in;
    if (!sc.closest(r, &in)) {
        px.value = V3(p.ao_background);
        return px;
    }
    const V3 low(p.ao_low), high(p.ao_high);
    px.albedo = high;
    px.normal = in.geo.z;
    px.denoise = in.ent->no_denoise ? 0.0f : 1.0f;
    const V3 start = in.eps_offset(in.geo.z);
    float ao = 0;
    for (int i = 0; i < p.ao_sample_count; ++i) {
        const float u = s.u(), v = s.u();
        float pdf;
        const V3 dir = normalize(in.geo.local_to_global(zweighted_on_hemisphere(u, v, &pdf)));
        if (sc.visible(start, start + dir * p.ao_max_distance)) ao += 1;
    }
    ao /= float(p.ao_sample_count);
    const float t = clampf(ao, 0, 1);
    px.value = low * (1 - t) + high * t;
    return px;
}

// Film filter values (box_filter.cpp:6-34, gaussian_filter.cpp:6-78)
struct Filter {
    int type = ATRC_FILTER_BOX;
    float radius = 0.5f, alpha = 2, value = 1, exp_r = 0;
    void init(const AtrcRenderDesc& d, float eps) {
        type = d.filter_type;
        if (type == ATRC_FILTER_BOX) {
            radius = d.filter_radius - eps;
            value = 1 / (4 * radius * radius);
        } else {
            radius = d.filter_radius;
            alpha = d.filter_alpha;
            exp_r = std::exp(-alpha * radius * radius);
        }
    }
    float eval(float x, float y) const {
        if (type == ATRC_FILTER_BOX) return value;
        auto g = [&](float d) { return std::max(0.0f, std::exp(-alpha * d * d) - exp_r); };
        return g(x) * g(y);
    }
};

}  // namespace

// ======================================================================= C ABI
extern "C" {

const char* oracle_last_error(void) { return g_err.c_str(); }

int oracle_hardware_threads(void) { return int(std::max(1u, std::thread::hardware_concurrency())); }

int oracle_scene_create(const AtrcSceneDesc* d, float eps, OracleScene** out) {
    if (!d || !out) { g_err = "null argument"; return ATRC_ERR_INVALID_ARG; }
    try {
        g_eps = eps;
        auto sc = std::make_unique<OracleScene>();
        sc->eps = eps;
        sc->tex2d.resize(d->texture2d_count);
        for (uint32_t i = 0; i < d->texture2d_count; ++i) sc->tex2d[i].d = d->textures2d[i];
        sc->tex3d.resize(d->texture3d_count);
        for (uint32_t i = 0; i < d->texture3d_count; ++i) sc->tex3d[i].d = d->textures3d[i];
        for (Tex2D& t : sc->tex2d)
            if (t.d.type == ATRC_TEX_SOLID) {
                if (t.d.tex3d < 0 || uint32_t(t.d.tex3d) >= d->texture3d_count) throw std::runtime_error("bad solid_image");
                t.solid = &sc->tex3d[size_t(t.d.tex3d)];
            }
        sc->materials.assign(d->materials, d->materials + d->material_count);
        sc->media.resize(d->medium_count);
        for (uint32_t i = 0; i < d->medium_count; ++i) {
            const AtrcMediumDesc& md = d->media[i];
            Medium& m = sc->media[i];
            m.type = md.type;
            m.sa = V3(md.sigma_a); m.ss = V3(md.sigma_s); m.st = m.sa + m.ss;
            m.g = md.g;
            m.max_scat = md.max_scattering_count;
            m.xf = to_xform(md.transform);
            m.white_for_indirect = md.white_for_indirect;
            if (md.type == ATRC_MED_HETEROGENEOUS) {
                m.density = &sc->tex3d[md.density];
                m.albedo = &sc->tex3d[md.albedo];
                m.gtex = &sc->tex3d[md.g_tex];
                m.max_density = std::max(md.density >= 0 ? d->textures3d[md.density].max_real : 1.0f, eps);
                m.inv_max_density = 1 / m.max_density;
            }
        }
        sc->leaves.resize(d->geometry_count);
        for (uint32_t i = 0; i < d->geometry_count; ++i) sc->leaves[i].init(d->geometries[i], *d);
        sc->entities.resize(d->entity_count);
        AABB world;
        for (uint32_t i = 0; i < d->entity_count; ++i) {
            const AtrcEntityDesc& ed = d->entities[i];
            Entity& e = sc->entities[i];
            e.index = int(i);
            e.leaf = &sc->leaves[ed.geometry];
            e.has_wrap = ed.has_instance;
            e.wrap = to_xform(ed.instance);
            e.double_sided = ed.double_sided;
            e.material = ed.material;
            e.med_in = ed.medium_in;
            e.med_out = ed.medium_out;
            e.emit = V3(ed.emit_radiance);
            e.is_light = !e.emit.black();
            e.no_denoise = ed.no_denoise;
            e.power = ed.power;
            if (e.has_wrap) {  // transform_wrapper.cpp:13-27
                e.scale_ratio = len(xvec(e.wrap.m, V3(0, 0, 1)));
                V3 L = e.leaf->bound.low, H = e.leaf->bound.high;
                e.bound = AABB();
                for (int k = 0; k < 8; ++k)
                    e.bound.add(xpoint(e.wrap.m, V3(k & 4 ? H.x : L.x, k & 2 ? H.y : L.y, k & 1 ? H.z : L.z)));
            } else {
                e.bound = e.leaf->bound;
            }
            world.add(e.bound);
        }
        // lights (scene_default.cpp:66-82): env first, then entity lights
        sc->env.type = d->env.type;
        if (d->env.type != ATRC_ENV_NONE) {
            Light l;
            l.is_env = true;
            sc->lights.push_back(l);
            if (d->env.type == ATRC_ENV_IBL) {
                if (sc->tex2d[d->env.tex].d.type == ATRC_TEX_SOLID)
                    throw std::runtime_error("solid_image is not supported as an environment map");
                sc->env.tex = &sc->tex2d[d->env.tex];
                const Tex2D* t = sc->env.tex;
                if (d->env.no_importance_sampling) {
                    sc->env.sampler.init([](V2) { return V3(1.0f); }, 1, 1);
                } else {
                    int tw = t->d.type == ATRC_TEX_IMAGE ? t->d.width : 1;
                    int th = t->d.type == ATRC_TEX_IMAGE ? t->d.height : 1;
                    sc->env.sampler.init([t](V2 uv) { return t->sample(uv); }, tw, th);
                }
            } else {
                sc->env.top = V3(d->env.top);
                sc->env.bottom = V3(d->env.bottom);
            }
            // EnvirLight::preprocess (light.cpp:6-14)
            if (d->entity_count) {
                sc->env.radius = 1.1f * len(world.high - world.low) / 2;
                sc->env.centre = 0.5f * (world.low + world.high);
            }
        }
        for (auto& e : sc->entities) {
            if (e.is_light) { Light l; l.ent = &e; sc->lights.push_back(l); }
        }
        sc->aggregate = d->aggregate;
        sc->max_leaf = d->aggregate_max_leaf_size > 0 ? d->aggregate_max_leaf_size : 5;
        if (sc->aggregate == ATRC_AGG_BVH) {
            if (sc->entities.empty()) {
                AABB b;
                b.low = V3(0.0f); b.high = V3(1.0f);
                sc->nodes.push_back({b, true, 0, 0});
            } else {
                std::vector<std::pair<const Entity*, AABB>> recs;
                for (auto& e : sc->entities) recs.push_back({&e, e.bound});
                sc->build_aux(recs, 0, recs.size());
            }
        }
        *out = sc.release();
        return ATRC_OK;
    } catch (const std::exception& e) {
        g_err = e.what();
        return ATRC_ERR_INVALID_ARG;
    }
}

void oracle_scene_destroy(OracleScene* s) { delete s; }

static void parallel_for(size_t n, int threads, const std::function<void(size_t)>& fn) {
    int t = threads > 0 ? threads : oracle_hardware_threads();
    if (t <= 1 || n < 2) { for (size_t i = 0; i < n; ++i) fn(i); return; }
    std::atomic<size_t> next{0};
    std::vector<std::thread> pool;
    for (int k = 0; k < t; ++k)
        pool.emplace_back([&] {
            for (;;) {
                size_t i = next.fetch_add(1);
                if (i >= n) break;
                fn(i);
            }
        });
    for (auto& th : pool) th.join();
}

// Sets the calling thread's ray-primitive test for a scope.
struct IsectScope {
    int saved;
    explicit IsectScope(int mode) : saved(g_isect) { g_isect = mode; }
    ~IsectScope() { g_isect = saved; }
};

int oracle_trace_rays(OracleScene* s, const AtrcRay* rays, size_t n, AtrcHit* hits, int mode, int isect, int threads) {
    if (!s || (!rays && n) || (!hits && n)) { g_err = "null argument"; return ATRC_ERR_INVALID_ARG; }
    if (isect != ATRC_ISECT_EXACT && isect != ATRC_ISECT_WATERTIGHT) { g_err = "bad isect mode"; return ATRC_ERR_INVALID_ARG; }
    const size_t chunk = 4096;
    parallel_for((n + chunk - 1) / chunk, threads, [&](size_t c) {
        IsectScope scope(isect);
        for (size_t i = c * chunk; i < std::min(n, (c + 1) * chunk); ++i) {
            const AtrcRay& q = rays[i];
            Ray r(V3(q.o), V3(q.d), q.t_min, q.t_max);
            AtrcHit& h = hits[i];
            if (mode == ATRC_QUERY_ANY) {
                bool occ = s->has(r);
                h.t = occ ? 1.0f : -1.0f;
                h.entity = occ ? 0 : -1;
                h.prim = 0;
                h.u = 0;
            } else {
                EntInct in;
                if (s->closest(r, &in)) {
                    h.t = in.t;
                    h.entity = in.ent->index;
                    h.prim = in.prim;
                    h.u = 0;
                } else {
                    h.t = -1; h.entity = -1; h.prim = -1; h.u = 0;
                }
            }
        }
    });
    return ATRC_OK;
}

int oracle_prim_hit(OracleScene* s, const AtrcRay* q, int entity, int prim, int isect, float* t_out) {
    if (!s || !q || !t_out || entity < 0 || size_t(entity) >= s->entities.size()) return ATRC_ERR_INVALID_ARG;
    if (isect != ATRC_ISECT_EXACT && isect != ATRC_ISECT_WATERTIGHT) return ATRC_ERR_INVALID_ARG;
    IsectScope scope(isect);
    const Entity& e = s->entities[entity];
    Ray r(V3(q->o), V3(q->d), q->t_min, q->t_max);
    if (e.has_wrap) r = Ray(xpoint(e.wrap.inv, r.o), xvec(e.wrap.inv, r.d), r.t_min, r.t_max);
    const Leaf& l = *e.leaf;
    float t;
    V2 uv;
    *t_out = -1;
    if (l.type == ATRC_GEOM_TRIANGLE_BVH) {
        const TriBVH& b = *l.bvh;
        for (size_t i = 0; i < b.orig.size(); ++i) {
            if (int(b.orig[i]) != prim) continue;
            const TriBVH::Prim& pr = b.prims[i];
            if (tri_closest(r, pr.a, pr.b_a, pr.c_a, pr.b, pr.c, &t, &uv)) *t_out = t;
            return ATRC_OK;
        }
        return ATRC_ERR_INVALID_ARG;
    }
    if (l.type == ATRC_GEOM_QUAD) {
        bool ok = prim == 0 ? tri_closest(r, l.a, l.b_a, l.c_a, l.b, l.c, &t, &uv)
                            : tri_closest(r, l.a, l.c_a, l.d_a, l.c, l.d, &t, &uv);
        if (ok) *t_out = t;
        return ATRC_OK;
    }
    GeoInct g;
    if (l.closest(r, &g)) *t_out = g.t;
    return ATRC_OK;
}

int oracle_render(OracleScene* s, const AtrcRenderDesc* d, AtrcFilm* film, int threads) {
    return oracle_render_sample(s, d, film, threads, 1);
}

int oracle_render_sample(OracleScene* s, const AtrcRenderDesc* d, AtrcFilm* film, int threads, int tile_stride) {
    if (!s || !d || !film || !film->value || !film->weight) { g_err = "null argument"; return ATRC_ERR_INVALID_ARG; }
    if (tile_stride < 1) { g_err = "tile_stride must be >= 1"; return ATRC_ERR_INVALID_ARG; }
    if (film->on_device) { g_err = "the oracle renders into host memory only"; return ATRC_ERR_INVALID_ARG; }
    g_eps = s->eps = d->eps;
    g_disney_fixed = d->disney_fixed;
    const int isect = d->isect_mode == ATRC_ISECT_WATERTIGHT ? ATRC_ISECT_WATERTIGHT : ATRC_ISECT_EXACT;
    const int W = d->width, H = d->height;
    const int spp = d->spp_count > 0 ? d->spp_count : d->spp;
    // camera (thin_lens.cpp:34-94); look-at frame: z = forward, x = up x z
    const AtrcCameraDesc& c = d->camera;
    V3 pos(c.pos), dst(c.dst), up(c.up);
    V3 fz = normalize(dst - pos);
    V3 fx = normalize(cross(up, fz));
    V3 fy = cross(fz, fx);
    const float aspect = float(W) / float(H);
    const float film_h = 2 * c.focal_distance * std::tan(c.fov / 2);
    const float film_w = aspect * film_h;
    Filter filter;
    filter.init(*d, s->eps);
    const int grid = d->task_grid_size > 0 ? d->task_grid_size : 32;  // renderer_creators.cpp:128
    const int tx = (W + grid - 1) / grid, ty = (H + grid - 1) / grid;
    std::mutex mtx;
    const size_t n_tiles = size_t(tx) * ty;
    parallel_for((n_tiles + tile_stride - 1) / tile_stride, threads, [&](size_t tile_k) {
        IsectScope scope(isect);
        const size_t tile = tile_k * size_t(tile_stride);
        const int gx = int(tile % tx), gy = int(tile / tx);
        const int x0 = gx * grid, y0 = gy * grid;
        const int x1 = std::min(W, x0 + grid) - 1, y1 = std::min(H, y0 + grid) - 1;
        const uint64_t seed = mix64(d->seed ^ mix64(uint64_t(d->first_spp) * 0x1000193ULL + tile));
        Sampler smp(seed, tile);
        // FilmGrid sample bound (framebuffer.h sample_bound_of)
        const int sx0 = int(std::floor(x0 + 0.5f - filter.radius));
        const int sy0 = int(std::floor(y0 + 0.5f - filter.radius));
        const int sx1 = int(std::floor(x1 + 0.49999f + filter.radius));
        const int sy1 = int(std::floor(y1 + 0.49999f + filter.radius));
        const int gw = x1 - x0 + 1, gh = y1 - y0 + 1;
        std::vector<double> acc(size_t(gw) * gh * 14, 0.0);
        for (int py = sy0; py <= sy1; ++py) {
            for (int pxi = sx0; pxi <= sx1; ++pxi) {
                for (int i = 0; i < spp; ++i) {
                    // render_grid (perpixel_renderer.cpp:21-53)
                    const float fu = smp.u(), fv = smp.u();
                    const float pixel_x = pxi + fu, pixel_y = py + fv;
                    const float film_x = pixel_x / W, film_y = pixel_y / H;
                    const float au = smp.u(), av = smp.u();
                    V3 focal((0.5f - film_x) * film_w, (film_y - 0.5f) * film_h, c.focal_distance);
                    V2 disk = concentric_disk(au, av);
                    V3 lens(c.lens_radius * disk.x, c.lens_radius * disk.y, 0);
                    V3 o = pos + fx * lens.x + fy * lens.y + fz * lens.z;
                    V3 ld = focal - lens;
                    V3 dir = normalize(fx * ld.x + fy * ld.y + fz * ld.z);
                    Pixel pv = d->renderer == ATRC_RENDERER_AO ? trace_ao(*s, *d, Ray(o, dir), smp)
                               : d->use_mis                     ? trace_std(*s, *d, Ray(o, dir), smp)
                                                                : trace_nomis(*s, *d, Ray(o, dir), smp);
                    if (!finite3(pv.value)) continue;
                    // apply_image_filter (framebuffer.h:49-80)
                    const int xmin = std::max(x0, int(std::ceil(pixel_x - filter.radius - 0.5f)));
                    const int ymin = std::max(y0, int(std::ceil(pixel_y - filter.radius - 0.5f)));
                    const int xmax = std::min(x1, int(std::floor(pixel_x + filter.radius - 0.5f)));
                    const int ymax = std::min(y1, int(std::floor(pixel_y + filter.radius - 0.5f)));
                    float yrel = std::abs(ymin + 0.5f - pixel_y);
                    for (int yy = ymin; yy <= ymax; ++yy, yrel += 1) {
                        if (yrel > filter.radius) continue;
                        float xrel = std::abs(xmin + 0.5f - pixel_x);
                        for (int xx = xmin; xx <= xmax; ++xx, xrel += 1) {
                            if (xrel > filter.radius) continue;
                            const double w = filter.eval(xrel, yrel);
                            double* a = &acc[(size_t(yy - y0) * gw + (xx - x0)) * 14];
                            for (int k = 0; k < 3; ++k) {
                                a[k] += w * pv.value[k];
                                a[3 + k] += w * double(pv.value[k]) * double(pv.value[k]);
                                a[7 + k] += w * pv.albedo[k];
                                a[10 + k] += w * pv.normal[k];
                            }
                            a[6] += w;
                            a[13] += w * pv.denoise;
                        }
                    }
                }
            }
        }
        // GridFilm::merge_into
        std::lock_guard<std::mutex> lk(mtx);
        for (int yy = 0; yy < gh; ++yy)
            for (int xx = 0; xx < gw; ++xx) {
                const double* a = &acc[(size_t(yy) * gw + xx) * 14];
                const size_t p = size_t(y0 + yy) * W + (x0 + xx);
                for (int k = 0; k < 3; ++k) {
                    film->value[3 * p + k] += a[k];
                    if (film->value_sq) film->value_sq[3 * p + k] += a[3 + k];
                    if (film->albedo) film->albedo[3 * p + k] += a[7 + k];
                    if (film->normal) film->normal[3 * p + k] += a[10 + k];
                }
                film->weight[p] += a[6];
                if (film->denoise) film->denoise[p] += a[13];
            }
    });
    return ATRC_OK;
}

int oracle_env_pdf(OracleScene* s, const float* dirs, size_t n, float* pdf) {
    if (!s || s->env.type == ATRC_ENV_NONE) return ATRC_ERR_INVALID_ARG;
    for (size_t i = 0; i < n; ++i) pdf[i] = s->env.pdf(V3(dirs + 3 * i));
    return ATRC_OK;
}

int oracle_env_sample(OracleScene* s, const float* u3, size_t n, float* dirs, float* pdf) {
    if (!s || s->env.type == ATRC_ENV_NONE) return ATRC_ERR_INVALID_ARG;
    for (size_t i = 0; i < n; ++i) {
        V3 d = s->env.sample_dir(u3 + 3 * i, &pdf[i]);
        dirs[3 * i] = d.x; dirs[3 * i + 1] = d.y; dirs[3 * i + 2] = d.z;
    }
    return ATRC_OK;
}

static BSDF probe_bsdf(OracleScene* s, int material) {
    EntInct in;
    Entity fake;
    fake.material = material;
    in.ent = &fake;
    in.geo = Coord();
    in.user = Coord();
    in.uv = V2(0.5f, 0.5f);
    V3 sn;
    BSDF b = s->shade(in, &sn);
    return b;
}

int oracle_bsdf_eval(OracleScene* s, int material, const float* wi, const float* wo, size_t n, float* f, float* pdf) {
    if (!s || material < 0 || size_t(material) >= s->materials.size()) return ATRC_ERR_INVALID_ARG;
    BSDF b = probe_bsdf(s, material);
    for (size_t i = 0; i < n; ++i) {
        V3 v = b.eval(V3(wi + 3 * i), V3(wo + 3 * i));
        f[3 * i] = v.x; f[3 * i + 1] = v.y; f[3 * i + 2] = v.z;
        pdf[i] = b.pdf(V3(wi + 3 * i), V3(wo + 3 * i));
    }
    return ATRC_OK;
}

int oracle_bsdf_sample(OracleScene* s, int material, const float* wo, const float* u3, size_t n, float* wi, float* f,
                       float* pdf, int* is_delta, int disney_fixed) {
    if (!s || material < 0 || size_t(material) >= s->materials.size()) return ATRC_ERR_INVALID_ARG;
    g_disney_fixed = disney_fixed;
    BSDF b = probe_bsdf(s, material);
    for (size_t i = 0; i < n; ++i) {
        BSDFSample r = b.sample(V3(wo + 3 * i), u3 + 3 * i);
        wi[3 * i] = r.dir.x; wi[3 * i + 1] = r.dir.y; wi[3 * i + 2] = r.dir.z;
        f[3 * i] = r.f.x; f[3 * i + 1] = r.f.y; f[3 * i + 2] = r.f.z;
        pdf[i] = r.pdf;
        is_delta[i] = r.delta;
    }
    return ATRC_OK;
}

int oracle_subsurface(OracleScene* s, const float* o, const float* d, size_t n, uint64_t seed, float* w,
                      float* exit_pos) {
    if (!s || !o || !d || !w || !exit_pos) return ATRC_ERR_INVALID_ARG;
    EntInct in;
    if (!s->closest(Ray(V3(o), normalize(V3(d))), &in)) return ATRC_ERR_INVALID_ARG;
    const AtrcMaterialDesc& m = s->materials[in.ent->material];
    if (m.type != ATRC_MAT_DISNEY || m.bssrdf[1] < 0) return ATRC_ERR_INVALID_ARG;
    Sampler smp(seed, 7);
    for (size_t i = 0; i < n; ++i) {
        EntInct x;
        BSDF bx;
        V3 wv;
        if (!subsurface_sample(*s, m, in, smp, &x, &bx, &wv)) { wv = V3(); x.pos = V3(); }
        w[3 * i] = wv.x; w[3 * i + 1] = wv.y; w[3 * i + 2] = wv.z;
        exit_pos[3 * i] = x.pos.x; exit_pos[3 * i + 1] = x.pos.y; exit_pos[3 * i + 2] = x.pos.z;
    }
    return ATRC_OK;
}

}  // extern "C"
