// Device math: frames, random numbers and sampling distributions.
//
// The distributions restate the published mappings that the reference takes
// from agz-utils (absent from its checkout): Shirley-Chiu concentric disk,
// Malley's cosine-weighted hemisphere, sqrt-parameterised uniform triangle,
// uniform sphere and cone.  The frame conventions (from_z, rotate_to_new_z)
// are the ones the host loader and the CPU oracle use.
#pragma once

#include <cstdint>

#include "../host/vecmath.h"

namespace atrc {
namespace dev {

constexpr float kPi = 3.14159265358979323846f;
constexpr float kInvPi = 0.318309886183790671538f;

struct Coord {
    Vec3 x, y, z;
    __device__ Vec3 local_to_global(Vec3 v) const { return x * v.x + y * v.y + z * v.z; }
    __device__ Vec3 global_to_local(Vec3 v) const { return Vec3(dot(v, x), dot(v, y), dot(v, z)); }
    __device__ bool positive(Vec3 v) const { return dot(v, z) > 0; }
    __device__ Coord neg() const { return Coord{-x, -y, -z}; }
};

__device__ __forceinline__ Coord coord_from_z(Vec3 zz) {
    Vec3 z = normalize(zz);
    Vec3 t = fabsf(z.x) > 0.9f ? Vec3(0, 1, 0) : Vec3(1, 0, 0);
    Vec3 y = normalize(cross(z, t));
    Vec3 x = cross(y, z);
    return Coord{x, y, z};
}

// Gram-Schmidt of the old x against the new z
__device__ __forceinline__ Coord rotate_to_new_z(const Coord& c, Vec3 nz_) {
    Vec3 nz = normalize(nz_);
    Vec3 nx = c.x - nz * dot(c.x, nz);
    float l = length(nx);
    if (!(l > 1e-6f)) return coord_from_z(nz);
    nx = nx * (1.0f / l);
    return Coord{nx, cross(nz, nx), nz};
}

__device__ __forceinline__ Coord xform_coord(const float* m, const Coord& c) {
    return Coord{normalize(apply_vector_rn(m, c.x)), normalize(apply_vector_rn(m, c.y)),
                 normalize(apply_vector_rn(m, c.z))};
}

__device__ __forceinline__ float cosv(Vec3 a, Vec3 b) { return dot(a, b) / (length(a) * length(b)); }
__device__ __forceinline__ float sqrf(float x) { return x * x; }
__device__ __forceinline__ float clampf(float x, float lo, float hi) { return fminf(fmaxf(x, lo), hi); }
__device__ __forceinline__ float lum(Vec3 c) { return 0.2126f * c.x + 0.7152f * c.y + 0.0722f * c.z; }
__device__ __forceinline__ bool black(Vec3 c) { return c.x == 0.0f && c.y == 0.0f && c.z == 0.0f; }
__device__ __forceinline__ Vec3 mix(Vec3 a, Vec3 b, float t) { return a * (1 - t) + b * t; }

// ------------------------------------------------------------------ RNG
// PCG32 (O'Neill, XSH-RR 64/32) stream per path.
struct Rng {
    uint64_t state;
    __device__ __forceinline__ uint32_t next() {
        uint64_t old = state;
        state = old * 6364136223846793005ULL + 1442695040888963407ULL;
        uint32_t xs = uint32_t(((old >> 18u) ^ old) >> 27u);
        uint32_t rot = uint32_t(old >> 59u);
        return (xs >> rot) | (xs << ((32u - rot) & 31u));
    }
    __device__ __forceinline__ float u() { return float(next() >> 8) * (1.0f / 16777216.0f); }
};

__host__ __device__ __forceinline__ uint64_t mix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

// --------------------------------------------------------- distributions
__device__ __forceinline__ void concentric_disk(float u, float v, float* dx, float* dy) {
    float a = 2 * u - 1, b = 2 * v - 1;
    if (a == 0 && b == 0) { *dx = 0; *dy = 0; return; }
    float r, phi;
    if (fabsf(a) > fabsf(b)) { r = a; phi = (kPi / 4) * (b / a); }
    else { r = b; phi = kPi / 2 - (kPi / 4) * (a / b); }
    float s, c;
    sincosf(phi, &s, &c);
    *dx = r * c;
    *dy = r * s;
}

__device__ __forceinline__ float zweighted_pdf(float z) { return z > 0 ? z * kInvPi : 0.0f; }

__device__ __forceinline__ Vec3 zweighted_on_hemisphere(float u, float v, float* pdf) {
    float x, y;
    concentric_disk(u, v, &x, &y);
    float z = sqrtf(fmaxf(0.0f, 1 - x * x - y * y));
    *pdf = z * kInvPi;
    return Vec3(x, y, z);
}

__device__ __forceinline__ void uniform_on_triangle(float u, float v, float* b0, float* b1) {
    float t = sqrtf(u);
    *b0 = 1 - t;
    *b1 = t * v;
}

__device__ __forceinline__ Vec3 uniform_on_sphere(float u, float v, float* pdf) {
    float z = 1 - 2 * u;
    float r = sqrtf(fmaxf(0.0f, 1 - z * z));
    float s, c;
    sincosf(2 * kPi * v, &s, &c);
    *pdf = 1 / (4 * kPi);
    return Vec3(r * c, r * s, z);
}

__device__ __forceinline__ float uniform_on_cone_pdf(float cos_max) { return 1 / (2 * kPi * (1 - cos_max)); }

__device__ __forceinline__ Vec3 uniform_on_cone(float cos_max, float u, float v, float* pdf) {
    float ct = (1 - u) + u * cos_max;
    float st = sqrtf(fmaxf(0.0f, 1 - ct * ct));
    float s, c;
    sincosf(2 * kPi * v, &s, &c);
    *pdf = uniform_on_cone_pdf(cos_max);
    return Vec3(c * st, s * st, ct);
}

__device__ __forceinline__ int alias_sample(const float* prob, const int32_t* alias, int n, float u) {
    float nu = u * n;
    int i = min(int(nu), n - 1);
    float frac = nu - float(i);
    return frac < prob[i] ? i : alias[i];
}

__device__ __forceinline__ float phi_of(Vec3 w) {  // local_angle::phi (common.h)
    if (w.y == 0.0f && w.x == 0.0f) return 0;
    float r = atan2f(w.y, w.x);
    return r < 0 ? r + 2 * kPi : r;
}

}  // namespace dev
}  // namespace atrc
