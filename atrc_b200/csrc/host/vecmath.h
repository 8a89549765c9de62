// Small vector / affine-transform library shared by the host loader and the
// device kernels.
//
// The reference takes these types from agz-utils (math::tvec3, ttransform3,
// tcoord3 ...; used throughout src/tracer, e.g.
// src/tracer/include/agz/tracer/common.h:48-88).  That submodule is not part of
// the reference checkout, so its conventions are fixed here and documented:
//  - dot(a, b) = (a.x*b.x + a.y*b.y) + a.z*b.z, evaluated left to right;
//  - cross(a, b) = (a.y*b.z - a.z*b.y, a.z*b.x - a.x*b.z, a.x*b.y - a.y*b.x);
//  - an affine transform applies as ((m0*x + m1*y) + m2*z) + m3 per row;
//  - normalize(v) = v * (1 / length(v)).
// Functions that must be bit-reproducible between the host and the device
// (geometry baking, Moller-Trumbore, ray transforms) use the *_rn helpers,
// which never contract into fused multiply-adds on the device.
#pragma once

#include <cmath>
#include <cstdint>

#if defined(__CUDACC__)
#define ATRC_HD __host__ __device__ __forceinline__
#else
#define ATRC_HD inline
#endif

namespace atrc {

// ---- non-contracting float arithmetic (IEEE round-to-nearest) -------------
ATRC_HD float fmul_rn(float a, float b) {
#if defined(__CUDA_ARCH__)
    return __fmul_rn(a, b);
#else
    return a * b;
#endif
}
ATRC_HD float fadd_rn(float a, float b) {
#if defined(__CUDA_ARCH__)
    return __fadd_rn(a, b);
#else
    return a + b;
#endif
}
ATRC_HD float fsub_rn(float a, float b) {
#if defined(__CUDA_ARCH__)
    return __fsub_rn(a, b);
#else
    return a - b;
#endif
}
ATRC_HD float fdiv_rn(float a, float b) {
#if defined(__CUDA_ARCH__)
    return __fdiv_rn(a, b);
#else
    return a / b;
#endif
}

struct Vec2 {
    float x, y;
    ATRC_HD Vec2() : x(0), y(0) {}
    ATRC_HD explicit Vec2(float v) : x(v), y(v) {}
    ATRC_HD Vec2(float x_, float y_) : x(x_), y(y_) {}
};
ATRC_HD Vec2 operator+(Vec2 a, Vec2 b) { return Vec2(a.x + b.x, a.y + b.y); }
ATRC_HD Vec2 operator-(Vec2 a, Vec2 b) { return Vec2(a.x - b.x, a.y - b.y); }
ATRC_HD Vec2 operator*(float s, Vec2 a) { return Vec2(s * a.x, s * a.y); }

struct Vec3 {
    float x, y, z;
    ATRC_HD Vec3() : x(0), y(0), z(0) {}
    ATRC_HD explicit Vec3(float v) : x(v), y(v), z(v) {}
    ATRC_HD Vec3(float x_, float y_, float z_) : x(x_), y(y_), z(z_) {}
    ATRC_HD float operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
    ATRC_HD float& operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
};

ATRC_HD Vec3 operator+(Vec3 a, Vec3 b) { return Vec3(a.x + b.x, a.y + b.y, a.z + b.z); }
ATRC_HD Vec3 operator-(Vec3 a, Vec3 b) { return Vec3(a.x - b.x, a.y - b.y, a.z - b.z); }
ATRC_HD Vec3 operator-(Vec3 a) { return Vec3(-a.x, -a.y, -a.z); }
ATRC_HD Vec3 operator*(Vec3 a, Vec3 b) { return Vec3(a.x * b.x, a.y * b.y, a.z * b.z); }
ATRC_HD Vec3 operator*(float s, Vec3 a) { return Vec3(s * a.x, s * a.y, s * a.z); }
ATRC_HD Vec3 operator*(Vec3 a, float s) { return Vec3(a.x * s, a.y * s, a.z * s); }
ATRC_HD Vec3 operator/(Vec3 a, float s) { return Vec3(a.x / s, a.y / s, a.z / s); }
ATRC_HD Vec3 operator/(Vec3 a, Vec3 b) { return Vec3(a.x / b.x, a.y / b.y, a.z / b.z); }
ATRC_HD Vec3& operator+=(Vec3& a, Vec3 b) { a.x += b.x; a.y += b.y; a.z += b.z; return a; }
ATRC_HD Vec3& operator*=(Vec3& a, Vec3 b) { a.x *= b.x; a.y *= b.y; a.z *= b.z; return a; }
ATRC_HD Vec3& operator*=(Vec3& a, float s) { a.x *= s; a.y *= s; a.z *= s; return a; }

ATRC_HD float dot(Vec3 a, Vec3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
ATRC_HD Vec3 cross(Vec3 a, Vec3 b) {
    return Vec3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
ATRC_HD float length_sq(Vec3 a) { return dot(a, a); }
ATRC_HD float length(Vec3 a) { return sqrtf(dot(a, a)); }
ATRC_HD Vec3 normalize(Vec3 a) { return a * (1.0f / length(a)); }
ATRC_HD bool is_zero(Vec3 a) { return a.x == 0.0f && a.y == 0.0f && a.z == 0.0f; }
ATRC_HD float max_elem(Vec3 a) { return fmaxf(a.x, fmaxf(a.y, a.z)); }
ATRC_HD Vec3 vmin(Vec3 a, Vec3 b) { return Vec3(fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z)); }
ATRC_HD Vec3 vmax(Vec3 a, Vec3 b) { return Vec3(fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z)); }

// bit-reproducible variants (no FMA contraction on the device)
ATRC_HD Vec3 sub_rn(Vec3 a, Vec3 b) {
    return Vec3(fsub_rn(a.x, b.x), fsub_rn(a.y, b.y), fsub_rn(a.z, b.z));
}
ATRC_HD Vec3 add_rn(Vec3 a, Vec3 b) {
    return Vec3(fadd_rn(a.x, b.x), fadd_rn(a.y, b.y), fadd_rn(a.z, b.z));
}
ATRC_HD float dot_rn(Vec3 a, Vec3 b) {
    return fadd_rn(fadd_rn(fmul_rn(a.x, b.x), fmul_rn(a.y, b.y)), fmul_rn(a.z, b.z));
}
ATRC_HD Vec3 cross_rn(Vec3 a, Vec3 b) {
    return Vec3(fsub_rn(fmul_rn(a.y, b.z), fmul_rn(a.z, b.y)),
                fsub_rn(fmul_rn(a.z, b.x), fmul_rn(a.x, b.z)),
                fsub_rn(fmul_rn(a.x, b.y), fmul_rn(a.y, b.x)));
}

// Row-major 3x4 affine transform with a host-computed inverse.
struct Affine {
    float m[12];
    float inv[12];
};

ATRC_HD void affine_identity(float* m) {
    for (int i = 0; i < 12; ++i) m[i] = 0.0f;
    m[0] = m[5] = m[10] = 1.0f;
}

ATRC_HD Vec3 apply_point_rn(const float* m, Vec3 p) {
    return Vec3(
        fadd_rn(fadd_rn(fadd_rn(fmul_rn(m[0], p.x), fmul_rn(m[1], p.y)), fmul_rn(m[2], p.z)), m[3]),
        fadd_rn(fadd_rn(fadd_rn(fmul_rn(m[4], p.x), fmul_rn(m[5], p.y)), fmul_rn(m[6], p.z)), m[7]),
        fadd_rn(fadd_rn(fadd_rn(fmul_rn(m[8], p.x), fmul_rn(m[9], p.y)), fmul_rn(m[10], p.z)), m[11]));
}
ATRC_HD Vec3 apply_vector_rn(const float* m, Vec3 v) {
    return Vec3(
        fadd_rn(fadd_rn(fmul_rn(m[0], v.x), fmul_rn(m[1], v.y)), fmul_rn(m[2], v.z)),
        fadd_rn(fadd_rn(fmul_rn(m[4], v.x), fmul_rn(m[5], v.y)), fmul_rn(m[6], v.z)),
        fadd_rn(fadd_rn(fmul_rn(m[8], v.x), fmul_rn(m[9], v.y)), fmul_rn(m[10], v.z)));
}
// normals transform with the inverse transpose
ATRC_HD Vec3 apply_normal(const float* inv, Vec3 n) {
    return Vec3(inv[0] * n.x + inv[4] * n.y + inv[8] * n.z,
                inv[1] * n.x + inv[5] * n.y + inv[9] * n.z,
                inv[2] * n.x + inv[6] * n.y + inv[10] * n.z);
}

// 2D affine (row-major 2x3) used for texture coordinates.
struct Affine2 {
    float m[6];
};

}  // namespace atrc
