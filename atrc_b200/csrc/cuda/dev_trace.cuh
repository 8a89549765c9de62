// Two-level BVH traversal (top level over entities, bottom level per leaf
// geometry) with the reference's ray-primitive tests.
//
// Replaces, for a batch of rays, the reference's EntityBVH / NativeAggregate
// traversal (src/tracer/src/core/aggregate/entity_bvh.cpp:118-172), the
// transform_wrapper ray transform (src/tracer/src/core/geometry/
// transform_wrapper.cpp:51-68), the per-mesh BVH
// (src/tracer/src/core/geometry/triangle_bvh.cpp:363-488) and the
// Moller-Trumbore test (src/tracer/include/agz/tracer/utility/
// triangle_aux.h:9-69).  The intersection mode (IsectMode) is a template
// parameter of the traversal:
//   ISECT_FAST       Moller-Trumbore as the compiler schedules it (FMAs);
//   ISECT_EXACT      every float operation of the ray transform and of
//                    Moller-Trumbore in the reference's order without fused
//                    multiply-adds, so hit distances are bit-identical;
//   ISECT_WATERTIGHT the watertight triangle test of Woop, Benthin and Wald
//                    (JCGT 2(1), 2013) on the triangles' exact vertices, and
//                    sphere roots without cancellation.  A ray through an
//                    edge or vertex shared by two triangles of a mesh hits at
//                    least one of them; Moller-Trumbore with alpha >= 0 and
//                    alpha + beta <= 1 rounded per triangle can miss both.
#pragma once

#include <climits>

#include "dev_math.cuh"
#include "dev_scene.h"

namespace atrc {
namespace dev {

constexpr int kStackSize = 96;
// Optional traversal short stack (ATRC_STACK_RING > 0): the top entries of
// each thread's stack live in shared memory (a ring, entry i in slot
// i % kStackRing, slots strided by the block size so a warp's accesses hit
// 32 banks); deeper entries spill to local memory.  Off by default: on the
// instanced 3.08M-triangle workload a 16-entry ring ran 3.7 % slower than the
// plain local-memory stack (597 vs 620 Msamples/s), whose top entries stay
// in L1 anyway, while the ring's shared memory shrinks L1 for BVH nodes.
// Every kernel that traces launches blocks of at most kTraceBlock threads
// (__launch_bounds__ enforces it).
#ifndef ATRC_STACK_RING
#define ATRC_STACK_RING 0
#endif
constexpr int kStackRing = ATRC_STACK_RING;
constexpr int kTraceBlock = 128;
static_assert(kStackRing == 0 || (kStackRing & (kStackRing - 1)) == 0, "ring size must be a power of two");
static_assert(kStackRing < kStackSize, "ring must be smaller than the stack");
constexpr int32_t kSentinel = INT_MIN;      // "return from a bottom-level tree"
constexpr int32_t kDone = INT_MIN + 1;      // empty stack
constexpr int kMaxTraversalSteps = 1 << 20; // node + leaf visits per ray before the watchdog trips

struct Hit {
    float t;
    float u, v;      // barycentrics (alpha, beta) for triangles
    int32_t entity;  // -1 when nothing was hit
    int32_t tri;     // pool triangle index (-1 for analytic shapes)
};

struct RayState {
    Vec3 o, d, inv;
    float tmin, tmax;
};

// Reciprocal direction for the slab tests.  The slab test evaluates
// lo * inv - o * inv (one FMA per plane), which for a zero component would
// be inf - inf = NaN and cull every box; a zero (or denormal-small)
// component is replaced by +-1e-20 (sign kept), so the slab of that axis is
// a huge finite interval on the correct side.
__device__ __forceinline__ float safe_rcp(float x) { return 1.0f / (fabsf(x) > 1e-20f ? x : copysignf(1e-20f, x)); }
__device__ __forceinline__ Vec3 safe_inv(Vec3 d) { return Vec3(safe_rcp(d.x), safe_rcp(d.y), safe_rcp(d.z)); }

enum IsectMode : int { ISECT_FAST = 0, ISECT_EXACT = 1, ISECT_WATERTIGHT = 2 };

// Moller-Trumbore.  ANY selects has_intersection_with_triangle (alpha <= 1
// also checked), otherwise closest_intersection_with_triangle.
template <bool EXACT, bool ANY>
__device__ __forceinline__ bool mt_test(const RayState& r, const float4& p0, const float4& p1, const float4& p2,
                                        float tmax, float* t_out, float* u_out, float* v_out) {
    const Vec3 A(p0.x, p0.y, p0.z), B_A(p1.x, p1.y, p1.z), C_A(p2.x, p2.y, p2.z);
    if (EXACT) {
        const Vec3 s1 = cross_rn(r.d, C_A);
        const float div = dot_rn(s1, B_A);
        if (div == 0.0f) return false;
        const float inv_div = __fdiv_rn(1.0f, div);
        const Vec3 o_A = sub_rn(r.o, A);
        const float alpha = __fmul_rn(dot_rn(o_A, s1), inv_div);
        if (alpha < 0 || (ANY && alpha > 1)) return false;
        const Vec3 s2 = cross_rn(o_A, B_A);
        const float beta = __fmul_rn(dot_rn(r.d, s2), inv_div);
        if (beta < 0 || __fadd_rn(alpha, beta) > 1) return false;
        const float t = __fmul_rn(dot_rn(C_A, s2), inv_div);
        if (!(r.tmin <= t && t <= tmax)) return false;
        *t_out = t;
        *u_out = alpha;
        *v_out = beta;
        return true;
    } else {
        const Vec3 s1 = cross(r.d, C_A);
        const float div = dot(s1, B_A);
        if (div == 0.0f) return false;
        const float inv_div = 1.0f / div;
        const Vec3 o_A = r.o - A;
        const float alpha = dot(o_A, s1) * inv_div;
        if (alpha < 0 || (ANY && alpha > 1)) return false;
        const Vec3 s2 = cross(o_A, B_A);
        const float beta = dot(r.d, s2) * inv_div;
        if (beta < 0 || alpha + beta > 1) return false;
        const float t = dot(C_A, s2) * inv_div;
        if (!(r.tmin <= t && t <= tmax)) return false;
        *t_out = t;
        *u_out = alpha;
        *v_out = beta;
        return true;
    }
}

// Per-ray constants of the watertight test: the axis of the largest
// direction component becomes z (kz), kx and ky follow cyclically and swap
// when d[kz] < 0 (which keeps the triangles' winding), and the shear that
// maps the direction onto +z.
struct WtRay {
    int kx, ky, kz;
    float sx, sy, sz;
};

__device__ __forceinline__ float comp(const Vec3& v, int k) { return k == 0 ? v.x : (k == 1 ? v.y : v.z); }

__device__ __forceinline__ WtRay wt_setup(const Vec3& d) {
    const float ax = fabsf(d.x), ay = fabsf(d.y), az = fabsf(d.z);
    WtRay w;
    w.kz = ax > ay ? (ax > az ? 0 : 2) : (ay > az ? 1 : 2);
    w.kx = w.kz == 2 ? 0 : w.kz + 1;
    w.ky = w.kx == 2 ? 0 : w.kx + 1;
    const float dz = comp(d, w.kz);
    if (dz < 0) {
        const int t = w.kx;
        w.kx = w.ky;
        w.ky = t;
    }
    w.sx = __fdiv_rn(comp(d, w.kx), dz);
    w.sy = __fdiv_rn(comp(d, w.ky), dz);
    w.sz = __fdiv_rn(1.0f, dz);
    return w;
}

// Watertight ray-triangle test on the exact vertices A, B, C (Woop, Benthin
// and Wald 2013).  The vertices are moved to the ray origin and sheared so
// that the ray is the +z axis; the signs of the three 2D edge functions
// decide the hit.  An edge function is evaluated from the same two rounded
// vertex coordinates in both triangles that share the edge, with opposite
// signs, so no ray passes between them; edge functions that round to zero
// are evaluated again in double precision, where the products are exact.
// Both windings are accepted (no culling).  alpha / beta are the weights of
// B and C, as Moller-Trumbore's.  No fused multiply-adds: a contracted
// a*b - c*d is not antisymmetric under the swap that the neighbour makes.
template <bool ANY>
__device__ __forceinline__ bool wt_test(const RayState& r, const WtRay& w, const float4& pa, const float4& pb,
                                        const float4& pc, float tmax, float* t_out, float* u_out, float* v_out) {
    const Vec3 A = sub_rn(Vec3(pa.x, pa.y, pa.z), r.o);
    const Vec3 B = sub_rn(Vec3(pb.x, pb.y, pb.z), r.o);
    const Vec3 C = sub_rn(Vec3(pc.x, pc.y, pc.z), r.o);
    const float az = comp(A, w.kz), bz = comp(B, w.kz), cz = comp(C, w.kz);
    const float Ax = __fsub_rn(comp(A, w.kx), __fmul_rn(w.sx, az)), Ay = __fsub_rn(comp(A, w.ky), __fmul_rn(w.sy, az));
    const float Bx = __fsub_rn(comp(B, w.kx), __fmul_rn(w.sx, bz)), By = __fsub_rn(comp(B, w.ky), __fmul_rn(w.sy, bz));
    const float Cx = __fsub_rn(comp(C, w.kx), __fmul_rn(w.sx, cz)), Cy = __fsub_rn(comp(C, w.ky), __fmul_rn(w.sy, cz));
    float U = __fsub_rn(__fmul_rn(Cx, By), __fmul_rn(Cy, Bx));
    float V = __fsub_rn(__fmul_rn(Ax, Cy), __fmul_rn(Ay, Cx));
    float W = __fsub_rn(__fmul_rn(Bx, Ay), __fmul_rn(By, Ax));
    if (U == 0.0f || V == 0.0f || W == 0.0f) {
        U = __double2float_rn(__dsub_rn(__dmul_rn(double(Cx), double(By)), __dmul_rn(double(Cy), double(Bx))));
        V = __double2float_rn(__dsub_rn(__dmul_rn(double(Ax), double(Cy)), __dmul_rn(double(Ay), double(Cx))));
        W = __double2float_rn(__dsub_rn(__dmul_rn(double(Bx), double(Ay)), __dmul_rn(double(By), double(Ax))));
    }
    if ((U < 0 || V < 0 || W < 0) && (U > 0 || V > 0 || W > 0)) return false;
    const float det = __fadd_rn(__fadd_rn(U, V), W);
    if (det == 0.0f) return false;
    const float T = __fadd_rn(__fadd_rn(__fmul_rn(U, __fmul_rn(w.sz, az)), __fmul_rn(V, __fmul_rn(w.sz, bz))),
                              __fmul_rn(W, __fmul_rn(w.sz, cz)));
    const float rcp = __fdiv_rn(1.0f, det);
    const float t = __fmul_rn(T, rcp);
    if (!(r.tmin <= t && t <= tmax)) return false;
    *t_out = t;
    *u_out = __fmul_rn(V, rcp);
    *v_out = __fmul_rn(W, rcp);
    return true;
}

// Sphere (sphere_aux.h:53-86) in local space.
template <bool ANY>
__device__ __forceinline__ bool sphere_test(const RayState& r, float radius, float tmax, float* t_out) {
    const float A = dot(r.d, r.d), B = 2 * dot(r.d, r.o), C = dot(r.o, r.o) - radius * radius;
    float delta = B * B - 4 * A * C;
    if (delta < 0) return false;
    delta = sqrtf(delta);
    const float inv2A = 0.5f / A;
    const float t0 = (-B - delta) * inv2A, t1 = (-B + delta) * inv2A;
    if (ANY) {
        if (r.tmin <= t0 && t0 <= tmax) { *t_out = t0; return true; }
        if (r.tmin <= t1 && t1 <= tmax) { *t_out = t1; return true; }
        return false;
    }
    if (tmax < t0 || t1 < r.tmin) return false;
    const bool not_t0 = t0 < r.tmin;
    if (not_t0 && t1 > tmax) return false;
    *t_out = not_t0 ? t1 : t0;
    return true;
}

// Sphere without cancellation (watertight mode): with b = o.d, the
// discriminant is a (r^2 - |o - (b/a) d|^2) instead of b^2 - a (o.o - r^2),
// which loses every digit when the ray passes far from the centre, and the
// roots are q / a and c / q with q = -(b + sign(b) sqrt(disc)) instead of
// (-b -+ sqrt(disc)) / a, which cancels for the root near the origin (Haines
// et al., "Precision Improvements for Ray/Sphere Intersection", Ray Tracing
// Gems, 2019).  Same root selection as sphere_test.
template <bool ANY>
__device__ __forceinline__ bool sphere_test_robust(const RayState& r, float radius, float tmax, float* t_out) {
    const float a = dot(r.d, r.d);
    if (!(a > 0)) return false;
    const float b = dot(r.o, r.d);
    const Vec3 l = r.o - (b / a) * r.d;
    const float disc = a * (radius * radius - dot(l, l));
    if (disc < 0) return false;
    const float c = dot(r.o, r.o) - radius * radius;
    const float q = -(b + copysignf(sqrtf(disc), b));
    float t0 = q / a, t1 = q != 0.0f ? c / q : t0;
    if (t0 > t1) {
        const float tt = t0;
        t0 = t1;
        t1 = tt;
    }
    if (ANY) {
        if (r.tmin <= t0 && t0 <= tmax) { *t_out = t0; return true; }
        if (r.tmin <= t1 && t1 <= tmax) { *t_out = t1; return true; }
        return false;
    }
    if (tmax < t0 || t1 < r.tmin) return false;
    const bool not_t0 = t0 < r.tmin;
    if (not_t0 && t1 > tmax) return false;
    *t_out = not_t0 ? t1 : t0;
    return true;
}

// Disk (disk.cpp:43-74) in local space.
__device__ __forceinline__ bool disk_test(const RayState& r, float radius, float tmax, float* t_out) {
    const float t = -r.o.z / r.d.z;
    if (isinf(t) || !(r.tmin <= t && t <= tmax)) return false;
    const float px = r.o.x + t * r.d.x, py = r.o.y + t * r.d.y;
    if (px * px + py * py > radius * radius) return false;
    *t_out = t;
    return true;
}

// Slab test of the four children of a wide node (seven 128-bit loads):
// t[k] = entry distance of child k, +inf when it is missed or the slot is
// empty.  Boxes are widened by 1.0000005 as in the binary test, so a box
// that touches the ray in exact arithmetic is never culled.
__device__ __forceinline__ void box4(const Bvh4Node* node, const RayState& r, float* t, int32_t* l) {
    const float4* p = reinterpret_cast<const float4*>(node);
    const float4 lx = __ldg(p), hx = __ldg(p + 1), ly = __ldg(p + 2), hy = __ldg(p + 3);
    const float4 lz = __ldg(p + 4), hz = __ldg(p + 5);
    const int4 lk = __ldg(reinterpret_cast<const int4*>(p + 6));
    const float ox = r.o.x * r.inv.x, oy = r.o.y * r.inv.y, oz = r.o.z * r.inv.z;
    const float alx[4] = {lx.x, lx.y, lx.z, lx.w}, ahx[4] = {hx.x, hx.y, hx.z, hx.w};
    const float aly[4] = {ly.x, ly.y, ly.z, ly.w}, ahy[4] = {hy.x, hy.y, hy.z, hy.w};
    const float alz[4] = {lz.x, lz.y, lz.z, lz.w}, ahz[4] = {hz.x, hz.y, hz.z, hz.w};
    const int32_t al[4] = {lk.x, lk.y, lk.z, lk.w};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const float a0 = fmaf(alx[k], r.inv.x, -ox), b0 = fmaf(ahx[k], r.inv.x, -ox);
        const float a1 = fmaf(aly[k], r.inv.y, -oy), b1 = fmaf(ahy[k], r.inv.y, -oy);
        const float a2 = fmaf(alz[k], r.inv.z, -oz), b2 = fmaf(ahz[k], r.inv.z, -oz);
        const float lo = fmaxf(fmaxf(fminf(a0, b0), fminf(a1, b1)), fmaxf(fminf(a2, b2), r.tmin));
        const float hi = fminf(fminf(fmaxf(a0, b0), fmaxf(a1, b1)), fminf(fmaxf(a2, b2), r.tmax));
        const bool hit = al[k] != kEmptyLink && lo <= hi * 1.0000005f + 1e-30f;
        t[k] = hit ? lo : INFINITY;
        l[k] = al[k];
    }
}

// Sort four (distance, link) pairs by distance (five compare-exchanges).
__device__ __forceinline__ void sort4(float* t, int32_t* l) {
    auto cx = [&](int a, int b) {
        if (t[b] < t[a]) {
            const float tt = t[a]; t[a] = t[b]; t[b] = tt;
            const int32_t ll = l[a]; l[a] = l[b]; l[b] = ll;
        }
    };
    cx(0, 1); cx(2, 3); cx(0, 2); cx(1, 3); cx(1, 2);
}

// Move a world ray into an entity's primitive space (wrapper, then the
// geometry's own transform), as transform_wrapper / TransformedGeometry do.
__device__ __forceinline__ void to_entity_space(const Entity& e, Vec3 o, Vec3 d, Vec3* lo, Vec3* ld) {
    if (e.flags & ENT_WRAP) {
        o = apply_point_rn(e.wrap_inv, o);
        d = apply_vector_rn(e.wrap_inv, d);
    }
    if (e.flags & ENT_LOCAL) {
        o = apply_point_rn(e.local_inv, o);
        d = apply_vector_rn(e.local_inv, d);
    }
    *lo = o;
    *ld = d;
}

// Functional work counts of one traversal (for the roofline's algorithmic bytes).
struct TraceCount {
    uint32_t nodes;  // 64-byte node fetches
    uint32_t tris;   // 48-byte triangle fetches + tests
    uint32_t ents;   // entity (instance) visits
};

// Traversal of one ray, resumable: step() runs one round of the traversal
// (descend to leaves, then the leaves) and says whether the ray is done, so
// a kernel can refill the lanes of finished rays between rounds (k_extend);
// trace_ray() runs the rounds to the end.  ANY stops at the first hit
// (occlusion); with COUNT the work done is added to a TraceCount.
//
// Structure (after Aila and Laine, "Understanding the efficiency of ray
// traversal on GPUs", 2009): a thread that reaches a leaf while descending
// parks it and keeps descending; the warp switches to leaf processing only
// once every active lane holds a leaf, so node and leaf code run with most
// lanes converged.  Top-level leaves (entities) switch the ray into the
// entity's space and push a sentinel that restores the world ray when the
// bottom-level tree is exhausted.  A ray whose stack would overflow or
// whose visits exceed kMaxTraversalSteps ends with the watchdog set.
// The traversal stack is the caller's local array (kStackSize entries, the
// deeper ones past a shared-memory ring with ATRC_STACK_RING), kept out of
// the struct so that the scalar state stays in registers.
template <int ISECT, bool ANY, bool COUNT = false>
struct Tracer {
#if ATRC_STACK_RING > 0
    int32_t* ring;
#endif
    int32_t* stack;
    int sp;
    RayState r;
    WtRay w;  // watertight mode: shear of the current (world or entity) ray
    Vec3 wo, wd, winv;
    float tmin0, best_t, best_u, best_v;
    int32_t best_e, best_tri, cur_entity, link, held;
    int steps;
    bool overflow, found;

    __device__ __forceinline__ void init(const Scene& S, int32_t* stk, Vec3 o, Vec3 d, float tmin, float tmax) {
        stack = stk;
#if ATRC_STACK_RING > 0
        // entry i sits in ring slot i % R; pushing entry sp evicts entry
        // sp - R to the spill array, popping entry sp refills its slot
        __shared__ int32_t s_ring[kStackRing * kTraceBlock];
        ring = s_ring + threadIdx.x;
#endif
        sp = 0;
        wo = o; wd = d; winv = safe_inv(d);
        r.o = o; r.d = d; r.inv = winv; r.tmin = tmin; r.tmax = tmax;
        if (ISECT == ISECT_WATERTIGHT) w = wt_setup(d);
        tmin0 = tmin;
        best_t = tmax; best_u = 0; best_v = 0;
        best_e = -1; best_tri = -1; cur_entity = -1;
        link = S.entity_count == 0 ? kDone : S.tlas_root;
        held = 0;
        steps = 0;
        overflow = false;
        found = false;
    }

#if ATRC_STACK_RING > 0
    __device__ __forceinline__ void push(int32_t v) {
        if (sp >= kStackSize) { overflow = true; return; }
        int32_t& slot = ring[(sp & (kStackRing - 1)) * kTraceBlock];
        if (sp >= kStackRing) stack[sp - kStackRing] = slot;
        slot = v;
        ++sp;
    }
    __device__ __forceinline__ int32_t pop() {
        if (sp <= 0) return kDone;
        --sp;
        int32_t& slot = ring[(sp & (kStackRing - 1)) * kTraceBlock];
        const int32_t v = slot;
        if (sp >= kStackRing) slot = stack[sp - kStackRing];
        return v;
    }
#else
    __device__ __forceinline__ void push(int32_t v) {
        if (sp >= kStackSize) { overflow = true; return; }
        stack[sp++] = v;
    }
    __device__ __forceinline__ int32_t pop() { return sp > 0 ? stack[--sp] : kDone; }
#endif

    // Visit leaf `lf`; `next` is what follows it.  Returns the new link.
    // Sets `found` in ANY mode when something was hit.
    __device__ __forceinline__ int32_t visit_leaf(const Scene& S, int32_t lf, int32_t next, TraceCount* cnt) {
        const uint32_t enc = uint32_t(~lf);
        const int32_t first = int32_t(enc >> 4), count = int32_t(enc & 15) + 1;
        if (cur_entity < 0) {
            // top level: one entity per leaf slot (the builder uses leaves of 1)
            for (int32_t k = 0; k < count; ++k) {
                const int32_t ei = int32_t(__ldg(S.tlas_order + first + k));
                const Entity& e = S.entities[ei];
                if (COUNT) cnt->ents++;
                Vec3 lo, ld;
                to_entity_space(e, wo, wd, &lo, &ld);
                if (e.kind == LEAF_TRIANGLES) {
                    push(next);
                    push(kSentinel);
                    r.o = lo; r.d = ld; r.inv = safe_inv(ld);
                    if (ISECT == ISECT_WATERTIGHT) w = wt_setup(ld);
                    cur_entity = ei;
                    return e.blas_root;
                }
                RayState lr;
                lr.o = lo; lr.d = ld; lr.tmin = tmin0; lr.inv = Vec3();
                float t;
                const bool h = e.kind == LEAF_SPHERE
                                   ? (ISECT == ISECT_WATERTIGHT ? sphere_test_robust<ANY>(lr, e.radius, best_t, &t)
                                                                : sphere_test<ANY>(lr, e.radius, best_t, &t))
                                   : disk_test(lr, e.radius, best_t, &t);
                if (h) {
                    if (ANY) { best_e = ei; best_t = t; found = true; return kDone; }
                    if (t < best_t || (t == best_t && ei < best_e)) {
                        best_t = t; best_e = ei; best_tri = -1; best_u = 0; best_v = 0;
                        r.tmax = t;
                    }
                }
            }
            return next;
        }
        for (int32_t k = 0; k < count; ++k) {
            const int32_t ti = first + k;
            const float4* tp = reinterpret_cast<const float4*>(S.tris) + size_t(ti) * 3;
            if (COUNT) cnt->tris++;
            float t, u, v;
            bool hit;
            if (ISECT == ISECT_WATERTIGHT) {
                const float4* bc = reinterpret_cast<const float4*>(S.tri_bc) + size_t(ti) * 2;
                hit = wt_test<ANY>(r, w, __ldg(tp), __ldg(bc), __ldg(bc + 1), best_t, &t, &u, &v);
            } else {
                hit = mt_test<ISECT == ISECT_EXACT, ANY>(r, __ldg(tp), __ldg(tp + 1), __ldg(tp + 2), best_t, &t, &u, &v);
            }
            if (hit) {
                if (ANY) { best_e = cur_entity; best_t = t; found = true; return kDone; }
                if (t < best_t || (t == best_t && (cur_entity < best_e || (cur_entity == best_e && ti < best_tri)))) {
                    best_t = t; best_e = cur_entity; best_tri = ti; best_u = u; best_v = v;
                    r.tmax = t;
                }
            }
        }
        return next;
    }

    // One round: descend (parking the first leaf found) until every active
    // lane holds a leaf, then the leaves.  Returns true when the ray is done.
    __device__ __forceinline__ bool step(const Scene& S, int* watchdog, TraceCount* cnt) {
        if (link == kDone && held == 0) return true;
        while (link >= 0) {
            if (++steps > kMaxTraversalSteps) { overflow = true; break; }
            if (COUNT) cnt->nodes++;
            // four children: entry distances (+inf when missed or empty),
            // sorted near to far; the far ones go on the stack
            float tc[4];
            int32_t lc[4];
            box4(S.nodes + link, r, tc, lc);
            if (ANY) {
                // occlusion needs any hit, not the nearest: children in slot
                // order, no sort
                int32_t nxt = kDone;
                for (int k = 3; k >= 0; --k) {
                    if (tc[k] == INFINITY) continue;
                    if (nxt != kDone) push(nxt);
                    nxt = lc[k];
                }
                link = nxt != kDone ? nxt : pop();
            } else {
                sort4(tc, lc);
                if (tc[0] == INFINITY) {
                    link = pop();
                } else {
                    if (tc[3] != INFINITY) push(lc[3]);
                    if (tc[2] != INFINITY) push(lc[2]);
                    if (tc[1] != INFINITY) push(lc[1]);
                    link = lc[0];
                }
            }
            if (link < 0 && link != kSentinel && link != kDone && held == 0) {
                held = link;
                link = pop();
            }
            if (overflow) break;
            if (!__any_sync(__activemask(), held == 0)) break;
        }
        if (overflow) { *watchdog = 1; return true; }
        // leaves: the parked one first, then any leaf / sentinel in `link`
        if (held != 0) {
            link = visit_leaf(S, held, link, cnt);
            held = 0;
            if (found) return true;
        }
        while (link < 0) {
            if (link == kDone) break;
            if (++steps > kMaxTraversalSteps) { overflow = true; break; }
            if (link == kSentinel) {
                cur_entity = -1;
                r.o = wo; r.d = wd; r.inv = winv;
                if (ISECT == ISECT_WATERTIGHT) w = wt_setup(wd);
                link = pop();
                continue;
            }
            const int32_t next = pop();
            link = visit_leaf(S, link, next, cnt);
            if (found) break;
        }
        if (overflow) { *watchdog = 1; return true; }
        return found || link == kDone;
    }

    // The result once step() said done: true if something was hit.
    __device__ __forceinline__ bool result(Hit* hit) const {
        if (ANY) {
            if (found) { hit->entity = best_e; hit->t = best_t; }
            return found;
        }
        if (best_e < 0) return false;
        hit->t = best_t;
        hit->u = best_u;
        hit->v = best_v;
        hit->entity = best_e;
        hit->tri = best_tri;
        return true;
    }
};

// Trace one ray to the end.  Returns true if something was hit (ANY:
// occluded); `watchdog` is set when the traversal stack would overflow.
template <int ISECT, bool ANY, bool COUNT = false>
__device__ bool trace_ray(const Scene& S, Vec3 wo, Vec3 wd, float tmin, float tmax, Hit* hit, int* watchdog,
                          TraceCount* cnt = nullptr) {
    int32_t stack[kStackSize];
    Tracer<ISECT, ANY, COUNT> t;
    t.init(S, stack, wo, wd, tmin, tmax);
    while (!t.step(S, watchdog, cnt)) {
    }
    return t.result(hit);
}

// Closest hit of a ray with one entity in [tmin, tmax]
// (GeometricEntity::closest_intersection), for the subsurface probe: the
// entity's own tree only, depth-first with a private stack.  Returns false
// on a miss; sets *watchdog when the stack or the step bound would be
// exceeded.
template <bool EXACT>
__device__ bool trace_entity(const Scene& S, int32_t ei, Vec3 wo, Vec3 wd, float tmin, float tmax, Hit* hit,
                             int* watchdog) {
    const Entity& e = S.entities[ei];
    Vec3 lo, ld;
    to_entity_space(e, wo, wd, &lo, &ld);
    if (e.kind != LEAF_TRIANGLES) {
        RayState lr;
        lr.o = lo; lr.d = ld; lr.tmin = tmin; lr.tmax = tmax; lr.inv = Vec3();
        float t;
        const bool h = e.kind == LEAF_SPHERE ? sphere_test<false>(lr, e.radius, tmax, &t) : disk_test(lr, e.radius, tmax, &t);
        if (!h) return false;
        hit->t = t; hit->u = 0; hit->v = 0; hit->entity = ei; hit->tri = -1;
        return true;
    }
    RayState r;
    r.o = lo; r.d = ld; r.inv = safe_inv(ld); r.tmin = tmin; r.tmax = tmax;
    int32_t stack[kStackSize];
    int sp = 0;
    int32_t link = e.blas_root;
    float best_t = tmax, best_u = 0, best_v = 0;
    int32_t best_tri = -1;
    for (int steps = 0;; ++steps) {
        if (steps > kMaxTraversalSteps) { *watchdog = 1; return false; }
        if (link >= 0) {
            float tc[4];
            int32_t lc[4];
            box4(S.nodes + link, r, tc, lc);
            sort4(tc, lc);
            if (sp + 3 > kStackSize) { *watchdog = 1; return false; }
            if (tc[3] != INFINITY) stack[sp++] = lc[3];
            if (tc[2] != INFINITY) stack[sp++] = lc[2];
            if (tc[1] != INFINITY) stack[sp++] = lc[1];
            link = tc[0] != INFINITY ? lc[0] : (sp > 0 ? stack[--sp] : kDone);
            continue;
        }
        if (link == kDone) break;
        const uint32_t enc = uint32_t(~link);
        const int32_t first = int32_t(enc >> 4), count = int32_t(enc & 15) + 1;
        for (int32_t k = 0; k < count; ++k) {
            const int32_t ti = first + k;
            const float4* tp = reinterpret_cast<const float4*>(S.tris) + size_t(ti) * 3;
            float t, u, v;
            if (mt_test<EXACT, false>(r, __ldg(tp), __ldg(tp + 1), __ldg(tp + 2), best_t, &t, &u, &v)) {
                if (t < best_t || (t == best_t && ti < best_tri)) {
                    best_t = t; best_tri = ti; best_u = u; best_v = v;
                    r.tmax = t;
                }
            }
        }
        link = sp > 0 ? stack[--sp] : kDone;
    }
    if (best_tri < 0) return false;
    hit->t = best_t; hit->u = best_u; hit->v = best_v; hit->entity = ei; hit->tri = best_tri;
    return true;
}

}  // namespace dev
}  // namespace atrc
