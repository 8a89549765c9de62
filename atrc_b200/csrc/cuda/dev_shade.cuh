// Device shading: textures, surface interactions, BSDFs, lights and media.
//
// Reference algorithms (file:line inside src/tracer unless noted):
//   Texture2D::sample_spectrum          include/agz/tracer/core/texture2d.h:133-145
//   Texture3D::sample_spectrum          include/agz/tracer/core/texture3d.h
//   AggregateBSDF + DiffuseComponent    src/core/material/component/aggregate.h:40-245,
//                                       src/core/material/component/diffuse_comp.cpp:10-45
//   LocalBSDF black-fringe handling     include/agz/tracer/core/bsdf.h:113-202
//   DisneyBSDF                          src/core/material/disney.cpp:18-670
//   microfacet helpers                  src/core/material/utility/microfacet.cpp:18-128
//   InvisibleSurfaceBSDF                src/core/material/invisible_surface.cpp:9-59
//   GeometryToDiffuseLight              src/core/entity/area_light/geometry_to_diffuse_light.cpp
//   Quad / Triangle / Sphere / Disk     src/core/geometry/*.cpp, utility/sphere_aux.h
//   transform_wrapper / double_sided    src/core/geometry/transform_wrapper.cpp, double_sided.cpp
//   IBL + EnvironmentLightSampler       src/core/envir_light/ibl.cpp, env_sampler.h
//   NativeSky                           src/core/envir_light/native_sky.cpp
//   Homogeneous / Heterogeneous media   src/core/medium/homogeneous.cpp, heterogeneous.cpp
//   Henyey-Greenstein                   include/agz/tracer/utility/phase_function.h:8-90
// Angles are taken as sin/cos of phi directly from the normalised x/y
// components instead of atan2 followed by sin/cos (mathematically identical).
#pragma once

#include "dev_math.cuh"
#include "dev_scene.h"
#include "dev_trace.cuh"

namespace atrc {
namespace dev {

// ================================================================ textures
__device__ __forceinline__ float wrap_coord(int mode, float x) {
    if (mode == 1) return clampf(x - floorf(x), 0, 1);
    if (mode == 2) {
        const int ip = int(x >= 0 ? x : floorf(x));
        return clampf((ip & 1) ? 1 - x + ip : x - ip, 0, 1);
    }
    return clampf(x, 0, 1);
}

__device__ __forceinline__ Vec3 texel2(const float* base, int w, int x, int y) {
    const float* p = base + (size_t(y) * w + x) * 3;
    return Vec3(__ldg(p), __ldg(p + 1), __ldg(p + 2));
}

// A solid image's 3D lookup (defined after the 3D filter).
__device__ Vec3 solid_sample(const Scene& S, int t3, Vec3 p);

// Texture2D::sample_spectrum.  With SOLID, a solid image reads its 3D
// texture at (u, v, 0) (solid_image.cpp:12-15), or at `pos` where the
// material samples by intersection (solid_image.cpp:25-33); lookups that
// never meet a solid image (the environment map) pass SOLID = false.
template <bool SOLID>
__device__ __forceinline__ Vec3 tex2d_lookup(const Scene& S, int ti, float u0, float v0, Vec3 pos, bool at_pos) {
    const Texture2D& t = S.tex2d[ti];
    if (t.type == 0) return Vec3(t.texel[0], t.texel[1], t.texel[2]);
    if (SOLID && t.type == ATRC_TEX_SOLID && at_pos) return solid_sample(S, t.tex3d, pos);
    const float tu = t.uv[0] * u0 + t.uv[1] * v0 + t.uv[2];
    const float tv = t.uv[3] * u0 + t.uv[4] * v0 + t.uv[5];
    const float u = wrap_coord(t.wrap_u, tu), v = wrap_coord(t.wrap_v, tv);
    if (SOLID && t.type == ATRC_TEX_SOLID) return solid_sample(S, t.tex3d, Vec3(u, v, 0.0f));
    const float* base = S.texels + t.data_offset;
    Vec3 r;
    if (t.type == ATRC_TEX_CHECKER) {  // CheckerBoard::sample_spectrum_impl (checker_board.cpp:15-22)
        const int ui = int(clampf(u, 0, 1) / t.grid_size), vi = int(clampf(v, 0, 1) / t.grid_size);
        r = ((ui + vi) & 1) ? Vec3(t.texel[0], t.texel[1], t.texel[2]) : Vec3(t.texel2[0], t.texel2[1], t.texel2[2]);
    } else if (t.nearest) {
        r = texel2(base, t.width, min(int(u * t.width), t.width - 1), min(int(v * t.height), t.height - 1));
    } else {
        const float fx = u * t.width - 0.5f, fy = v * t.height - 0.5f;
        const float flx = floorf(fx), fly = floorf(fy);
        int x0 = int(flx), y0 = int(fly);
        const float ax = fx - flx, ay = fy - fly;
        const int x1 = max(min(x0 + 1, t.width - 1), 0), y1 = max(min(y0 + 1, t.height - 1), 0);
        x0 = max(x0, 0);
        y0 = max(y0, 0);
        const Vec3 a = texel2(base, t.width, x0, y0) * (1 - ax) + texel2(base, t.width, x1, y0) * ax;
        const Vec3 b = texel2(base, t.width, x0, y1) * (1 - ax) + texel2(base, t.width, x1, y1) * ax;
        r = a * (1 - ay) + b * ay;
    }
    if (t.inv_gamma != 1.0f) r = Vec3(powf(r.x, t.inv_gamma), powf(r.y, t.inv_gamma), powf(r.z, t.inv_gamma));
    return r;
}

__device__ __forceinline__ Vec3 tex2d_sample(const Scene& S, int ti, float u, float v) {
    return tex2d_lookup<true>(S, ti, u, v, Vec3(), false);
}

__device__ __forceinline__ float tex3d_at(const float* base, const Texture3D& t, int x, int y, int z, int c) {
    return __ldg(base + ((size_t(z) * t.height + y) * t.width + x) * t.channels + (t.channels == 3 ? c : 0));
}

template <bool REAL_ONLY>
__device__ Vec3 tex3d_sample(const Scene& S, int ti, Vec3 uvw0) {
    const Texture3D& t = S.tex3d[ti];
    if (t.type == 0) return Vec3(t.texel[0], t.texel[1], t.texel[2]);
    const Vec3 p = apply_point_rn(t.uvw, uvw0);
    const float u = wrap_coord(t.wrap[0], p.x), v = wrap_coord(t.wrap[1], p.y), w = wrap_coord(t.wrap[2], p.z);
    const float* base = S.texels + t.data_offset;
    const int nc = REAL_ONLY ? 1 : 3;
    Vec3 r;
    if (t.nearest) {
        const int x = min(int(u * t.width), t.width - 1), y = min(int(v * t.height), t.height - 1),
                  z = min(int(w * t.depth), t.depth - 1);
        for (int c = 0; c < nc; ++c) r[c] = tex3d_at(base, t, x, y, z, c);
        if (REAL_ONLY) r.y = r.z = r.x;
    } else {
        const float f[3] = {u * t.width - 0.5f, v * t.height - 0.5f, w * t.depth - 0.5f};
        const int size[3] = {t.width, t.height, t.depth};
        int i0[3], i1[3];
        float a[3];
        for (int k = 0; k < 3; ++k) {
            const float fl = floorf(f[k]);
            a[k] = f[k] - fl;
            i0[k] = min(max(int(fl), 0), size[k] - 1);
            i1[k] = max(min(int(fl) + 1, size[k] - 1), 0);
        }
        for (int c = 0; c < nc; ++c) {
            const float c00 = tex3d_at(base, t, i0[0], i0[1], i0[2], c) * (1 - a[0]) + tex3d_at(base, t, i1[0], i0[1], i0[2], c) * a[0];
            const float c10 = tex3d_at(base, t, i0[0], i1[1], i0[2], c) * (1 - a[0]) + tex3d_at(base, t, i1[0], i1[1], i0[2], c) * a[0];
            const float c01 = tex3d_at(base, t, i0[0], i0[1], i1[2], c) * (1 - a[0]) + tex3d_at(base, t, i1[0], i0[1], i1[2], c) * a[0];
            const float c11 = tex3d_at(base, t, i0[0], i1[1], i1[2], c) * (1 - a[0]) + tex3d_at(base, t, i1[0], i1[1], i1[2], c) * a[0];
            const float c0 = c00 * (1 - a[1]) + c10 * a[1];
            const float c1 = c01 * (1 - a[1]) + c11 * a[1];
            r[c] = c0 * (1 - a[2]) + c1 * a[2];
        }
        if (REAL_ONLY) r.y = r.z = r.x;
    }
    if (t.inv_gamma != 1.0f) r = Vec3(powf(r.x, t.inv_gamma), powf(r.y, t.inv_gamma), powf(r.z, t.inv_gamma));
    return r;
}

__device__ Vec3 solid_sample(const Scene& S, int t3, Vec3 p) { return tex3d_sample<false>(S, t3, p); }

// ====================================================== surface interaction
struct Surface {
    Vec3 pos;
    float u, v;       // texture coordinates
    Coord geo, user;
    Vec3 wr;
    int32_t entity;
};

__device__ __forceinline__ void sphere_uv_coord(Vec3 p, float radius, float eps, float* u, float* v, Coord* c) {
    float phi = (p.x == 0.0f && p.y == 0.0f) ? 0.0f : atan2f(p.y, p.x);
    if (phi < 0) phi += 2 * kPi;
    const float st = clampf(p.z / radius, -1, 1);
    const float theta = asinf(st);
    *u = 0.5f * kInvPi * phi;
    *v = kInvPi * theta + 0.5f;
    Vec3 ex, ey, ez = normalize(p);
    if (fabsf(ez.z - 1) < eps) { ex = Vec3(1, 0, 0); ey = Vec3(0, 1, 0); ez = Vec3(0, 0, 1); }
    else if (fabsf(ez.z + 1) < eps) { ex = Vec3(0, 1, 0); ey = Vec3(1, 0, 0); ez = Vec3(0, 0, -1); }
    else { ex = cross(Vec3(0, 0, 1), ez); ey = cross(ez, ex); }
    *c = Coord{ex, ey, ez};
}

__device__ __forceinline__ void disk_point(Vec3 pos, float rad, float radius, float* u, float* v, Coord* c) {
    *u = phi_of(pos) / (2 * kPi);
    *v = rad / radius;
    const Vec3 cx = normalize(Vec3(pos.x, pos.y, 0)), cz(0, 0, 1);
    *c = Coord{cx, cross(cz, cx), cz};
}

// Rebuild the intersection record of a hit (GeometryIntersection).
__device__ Surface make_surface(const Scene& S, const Hit& h, Vec3 wo, Vec3 wd) {
    const Entity& e = S.entities[h.entity];
    Surface s;
    s.entity = h.entity;
    Vec3 lo, ld;
    to_entity_space(e, wo, wd, &lo, &ld);
    Vec3 p = lo + h.t * ld;
    if (e.kind == LEAF_TRIANGLES) {
        const TriShade& sh = S.tri_shade[h.tri];
        const Vec3 x(sh.x[0], sh.x[1], sh.x[2]), z(sh.z[0], sh.z[1], sh.z[2]);
        s.geo = Coord{x, cross(z, x), z};
        s.u = sh.t_a[0] + h.u * sh.t_ba[0] + h.v * sh.t_ca[0];
        s.v = sh.t_a[1] + h.u * sh.t_ba[1] + h.v * sh.t_ca[1];
        if (sh.pad[0] != 0.0f) {
            s.user = s.geo;
        } else {
            const Vec3 nz = Vec3(sh.n_a[0], sh.n_a[1], sh.n_a[2]) + h.u * Vec3(sh.n_ba[0], sh.n_ba[1], sh.n_ba[2]) +
                            h.v * Vec3(sh.n_ca[0], sh.n_ca[1], sh.n_ca[2]);
            s.user = rotate_to_new_z(s.geo, nz);
        }
    } else if (e.kind == LEAF_SPHERE) {
        sphere_uv_coord(p, e.radius, S.eps, &s.u, &s.v, &s.geo);
        s.user = s.geo;
    } else {
        const float rad = sqrtf(p.x * p.x + p.y * p.y);
        disk_point(p, rad, e.radius, &s.u, &s.v, &s.geo);
        s.user = s.geo;
    }
    if (e.flags & ENT_LOCAL) {
        p = apply_point_rn(e.local_m, p);
        s.geo = xform_coord(e.local_m, s.geo);
        s.user = xform_coord(e.local_m, s.user);
    }
    if (e.flags & ENT_WRAP) {
        p = apply_point_rn(e.wrap_m, p);
        s.geo = xform_coord(e.wrap_m, s.geo);
        s.user = xform_coord(e.wrap_m, s.user);
    }
    s.pos = p;
    s.wr = -wd;
    if ((e.flags & ENT_DOUBLE_SIDED) && dot(s.geo.z, s.wr) < 0) {
        s.geo = s.geo.neg();
        s.user = s.user.neg();
    }
    return s;
}

__device__ __forceinline__ Vec3 eps_offset(const Surface& s, Vec3 d, float eps) {
    return dot(d, s.geo.z) > 0 ? s.pos + s.geo.z * eps : s.pos - s.geo.z * eps;
}
__device__ __forceinline__ int medium_of(const Surface& s, const Entity& e, Vec3 d) {
    return dot(d, s.geo.z) >= 0 ? e.med_out : e.med_in;
}

// ==================================================================== BSDF
struct BSDFSample {
    Vec3 dir, f;
    float pdf;
    bool delta;
};

struct BSDF {
    int type;
    Coord geo, shd;
    Vec3 albedo;
    // disney
    Vec3 C, Ctint, spec_scale;
    float metallic, roughness, spec_tint, sheen, sheen_tint, clearcoat, transmission, IOR;
    float trans_ax, trans_ay, ax, ay, cc_rough;
    float w_diffuse, w_specular, w_clearcoat, w_transmission;
    float eps;
    bool disney_fixed;  // sample the diffuse lobe instead of falling through
    // mirror / metal: conductor Fresnel (eta_in / eta_out)^2, (k / eta_out)^2
    // and the colour it is multiplied with
    Vec3 eta2, etak2, rc;
    // glass: ior (inside), reflection and refraction colours
    float glass_ior;
    Vec3 refl_c, refr_c;
    // phong: diffuse and specular colours, exponent, component weights
    Vec3 pd, ps;
    float pns, wd, wsp;
    // separable subsurface exit (kMatSeparable): eta in IOR, 1 - 2 FM1(1/eta)
    float sep_ci;
};

// BSDF of the exit point of a subsurface walk (SeparableBSDF, separable.cpp:38-103);
// not a material of the scene description.
constexpr int kMatSeparable = 100;

__device__ __forceinline__ float one_minus_5(float x) { const float t = 1 - x, t2 = t * t; return t2 * t2 * t; }
__device__ __forceinline__ float cos_2_sin(float c) { return sqrtf(fmaxf(0.0f, 1 - c * c)); }
__device__ __forceinline__ float tan_theta(Vec3 w) { const float t = 1 - w.z * w.z; return t <= 0 ? 0.0f : sqrtf(t) / w.z; }
// sin / cos of local_angle::phi(w) without the angle
__device__ __forceinline__ void sincos_phi(Vec3 w, float* s, float* c) {
    const float r2 = w.x * w.x + w.y * w.y;
    if (r2 == 0.0f) { *s = 0; *c = 1; return; }
    const float ir = rsqrtf(r2);
    *s = w.y * ir;
    *c = w.x * ir;
}

__device__ __forceinline__ float dielectric_fresnel(float eta_i, float eta_o, float ci) {  // reflection.h:54-72
    if (ci < 0) { const float t = eta_i; eta_i = eta_o; eta_o = t; ci = -ci; }
    const float si = sqrtf(fmaxf(0.0f, 1 - ci * ci));
    const float st = eta_o / eta_i * si;
    if (st >= 1) return 1;
    const float ct = sqrtf(fmaxf(0.0f, 1 - st * st));
    const float para = (eta_i * ci - eta_o * ct) / (eta_i * ci + eta_o * ct);
    const float perp = (eta_o * ci - eta_i * ct) / (eta_o * ci + eta_i * ct);
    return 0.5f * (para * para + perp * perp);
}

__device__ __forceinline__ float aniso_gtr2(float sp, float cp, float st, float ct, float ax, float ay) {
    const float A = sqrf(cp / ax) + sqrf(sp / ay);
    const float RD = sqrf(st) * A + sqrf(ct);
    return 1 / (kPi * ax * ay * sqrf(RD));
}
__device__ __forceinline__ float smith_aniso_gtr2(float cp, float sp, float ax, float ay, float tan_t) {
    const float t = sqrf(ax * cp) + sqrf(ay * sp);
    const float lambda = -0.5f + 0.5f * sqrtf(1 + t * sqrf(tan_t));
    return 1 / (1 + lambda);
}
__device__ __forceinline__ float smith_gtr2(float tan_t, float alpha) {
    if (tan_t == 0.0f) return 1;
    const float root = alpha * tan_t;
    return 2 / (1 + sqrtf(1 + root * root));
}
__device__ __forceinline__ float gtr1(float st, float ct, float alpha) {
    return (sqrf(alpha) - 1) / (2 * kPi * logf(alpha) * (sqrf(alpha * ct) + sqrf(st)));
}
__device__ __forceinline__ Vec3 sample_aniso_gtr2(float ax, float ay, float u, float v) {
    float s, c;
    sincosf(2 * kPi * u, &s, &c);
    float sp = ay * s, cp = ax * c;
    const float nor = rsqrtf(sqrf(sp) + sqrf(cp));
    sp *= nor;
    cp *= nor;
    const float A = sqrf(cp / ax) + sqrf(sp / ay);
    const float ct = sqrtf(A * (1 - v) / ((1 - A) * v + A));
    const float st = sqrtf(fmaxf(0.0f, 1 - sqrf(ct)));
    return normalize(Vec3(st * cp, st * sp, ct));
}
__device__ __forceinline__ Vec3 sample_gtr1(float alpha, float u, float v) {
    float s, c;
    sincosf(2 * kPi * u, &s, &c);
    const float ct = sqrtf((powf(alpha, 2 - 2 * v) - 1) / (sqrf(alpha) - 1));
    const float st = cos_2_sin(ct);
    return normalize(Vec3(st * c, st * s, ct));
}
__device__ __forceinline__ Vec3 sample_gtr2_vnor(Vec3 ve, float ax, float ay, float u, float v, float eps) {
    const Vec3 vh = normalize(Vec3(ax * ve.x, ay * ve.y, ve.z));
    const float lensq = vh.x * vh.x + vh.y * vh.y;
    const Vec3 t1 = lensq > eps ? Vec3(-vh.y, vh.x, 0) * rsqrtf(lensq) : Vec3(1, 0, 0);
    const Vec3 t2 = cross(vh, t1);
    const float r = sqrtf(u);
    float s, c;
    sincosf(2 * kPi * v, &s, &c);
    const float ta = r * c, tb0 = r * s;
    const float sw = 0.5f * (1 + vh.z);
    const float tb = (1 - sw) * sqrtf(1 - ta * ta) + sw * tb0;
    const Vec3 nh = ta * t1 + tb * t2 + sqrtf(fmaxf(0.0f, 1 - ta * ta - tb * tb)) * vh;
    return normalize(Vec3(ax * nh.x, ay * nh.y, fmaxf(0.0f, nh.z)));
}

__device__ __forceinline__ bool fringes(const BSDF& b, Vec3 w) { return b.shd.positive(w) != b.geo.positive(w); }
__device__ __forceinline__ float normal_corr(const BSDF& b, Vec3 wi) {
    const float dem = fabsf(cosv(b.geo.z, wi));
    return dem < b.eps ? 1.0f : fabsf(cosv(b.shd.z, wi) / dem);
}

// ConductorPoint::eval (fresnel_point.h:44-64), per channel
__device__ __forceinline__ Vec3 conductor_fresnel(const BSDF& b, float ci) {
    if (ci <= 0) return Vec3();
    const float cos2 = ci * ci, sin2 = fmaxf(0.0f, 1 - cos2);
    const float e2[3] = {b.eta2.x, b.eta2.y, b.eta2.z}, k2[3] = {b.etak2.x, b.etak2.y, b.etak2.z};
    float r[3];
    for (int c = 0; c < 3; ++c) {
        const float t0 = e2[c] - k2[c] - sin2;
        const float a2b2 = sqrtf(t0 * t0 + 4 * e2[c] * k2[c]);
        const float t1 = a2b2 + cos2;
        const float a = sqrtf(0.5f * (a2b2 + t0));
        const float t2 = 2 * ci * a;
        const float rs = (t1 - t2) / (t1 + t2);
        const float t3 = cos2 * a2b2 + sin2 * sin2;
        const float t4 = t2 * sin2;
        const float rp = rs * (t3 - t4) / (t3 + t4);
        r[c] = 0.5f * (rp + rs);
    }
    return Vec3(r[0], r[1], r[2]);
}

// GGXMicrofacetReflectionComponent::eval / pdf (microfacet_refl_comp.cpp:9-55);
// the Fresnel term is the coloured conductor of `metal`.
__device__ __forceinline__ void ggx_refl(const BSDF& b, Vec3 lwi, Vec3 lwo, Vec3* f, float* pdf) {
    if (lwi.z <= 0 || lwo.z <= 0) {
        if (f) *f = Vec3();
        if (pdf) *pdf = 0;
        return;
    }
    const Vec3 lwh = normalize(lwi + lwo);
    const float cd = dot(lwi, lwh);
    float sph, cph, spi, cpi, spo, cpo;
    sincos_phi(lwh, &sph, &cph);
    sincos_phi(lwi, &spi, &cpi);
    sincos_phi(lwo, &spo, &cpo);
    const float D = aniso_gtr2(sph, cph, cos_2_sin(lwh.z), lwh.z, b.ax, b.ay);
    const float Gi = smith_aniso_gtr2(cpi, spi, b.ax, b.ay, tan_theta(lwi));
    const float Go = smith_aniso_gtr2(cpo, spo, b.ax, b.ay, tan_theta(lwo));
    if (f) *f = b.rc * conductor_fresnel(b, cd) * (D * Gi * Go / fabsf(4 * lwi.z * lwo.z));
    if (pdf) *pdf = Go * D / (4 * lwo.z);
}

// PhongSpecularComponent (phong_specular_comp.cpp:7-96): s (e+1)/2pi cos^e of
// the angle to the mirror direction (a negative cosine with a fractional
// exponent gives NaN, as in the reference)
__device__ __forceinline__ float pow_cos_pdf(float e, float c) { return (e + 1) / (2 * kPi) * powf(c, e); }
__device__ __forceinline__ Vec3 phong_spec_eval(const BSDF& b, Vec3 lwi, Vec3 lwo) {
    if (lwi.z <= 0 || lwo.z <= 0) return Vec3();
    const Vec3 ideal(-lwo.x, -lwo.y, lwo.z);  // refl_aux::reflect(lwo, z)
    return b.ps * pow_cos_pdf(b.pns, cosv(ideal, lwi));
}
__device__ __forceinline__ float phong_spec_pdf(const BSDF& b, Vec3 lwi, Vec3 lwo) {
    if (lwi.z <= 0 || lwo.z <= 0) return 0;
    const Vec3 ideal(-lwo.x, -lwo.y, lwo.z);
    const Vec3 l = coord_from_z(ideal).global_to_local(lwi);
    if (l.z <= 0) return 0;
    return pow_cos_pdf(b.pns, normalize(l).z);
}

__device__ void disney_init(BSDF& b, Vec3 base, float met, float rough, float trans, float trans_rough, float ior,
                            Vec3 spec_scale, float spec_tint, float aniso, float sheen, float sheen_tint, float cc,
                            float cc_gloss) {
    b.C = base;
    const float l = lum(base);
    b.Ctint = l > 0 ? base / l : Vec3(1.0f);
    b.metallic = met;
    b.roughness = rough;
    b.spec_scale = spec_scale;
    b.spec_tint = spec_tint;
    b.sheen = sheen;
    b.sheen_tint = sheen_tint;
    b.transmission = trans;
    b.IOR = fmaxf(1.01f, ior);
    const float aspect = aniso > 0 ? sqrtf(1 - 0.9f * aniso) : 1.0f;
    b.ax = fmaxf(0.001f, sqrf(rough) / aspect);
    b.ay = fmaxf(0.001f, sqrf(rough) * aspect);
    b.trans_ax = fmaxf(0.001f, sqrf(trans_rough) / aspect);
    b.trans_ay = fmaxf(0.001f, sqrf(trans_rough) * aspect);
    b.clearcoat = cc;
    float ccr = 0.1f * (1 - cc_gloss);
    ccr *= ccr;
    b.cc_rough = fmaxf(ccr, 0.0001f);
    const float A = clampf(lum(base) * (1 - met), 0.3f, 0.7f), B = 1 - A;
    b.w_diffuse = A * (1 - trans);
    b.w_transmission = A * trans;
    b.w_specular = B * 2 / (2 + cc);
    b.w_clearcoat = B * cc / (2 + cc);
    b.albedo = base;
}

__device__ Vec3 disney_f_trans(const BSDF& b, Vec3 lwi, Vec3 lwo) {
    const float ci = lwi.z, co = lwo.z;
    const float eta = co > 0 ? b.IOR : 1 / b.IOR;
    Vec3 lwh = normalize(lwo + eta * lwi);
    if (lwh.z < 0) lwh = -lwh;
    const float cd = dot(lwo, lwh);
    const float F = dielectric_fresnel(b.IOR, 1, cd);
    float sph, cph, spi, cpi, spo, cpo;
    sincos_phi(lwh, &sph, &cph);
    sincos_phi(lwi, &spi, &cpi);
    sincos_phi(lwo, &spo, &cpo);
    const float D = aniso_gtr2(sph, cph, cos_2_sin(lwh.z), lwh.z, b.trans_ax, b.trans_ay);
    const float G = smith_aniso_gtr2(cpi, spi, b.trans_ax, b.trans_ay, tan_theta(lwi)) *
                    smith_aniso_gtr2(cpo, spo, b.trans_ax, b.trans_ay, tan_theta(lwo));
    const float sdem = cd + eta * dot(lwi, lwh);
    const float corr = 1 / eta;
    const float val = (1 - F) * D * G * eta * eta * dot(lwi, lwh) * dot(lwo, lwh) * corr * corr / (ci * co * sdem * sdem);
    const float tf = co > 0 ? b.transmission : 1.0f;
    return (1 - b.metallic) * tf * Vec3(sqrtf(b.C.x), sqrtf(b.C.y), sqrtf(b.C.z)) * fabsf(val);
}

__device__ Vec3 disney_f_inner(const BSDF& b, Vec3 lwi, Vec3 lwo) {
    const Vec3 lwh = -normalize(lwi + lwo);
    const float F = dielectric_fresnel(b.IOR, 1, dot(lwo, lwh));
    float sph, cph, spi, cpi, spo, cpo;
    sincos_phi(lwh, &sph, &cph);
    sincos_phi(lwi, &spi, &cpi);
    sincos_phi(lwo, &spo, &cpo);
    const float D = aniso_gtr2(sph, cph, cos_2_sin(lwh.z), lwh.z, b.trans_ax, b.trans_ay);
    const float G = smith_aniso_gtr2(cpi, spi, b.trans_ax, b.trans_ay, tan_theta(lwi)) *
                    smith_aniso_gtr2(cpo, spo, b.trans_ax, b.trans_ay, tan_theta(lwo));
    return b.transmission * b.C * fabsf(F * D * G / (4 * lwi.z * lwo.z));
}

__device__ __forceinline__ bool is_aggregate(int type) { return type == ATRC_MAT_METAL || type == ATRC_MAT_PHONG; }

// SeparableBSDF::eval (separable.cpp:50-60): (1 - Fr(cos wi)) / (c pi) eta^2
// for any wi, below the surface too
__device__ __forceinline__ Vec3 separable_eval(const BSDF& b, Vec3 wi) {
    const float fr = dielectric_fresnel(b.IOR, 1.0f, cosv(wi, b.geo.z));
    return Vec3((1.0f - fr) / (b.sep_ci * kPi) * b.IOR * b.IOR);
}

__device__ Vec3 bsdf_eval(const BSDF& b, Vec3 wi, Vec3 wo) {
    if (b.type == kMatSeparable) return separable_eval(b, wi);
    if (is_aggregate(b.type)) {  // AggregateBSDF::eval (component/aggregate.h)
        if (fringes(b, wi) || fringes(b, wo)) {
            if (!b.geo.positive(wi) || !b.geo.positive(wo)) return Vec3();
            return b.albedo * kInvPi;
        }
        const Vec3 lwi = normalize(b.shd.global_to_local(wi)), lwo = normalize(b.shd.global_to_local(wo));
        if (lwi.z == 0.0f || lwo.z == 0.0f) return Vec3();
        if (b.type == ATRC_MAT_METAL) {
            Vec3 f;
            ggx_refl(b, lwi, lwo, &f, nullptr);
            return f;
        }
        const Vec3 fd = (lwi.z <= 0 || lwo.z <= 0) ? Vec3() : b.pd * kInvPi;
        return fd + phong_spec_eval(b, lwi, lwo);
    }
    if (b.type == ATRC_MAT_IDEAL_DIFFUSE || b.type == ATRC_MAT_DISNEY) {
        if (fringes(b, wi) || fringes(b, wo)) {
            if (!b.geo.positive(wi) || !b.geo.positive(wo)) return Vec3();
            return b.albedo * kInvPi;
        }
        const Vec3 lwi = normalize(b.shd.global_to_local(wi)), lwo = normalize(b.shd.global_to_local(wo));
        if (b.type == ATRC_MAT_IDEAL_DIFFUSE) {
            if (lwi.z <= 0 || lwo.z <= 0) return Vec3();
            return b.albedo * kInvPi;
        }
        if (fabsf(lwi.z) < b.eps || fabsf(lwo.z) < b.eps) return Vec3();
        if (lwi.z * lwo.z < 0) {
            if (b.transmission == 0.0f) return Vec3();
            return disney_f_trans(b, lwi, lwo) * normal_corr(b, wi);
        }
        if (lwi.z < 0 && lwo.z < 0) {
            if (b.transmission == 0.0f) return Vec3();
            return disney_f_inner(b, lwi, lwo) * normal_corr(b, wi);
        }
        if (lwi.z <= 0 || lwo.z <= 0) return Vec3();
        const float ci = lwi.z, co = lwo.z;
        const Vec3 lwh = normalize(lwi + lwo);
        const float cd = dot(lwi, lwh);
        Vec3 diffuse, sheen;
        if (b.metallic < 1) {
            const float FL = one_minus_5(ci), FV = one_minus_5(co);
            const float RR = 2 * b.roughness * cd * cd;
            const Vec3 lam = b.C * kInvPi;
            diffuse = lam * (1 - 0.5f * FL) * (1 - 0.5f * FV) + lam * (RR * (FL + FV + FL * FV * (RR - 1)));
            if (b.sheen > 0) sheen = 4 * b.sheen * mix(Vec3(1.0f), b.Ctint, b.sheen_tint) * one_minus_5(cd);
        }
        // f_specular (disney.cpp:213-249)
        const Vec3 Cspec = mix(mix(Vec3(1.0f), b.Ctint, b.spec_tint), b.C, b.metallic);
        const float fd = one_minus_5(cd);
        const Vec3 diel = Cspec * dielectric_fresnel(b.IOR, 1, cd);
        const Vec3 cond = Cspec + (Vec3(1.0f) - Cspec) * fd;
        const Vec3 F = mix(b.spec_scale * diel, cond, b.metallic);
        float sph, cph, spi, cpi, spo, cpo;
        sincos_phi(lwh, &sph, &cph);
        sincos_phi(lwi, &spi, &cpi);
        sincos_phi(lwo, &spo, &cpo);
        const float ch = lwh.z, sh = cos_2_sin(ch);
        const float ti = tan_theta(lwi), to = tan_theta(lwo);
        const float D = aniso_gtr2(sph, cph, sh, ch, b.ax, b.ay);
        const float G = smith_aniso_gtr2(cpi, spi, b.ax, b.ay, ti) * smith_aniso_gtr2(cpo, spo, b.ax, b.ay, to);
        const Vec3 specular = F * (D * G / fabsf(4 * ci * co));
        Vec3 cc;
        if (b.clearcoat > 0) {
            const float Dc = gtr1(sh, ch, b.cc_rough);
            const float Fc = 0.04f + (1 - 0.04f) * fd;
            const float Gc = smith_gtr2(ti, 0.25f) * smith_gtr2(to, 0.25f);
            cc = Vec3(b.clearcoat * Dc * Fc * Gc / fabsf(4 * ci * co));
        }
        const Vec3 value = (1 - b.metallic) * (1 - b.transmission) * (diffuse + sheen) + specular + cc;
        return value * normal_corr(b, wi);
    }
    return Vec3();
}

__device__ float disney_pdf_trans(const BSDF& b, Vec3 lwi, Vec3 lwo) {
    const float eta = lwo.z > 0 ? b.IOR : 1 / b.IOR;
    Vec3 lwh = normalize(lwo + eta * lwi);
    if (lwh.z < 0) lwh = -lwh;
    if (((lwo.z > 0) != (dot(lwh, lwo) > 0)) || ((lwi.z > 0) != (dot(lwh, lwi) > 0))) return 0;
    const float sdem = dot(lwo, lwh) + eta * dot(lwi, lwh);
    const float dwh_dwi = eta * eta * dot(lwi, lwh) / (sdem * sdem);
    float sph, cph;
    sincos_phi(lwh, &sph, &cph);
    const float D = aniso_gtr2(sph, cph, cos_2_sin(lwh.z), lwh.z, b.trans_ax, b.trans_ay);
    return fabsf(lwh.z * D * dwh_dwi);
}

__device__ float bsdf_pdf(const BSDF& b, Vec3 wi, Vec3 wo) {
    if (b.type == kMatSeparable) return zweighted_pdf(normalize(b.geo.global_to_local(wi)).z);
    if (b.type != ATRC_MAT_IDEAL_DIFFUSE && b.type != ATRC_MAT_DISNEY && !is_aggregate(b.type)) return 0;
    if (fringes(b, wi) || fringes(b, wo)) {
        if (b.geo.positive(wi) != b.geo.positive(wo)) return 0;
        return zweighted_pdf(normalize(b.geo.global_to_local(wi)).z);
    }
    const Vec3 lwi = normalize(b.shd.global_to_local(wi)), lwo = normalize(b.shd.global_to_local(wo));
    if (is_aggregate(b.type)) {  // sum of weighted component pdfs / sum of weights
        if (lwi.z == 0.0f || lwo.z == 0.0f) return 0;
        if (b.type == ATRC_MAT_METAL) {
            float pdf;
            ggx_refl(b, lwi, lwo, nullptr, &pdf);
            return pdf;
        }
        const float pdd = (lwi.z <= 0 || lwo.z <= 0) ? 0.0f : zweighted_pdf(lwi.z);
        const float wsum = b.wd + b.wsp;
        return wsum > 0 ? (b.wd * pdd + b.wsp * phong_spec_pdf(b, lwi, lwo)) / wsum : 0.0f;
    }
    if (b.type == ATRC_MAT_IDEAL_DIFFUSE) {
        if (lwi.z <= 0 || lwo.z <= 0) return 0;
        return zweighted_pdf(lwi.z);
    }
    if (fabsf(lwi.z) < b.eps || fabsf(lwo.z) < b.eps) return 0;
    if (lwo.z < 0) {
        if (b.transmission == 0.0f) return 0;
        const float mF = clampf(dielectric_fresnel(b.IOR, 1, lwo.z), 0.1f, 0.9f);
        if (lwi.z > 0) return (1 - mF) * disney_pdf_trans(b, lwi, lwo);
        // pdf_inner_refl (disney.cpp:386-401)
        const Vec3 lwh = -normalize(lwi + lwo);
        float sph, cph;
        sincos_phi(lwh, &sph, &cph);
        const float D = aniso_gtr2(sph, cph, cos_2_sin(lwh.z), lwh.z, b.trans_ax, b.trans_ay);
        return mF * fabsf(lwh.z * D / (4 * dot(lwi, lwh)));
    }
    if (lwi.z < 0) return b.w_transmission * disney_pdf_trans(b, lwi, lwo);
    // pdf_diffuse + pdf_specular_clearcoat (disney.cpp:328-356)
    const Vec3 lwh = normalize(lwi + lwo);
    float sph, cph, spo, cpo;
    sincos_phi(lwh, &sph, &cph);
    sincos_phi(lwo, &spo, &cpo);
    spo = cos_2_sin(cpo);
    const float ch = lwh.z, sh = cos_2_sin(ch);
    const float cd = dot(lwi, lwh);
    const float sD = aniso_gtr2(sph, cph, sh, ch, b.ax, b.ay);
    const float ps = smith_aniso_gtr2(cpo, spo, b.ax, b.ay, tan_theta(lwo)) * sD / (4 * lwo.z);
    const float cD = gtr1(sh, ch, b.cc_rough);
    const float pc = ch * cD / (4 * cd);
    return b.w_diffuse * zweighted_pdf(lwi.z) + b.w_specular * ps + b.w_clearcoat * pc;
}

__device__ BSDFSample bsdf_sample(const BSDF& b, Vec3 wo, float u0, float u1, float u2) {
    BSDFSample r;
    r.dir = Vec3();
    r.f = Vec3();
    r.pdf = 0;
    r.delta = false;
    if (b.type == ATRC_MAT_INVISIBLE_SURFACE) {
        const float c = fabsf(cosv(b.geo.z, wo));
        r.dir = -wo;
        r.f = Vec3(1.0f / (c < b.eps ? 1.0f : c));
        r.pdf = 1;
        r.delta = true;
        return r;
    }
    if (b.type == kMatSeparable) {  // SeparableBSDF::sample (separable.cpp:62-69)
        float pdf;
        const Vec3 lwi = zweighted_on_hemisphere(u0, u1, &pdf);
        r.dir = b.geo.local_to_global(lwi);
        r.f = separable_eval(b, r.dir);
        r.pdf = pdf;
        return r;
    }
    if (b.type == ATRC_MAT_MIRROR) {  // MirrorBSDF::sample (mirror.cpp:32-50)
        const Vec3 lo = b.shd.global_to_local(wo);
        if (lo.z <= 0) return r;
        const Vec3 nwo = normalize(lo);
        const Vec3 dir = b.shd.local_to_global(Vec3(0, 0, 2 * nwo.z) - nwo);
        r.dir = dir;
        r.f = conductor_fresnel(b, nwo.z) * b.rc / fabsf(nwo.z) * normal_corr(b, dir);
        r.pdf = 1;
        r.delta = true;
        return r;
    }
    if (b.type == ATRC_MAT_GLASS) {  // GlassBSDF::sample (glass.cpp:52-91), radiance transport
        const Vec3 nwo = normalize(b.shd.global_to_local(wo));
        const Vec3 nor = nwo.z > 0 ? Vec3(0, 0, 1) : Vec3(0, 0, -1);
        const float fr = dielectric_fresnel(b.glass_ior, 1.0f, nwo.z);
        if (u0 < fr) {
            const Vec3 lwi(-nwo.x, -nwo.y, nwo.z);
            const Vec3 wi = b.shd.local_to_global(lwi);
            r.dir = wi;
            r.f = b.refl_c * fr / fabsf(lwi.z) * normal_corr(b, wi);
            r.pdf = fr;
            r.delta = true;
            return r;
        }
        const float eta_i = nwo.z > 0 ? 1.0f : b.glass_ior, eta_t = nwo.z > 0 ? b.glass_ior : 1.0f;
        const float eta = eta_i / eta_t;
        const float ci = fabsf(nwo.z);
        const float st2 = eta * eta * fmaxf(0.0f, 1 - ci * ci);
        if (st2 >= 1) return r;
        const float ct = sqrtf(1 - st2);
        const Vec3 nwi = normalize((eta * ci - ct) * nor - eta * nwo);
        const Vec3 dir = b.shd.local_to_global(nwi);
        r.dir = dir;
        r.f = eta * eta * b.refr_c * (1 - fr) / fabsf(nwi.z) * normal_corr(b, dir);
        r.pdf = 1 - fr;
        r.delta = true;
        return r;
    }
    if (is_aggregate(b.type)) {  // AggregateBSDF::sample (component/aggregate.h)
        if (fringes(b, wo)) {
            if (!b.geo.positive(wo)) return r;
            float pdf;
            const Vec3 lwi = zweighted_on_hemisphere(u0, u1, &pdf);
            if (pdf < b.eps) return r;
            const Vec3 wi = normalize(b.geo.local_to_global(lwi));
            r.dir = wi;
            r.f = b.albedo * kInvPi * normal_corr(b, wi);
            r.pdf = pdf;
            return r;
        }
        const Vec3 lwo = normalize(b.shd.global_to_local(wo));
        if (lwo.z == 0.0f) return r;
        const bool metal = b.type == ATRC_MAT_METAL;
        const float w0 = metal ? 1.0f : b.wd, w1 = metal ? 0.0f : b.wsp;
        const int ncomp = metal ? 1 : 2;
        float sel = (u0 - 0.001f) * (w0 + w1);
        int comp = -1;
        if (sel <= w0) comp = 0;
        else if (ncomp > 1 && (sel -= w0) <= w1) comp = 1;
        if (comp < 0) return r;
        Vec3 lwi, f;
        float pdf = 0;
        if (lwo.z <= 0) return r;
        if (metal) {
            const Vec3 lwh = normalize(sample_gtr2_vnor(lwo, b.ax, b.ay, u1, u2, b.eps));
            if (lwh.z <= 0) return r;
            lwi = normalize(2 * dot(lwo, lwh) * lwh - lwo);
            if (lwi.z <= 0) return r;
            ggx_refl(b, lwi, lwo, &f, &pdf);
        } else if (comp == 0) {  // DiffuseComponent::sample
            lwi = zweighted_on_hemisphere(u1, u2, &pdf);
            if (pdf < 0.001f) return r;
            f = b.pd * kInvPi;
        } else {  // PhongSpecularComponent::sample
            const Vec3 ideal(-lwo.x, -lwo.y, lwo.z);
            const float ct = powf(u1, 1 / (b.pns + 1));
            const float st = cos_2_sin(ct);
            float sp, cp;
            sincosf(2 * kPi * u2, &sp, &cp);
            const Vec3 local = normalize(Vec3(st * cp, st * sp, ct));
            lwi = normalize(coord_from_z(ideal).local_to_global(local));
            if (lwi.z <= 0) return r;
            pdf = pow_cos_pdf(b.pns, local.z);
            f = phong_spec_eval(b, lwi, lwo);
        }
        if (!(pdf > 0)) return r;
        lwi = normalize(lwi);
        pdf *= comp == 0 ? w0 : w1;
        if (!metal) {  // the other component
            if (comp == 0) {
                f += phong_spec_eval(b, lwi, lwo);
                pdf += phong_spec_pdf(b, lwi, lwo) * w1;
            } else {
                f += (lwi.z <= 0 || lwo.z <= 0) ? Vec3() : b.pd * kInvPi;
                pdf += ((lwi.z <= 0 || lwo.z <= 0) ? 0.0f : zweighted_pdf(lwi.z)) * w0;
            }
        }
        const Vec3 wi = b.shd.local_to_global(lwi);
        r.dir = wi;
        r.f = f * normal_corr(b, wi);
        r.pdf = pdf;
        return r;
    }
    if (b.type != ATRC_MAT_IDEAL_DIFFUSE && b.type != ATRC_MAT_DISNEY) return r;
    if (fringes(b, wo)) {  // LocalBSDF::sample_black_fringes
        if (!b.geo.positive(wo)) return r;
        float pdf;
        const Vec3 lwi = zweighted_on_hemisphere(u0, u1, &pdf);
        if (pdf < b.eps) return r;
        const Vec3 wi = normalize(b.geo.local_to_global(lwi));
        r.dir = wi;
        r.f = b.albedo * kInvPi * normal_corr(b, wi);
        r.pdf = pdf;
        return r;
    }
    const Vec3 lwo = normalize(b.shd.global_to_local(wo));
    if (b.type == ATRC_MAT_IDEAL_DIFFUSE) {
        if (lwo.z == 0.0f) return r;
        if (!((u0 - 0.001f) <= 1.0f)) return r;  // component selector
        if (lwo.z <= 0) return r;
        float pdf;
        const Vec3 lwi = normalize(zweighted_on_hemisphere(u1, u2, &pdf));
        if (pdf < 0.001f) return r;
        const Vec3 wi = b.shd.local_to_global(lwi);
        r.dir = wi;
        r.f = b.albedo * kInvPi * normal_corr(b, wi);
        r.pdf = pdf;
        return r;
    }
    // Disney (disney.cpp:546-612)
    if (fabsf(lwo.z) < b.eps) return r;
    Vec3 lwi;
    bool ok = false;
    if (lwo.z < 0) {
        if (b.transmission == 0.0f) return r;
        const float mF = clampf(dielectric_fresnel(b.IOR, 1, lwo.z), 0.1f, 0.9f);
        if (u0 >= mF) {
            goto sample_trans;
        } else {
            const Vec3 lwh = sample_aniso_gtr2(b.trans_ax, b.trans_ay, u1, u2);
            if (lwh.z <= 0) return r;
            const Vec3 t = 2 * dot(lwo, lwh) * lwh - lwo;
            if (t.z > 0) return r;
            lwi = normalize(t);
            ok = true;
            goto done;
        }
    } else {
        // the diffuse choice is always overwritten (disney.cpp:578-589),
        // unless the fixed sampling mode is on
        float sel = u0;
        if (b.disney_fixed && sel < b.w_diffuse) {
            float pdf;
            lwi = zweighted_on_hemisphere(u1, u2, &pdf);
            ok = lwi.z > 0;
            goto done;
        }
        if (!(sel < b.w_diffuse)) sel -= b.w_diffuse;
        if (sel < b.w_transmission) goto sample_trans;
        sel -= b.w_transmission;
        if (sel < b.w_specular) {
            const Vec3 lwh = normalize(sample_gtr2_vnor(lwo, b.ax, b.ay, u1, u2, b.eps));
            if (lwh.z <= 0) return r;
            const Vec3 t = normalize(2 * dot(lwo, lwh) * lwh - lwo);
            if (t.z <= 0) return r;
            lwi = t;
            ok = true;
        } else {
            const Vec3 lwh = sample_gtr1(b.cc_rough, u1, u2);
            if (lwh.z <= 0) return r;
            const Vec3 t = normalize(2 * dot(lwo, lwh) * lwh - lwo);
            if (t.z <= 0) return r;
            lwi = t;
            ok = true;
        }
        goto done;
    }
sample_trans: {
        const Vec3 lwh = sample_aniso_gtr2(b.trans_ax, b.trans_ay, u1, u2);
        if (lwh.z <= 0) return r;
        if ((lwo.z > 0) != (dot(lwh, lwo) > 0)) return r;
        const float eta = lwo.z > 0 ? 1 / b.IOR : b.IOR;
        const Vec3 owh = dot(lwh, lwo) > 0 ? lwh : -lwh;
        const float ci = dot(lwo, owh);
        const float s2t = sqrf(eta) * (1 - sqrf(ci));
        const float c2t = 1 - s2t;
        if (c2t <= 0) return r;
        const Vec3 t = normalize(normalize((eta * ci - sqrtf(c2t)) * owh - eta * lwo));
        if (t.z * lwo.z > 0 || ((t.z > 0) != (dot(lwh, t) > 0))) return r;
        lwi = t;
        ok = true;
    }
done:
    if (!ok || black(lwi)) return r;
    const Vec3 wi = b.shd.local_to_global(lwi);
    r.dir = wi;
    r.f = bsdf_eval(b, wi, wo);
    r.pdf = bsdf_pdf(b, wi, wo);
    return r;
}

__device__ __forceinline__ Vec3 bsdf_albedo(const BSDF& b) {
    if (b.type == ATRC_MAT_INVISIBLE_SURFACE) return Vec3(1.0f);
    if (b.type == ATRC_MAT_IDEAL_BLACK || b.type == kMatSeparable) return Vec3();
    return b.albedo;
}

// ============================================================ subsurface
// Normalized diffusion (Christensen and Burley 2015, "Approximate
// reflectance profiles for efficient subsurface scattering";
// normalized_diffusion.cpp:357-397).  With x = r / d:
//   radial pdf   p(x) = (e^-x + e^-x/3) / 4           (integrates to 1)
//   cdf          P(x) = 1 - e^-x / 4 - 3 e^-x/3 / 4
// and the reference's profile eval_r(r) = A (e^-x + e^-x/3) / (8 pi d), i.e.
// R(r) r, matched to a pdf in r dr dphi / (2 pi).

// First moment of the dielectric Fresnel reflectance (the polynomial fits
// of d'Eon and Irving 2011 used by separable.cpp:12-35).
__device__ __forceinline__ float fresnel_moment1(float eta) {
    const float e2 = eta * eta, e3 = e2 * eta, e4 = e2 * e2, e5 = e2 * e3;
    if (eta < 1)
        return 0.45966f - 1.73965f * eta + 3.37668f * e2 - 3.904945f * e3 + 2.49277f * e4 - 0.68441f * e5;
    return -4.61686f + 11.1136f * eta - 10.4646f * e2 + 5.11455f * e3 - 1.27198f * e4 + 0.12746f * e5;
}

// P^-1(u) by Newton's method in double precision from a start that is
// within a factor of two everywhere (P(x) ~ x / 2 near 0, 1 - 3 e^-x/3 / 4
// far out); u is clamped below 1.
__device__ __forceinline__ float nd_inv_cdf(float uf) {
    const double u = fmin(fmax(double(uf), 0.0), 1.0 - 1e-7);
    double x = u < 0.5 ? 2.0 * u : 3.0 * log(0.75 / (1.0 - u));
    for (int k = 0; k < 24; ++k) {
        const double e1 = exp(-x), e3 = exp(-x / 3.0);
        const double f = 1.0 - 0.25 * e1 - 0.75 * e3 - u;
        const double df = 0.25 * (e1 + e3);
        const double step = f / df;
        x = fmax(x - step, 0.0);
        if (fabs(step) <= 1e-12 * fmax(x, 1e-12)) break;
    }
    return float(x);
}

__device__ __forceinline__ float nd_pdf_r(float d, float r) {  // pdf_r (normalized_diffusion.cpp:380-385)
    const float x = r / d;
    return 0.25f * (expf(-x) + expf(-x / 3.0f)) / d;
}

__device__ __forceinline__ Vec3 nd_eval_r(Vec3 A, Vec3 d, float r) {  // eval_r (normalized_diffusion.cpp:357-362)
    return Vec3(A.x * (expf(-r / d.x) + expf(-r / (3.0f * d.x))) / (8.0f * kPi * d.x),
                A.y * (expf(-r / d.y) + expf(-r / (3.0f * d.y))) / (8.0f * kPi * d.y),
                A.z * (expf(-r / d.z) + expf(-r / (3.0f * d.z))) / (8.0f * kPi * d.z));
}

// Scattering distance d = dmfp / s with s = 3.5 + 100 (A - 0.33)^4
// (NormalizedDiffusionBSSRDF ctor, normalized_diffusion.cpp:388-397).
__device__ __forceinline__ float nd_scale(float a) {
    const float t = a - 0.33f;
    return 3.5f + 100.0f * t * t * t * t;
}

// Material::shade
__device__ BSDF shade(const Scene& S, const Surface& s, Vec3* shading_normal) {
    const Entity& e = S.entities[s.entity];
    const Material& m = S.materials[e.material];
    BSDF b;
    b.type = m.type;
    b.geo = s.geo;
    b.eps = S.eps;
    b.disney_fixed = S.disney_fixed != 0;
    b.albedo = Vec3();
    Coord shd = s.user;
    // every texture slot the material reads, and its normal map last, from
    // one lookup site (the lookup is inlined once; its values stay in tv)
    const bool nmap = m.normal_map >= 0 && (m.type == ATRC_MAT_IDEAL_DIFFUSE || m.type == ATRC_MAT_DISNEY ||
                                            m.type == ATRC_MAT_METAL || m.type == ATRC_MAT_PHONG);
    int nsl = 0;
    if (!m.all_constant) {
        nsl = m.type == ATRC_MAT_DISNEY ? 13 : m.type == ATRC_MAT_IDEAL_DIFFUSE ? 1 : m.type == ATRC_MAT_METAL ? 5
            : (m.type == ATRC_MAT_MIRROR || m.type == ATRC_MAT_GLASS || m.type == ATRC_MAT_PHONG) ? 3 : 0;
    }
    // IdealDiffuse and Glass sample by intersection (ideal_diffuse.cpp:27, glass.cpp:184-192)
    const bool at_pos = m.type == ATRC_MAT_IDEAL_DIFFUSE || m.type == ATRC_MAT_GLASS;
    const int ntex = nsl + (nmap ? 1 : 0);
    Vec3 tv[14];
#pragma unroll 1
    for (int k = 0; k < ntex; ++k)
        tv[k] = tex2d_lookup<true>(S, k < nsl ? m.tex[k] : m.normal_map, s.u, s.v, s.pos, at_pos && k < nsl);
    if (nmap) {
        const Vec3 t = tv[nsl];  // NormalMapper::reorient
        const Vec3 ln = normalize(Vec3(t.x * 2 - 1, t.y * 2 - 1, t.z * 2 - 1));
        shd = rotate_to_new_z(s.user, s.user.local_to_global(ln));
    }
    b.shd = shd;
    *shading_normal = m.type == ATRC_MAT_INVISIBLE_SURFACE || m.type == ATRC_MAT_IDEAL_BLACK ? s.user.z : shd.z;
    if (m.type == ATRC_MAT_IDEAL_DIFFUSE) {
        // IdealDiffuse::shade samples by intersection (ideal_diffuse.cpp:27)
        b.albedo = m.all_constant ? Vec3(m.c[0], m.c[1], m.c[2]) : tv[0];
    } else if (m.type == ATRC_MAT_DISNEY) {
        if (m.all_constant) {
            disney_init(b, Vec3(m.c[0], m.c[1], m.c[2]), m.c[3], m.c[4], m.c[5], m.c[6], m.c[7],
                        Vec3(m.c[8], m.c[9], m.c[10]), m.c[11], m.c[12], m.c[13], m.c[14], m.c[15], m.cc_gloss);
        } else {
            auto T = [&](int slot) { return tv[slot]; };
            disney_init(b, T(ATRC_DISNEY_BASE_COLOR), T(ATRC_DISNEY_METALLIC).x, T(ATRC_DISNEY_ROUGHNESS).x,
                        T(ATRC_DISNEY_TRANSMISSION).x, T(ATRC_DISNEY_TRANSMISSION_ROUGHNESS).x, T(ATRC_DISNEY_IOR).x,
                        T(ATRC_DISNEY_SPECULAR_SCALE), T(ATRC_DISNEY_SPECULAR_TINT).x, T(ATRC_DISNEY_ANISOTROPIC).x,
                        T(ATRC_DISNEY_SHEEN).x, T(ATRC_DISNEY_SHEEN_TINT).x, T(ATRC_DISNEY_CLEARCOAT).x,
                        T(ATRC_DISNEY_CLEARCOAT_GLOSS).x);
        }
    } else if (m.type == ATRC_MAT_MIRROR || m.type == ATRC_MAT_GLASS || m.type == ATRC_MAT_METAL ||
               m.type == ATRC_MAT_PHONG) {
        auto T = [&](int slot) { return tv[slot]; };
        if (m.type == ATRC_MAT_MIRROR) {
            // Mirror::shade (mirror.cpp:98-115): ConductorPoint(ior, 1, k) puts
            // the ior on the OUTER side, so eta^2 = 1 / ior^2
            const Vec3 rc = T(0), ior = T(1), k = T(2);
            b.rc = rc;
            b.eta2 = Vec3(1 / sqrf(ior.x), 1 / sqrf(ior.y), 1 / sqrf(ior.z));
            b.etak2 = Vec3(sqrf(k.x / ior.x), sqrf(k.y / ior.y), sqrf(k.z / ior.z));
            b.albedo = rc;
        } else if (m.type == ATRC_MAT_GLASS) {  // Glass::shade (glass.cpp:180-206), by intersection
            b.glass_ior = T(2).x;
            b.refl_c = T(0);
            const Vec3 rr = T(1);
            b.refr_c = Vec3(sqrtf(rr.x), sqrtf(rr.y), sqrtf(rr.z));
            b.albedo = 0.5f * (b.refl_c + b.refr_c);
        } else if (m.type == ATRC_MAT_METAL) {  // Metal::shade (metal.cpp:39-62)
            const Vec3 color = T(0), eta = T(1), k = T(2);
            const float rough = T(3).x, aniso = T(4).x;
            b.rc = color;  // ColoredConductorPoint(color, 1, eta, k)
            b.eta2 = Vec3(sqrf(eta.x), sqrf(eta.y), sqrf(eta.z));
            b.etak2 = Vec3(sqrf(k.x), sqrf(k.y), sqrf(k.z));
            const float aspect = aniso > 0 ? sqrtf(1 - 0.9f * aniso) : 1.0f;
            b.ax = fmaxf(0.001f, sqrf(rough) / aspect);
            b.ay = fmaxf(0.001f, sqrf(rough) * aspect);
            b.roughness = rough;
            b.albedo = color;
        } else {  // Phong::shade (phong.cpp:33-79)
            Vec3 d = T(0), sp = T(1);
            const float ns = T(2).x;
            const float dem = fmaxf(1.0f, fmaxf(d.x + sp.x, fmaxf(d.y + sp.y, d.z + sp.z)));
            d = d / dem;
            sp = sp / dem;
            const float dl = lum(d), sl = lum(sp);
            b.wd = dl + sl > b.eps ? dl / (dl + sl) : 0.5f;
            b.wsp = 1 - b.wd;
            b.pd = d;
            b.ps = sp;
            b.pns = ns;
            b.albedo = d + sp;
        }
    }
    return b;
}

// ================================================================== lights
struct LightSample {
    Vec3 pos, nor, rad;
    float pdf;
};

// Geometry::sample(ref, ...) of an entity, with transform_wrapper and
// double_sided adapters (transform_wrapper.cpp:101-112, double_sided.cpp:58-78).
__device__ bool entity_sample(const Scene& S, const Entity& e, Vec3 ref, float u, float v, float w, Vec3* pos,
                              Coord* geo, float* pdf) {
    bool back = false;
    if (e.flags & ENT_DOUBLE_SIDED) {
        back = u < 0.5f;
        u = back ? 2 * u : 2 * (u - 0.5f);
    }
    if (e.flags & ENT_WRAP) ref = apply_point_rn(e.wrap_inv, ref);
    Vec3 p;
    Coord c;
    float pd;
    if (e.kind == LEAF_TRIANGLES) {
        int ti;
        if (e.geom_type == ATRC_GEOM_QUAD) {
            ti = e.tri_first + (w < e.quad_abc_prob ? 0 : 1);
            // pool order of the two quad halves may differ from ABC/ACD
            if (S.tri_orig[e.tri_first] != 0) ti = e.tri_first + (w < e.quad_abc_prob ? 1 : 0);
        } else if (e.geom_type == ATRC_GEOM_TRIANGLE) {
            ti = e.tri_first;
        } else {
            ti = e.tri_first + alias_sample(S.alias_prob + e.alias_first, S.alias_idx + e.alias_first, e.tri_count, u);
        }
        float b0, b1;
        if (e.geom_type == ATRC_GEOM_TRIANGLE_BVH) uniform_on_triangle(v, w, &b0, &b1);
        else uniform_on_triangle(u, v, &b0, &b1);
        const float4* tp = reinterpret_cast<const float4*>(S.tris) + size_t(ti) * 3;
        const float4 p0 = tp[0], p1 = tp[1], p2 = tp[2];
        p = Vec3(p0.x, p0.y, p0.z) + b0 * Vec3(p1.x, p1.y, p1.z) + b1 * Vec3(p2.x, p2.y, p2.z);
        const TriShade& sh = S.tri_shade[ti];
        const Vec3 x(sh.x[0], sh.x[1], sh.x[2]), z(sh.z[0], sh.z[1], sh.z[2]);
        c = Coord{x, cross(z, x), z};
        pd = 1 / e.leaf_area;
        if (e.flags & ENT_LOCAL) {
            p = apply_point_rn(e.local_m, p);
            c = xform_coord(e.local_m, c);
        }
    } else if (e.kind == LEAF_SPHERE) {
        const Vec3 lref = apply_point_rn(e.local_inv, ref);
        const float d = length(lref);
        const float wr2 = e.world_radius * e.world_radius;
        Vec3 lp;
        if (d <= e.radius) {
            float up;
            const Vec3 unit = uniform_on_sphere(u, v, &up);
            pd = up / wr2;
            lp = e.radius * unit;
        } else {
            const float ct = fminf(e.radius / d, 1.0f);
            float lpdf;
            const Vec3 dir = uniform_on_cone(ct, u, v, &lpdf);
            lp = e.radius * normalize(coord_from_z(lref).local_to_global(dir));
            pd = lpdf / wr2;
        }
        float tu, tv;
        sphere_uv_coord(lp, e.radius, S.eps, &tu, &tv, &c);
        p = apply_point_rn(e.local_m, lp);
        c = xform_coord(e.local_m, c);
    } else {
        float dx, dy;
        concentric_disk(u, v, &dx, &dy);
        const Vec3 lp(e.radius * dx, e.radius * dy, 0);
        float tu, tv;
        disk_point(lp, sqrtf(lp.x * lp.x + lp.y * lp.y), e.radius, &tu, &tv, &c);
        pd = 1 / e.leaf_area;
        p = apply_point_rn(e.local_m, lp);
        c = xform_coord(e.local_m, c);
    }
    if (e.flags & ENT_WRAP) {
        p = apply_point_rn(e.wrap_m, p);
        c = xform_coord(e.wrap_m, c);
        pd /= e.wrap_scale * e.wrap_scale;
    }
    if (e.flags & ENT_DOUBLE_SIDED) {
        pd *= 0.5f;
        if (back) c = c.neg();
    }
    *pos = p;
    *geo = c;
    *pdf = pd;
    return true;
}

// GeometryToDiffuseLight::sample (geometry_to_diffuse_light.cpp:16-31)
__device__ bool area_light_sample(const Scene& S, const Entity& e, Vec3 ref, float u, float v, float w,
                                  LightSample* ls) {
    Vec3 p;
    Coord c;
    float pdf_area;
    entity_sample(S, e, ref, u, v, w, &p, &c, &pdf_area);
    const Vec3 to_ref = ref - p;
    if (dot(c.z, to_ref) <= 0) return false;
    ls->pdf = pdf_area * dot(to_ref, to_ref) / fabsf(cosv(c.z, to_ref));
    ls->pos = p;
    ls->nor = c.z;
    ls->rad = Vec3(e.emit[0], e.emit[1], e.emit[2]);
    return true;
}

// GeometryToDiffuseLight::pdf (geometry_to_diffuse_light.cpp:79-90)
__device__ float area_light_pdf(const Scene& S, const Entity& e, Vec3 ref, Vec3 pos, Vec3 nor) {
    const Vec3 to_ref = ref - pos;
    if (dot(nor, to_ref) <= 0) return 0;
    float area_pdf = 1 / e.area;
    if (e.kind == LEAF_SPHERE) {  // sphere.cpp:135-147
        Vec3 lref = ref;
        if (e.flags & ENT_WRAP) lref = apply_point_rn(e.wrap_inv, lref);
        lref = apply_point_rn(e.local_inv, lref);
        const float d = length(lref);
        if (d > e.radius) {
            const float ct = fminf(e.radius / d, 1.0f);
            area_pdf = uniform_on_cone_pdf(ct) / (e.world_radius * e.world_radius);
            if (e.flags & ENT_WRAP) area_pdf /= e.wrap_scale * e.wrap_scale;
            if (e.flags & ENT_DOUBLE_SIDED) area_pdf *= 0.5f;
        }
    }
    return area_pdf * (dot(to_ref, to_ref) / fabsf(cosv(nor, to_ref)));
}

__device__ __forceinline__ Vec3 area_light_radiance(const Entity& e, Vec3 nor, Vec3 light_to_out) {
    return dot(nor, light_to_out) > 0 ? Vec3(e.emit[0], e.emit[1], e.emit[2]) : Vec3();
}

// ---- environment
__device__ Vec3 env_radiance(const Scene& S, Vec3 d) {
    const Env& env = S.env;
    const Vec3 dir = normalize(d);
    if (env.type == ATRC_ENV_NATIVE_SKY) {
        const float s = (clampf(dir.z, -1, 1) + 1) / 2;
        return s * Vec3(env.top[0], env.top[1], env.top[2]) + (1 - s) * Vec3(env.bottom[0], env.bottom[1], env.bottom[2]);
    }
    const float u = clampf(phi_of(dir) / (2 * kPi), 0, 1);
    const float v = clampf(acosf(clampf(dir.z, -1, 1)) / kPi, 0, 1);
    return tex2d_lookup<false>(S, env.tex, u, v, Vec3(), false);
}

__device__ float env_pdf(const Scene& S, Vec3 d) {
    const Env& env = S.env;
    if (env.type == ATRC_ENV_NATIVE_SKY) return 1 / (4 * kPi);
    const Vec3 dir = normalize(d);
    const float u = phi_of(dir) / (2 * kPi), v = acosf(clampf(dir.z, -1, 1)) / kPi;
    const int px = min(max(int(floorf(u * env.pw)), 0), env.pw - 1);
    const int py = min(max(int(floorf(v * env.ph)), 0), env.ph - 1);
    const float pp = env.probs[py * env.pw + px];
    const float u0 = float(px) / env.pw, u1 = float(px + 1) / env.pw;
    const float a = cosf(kPi * float(py + 1) / env.ph), b = cosf(kPi * float(py) / env.ph);
    return pp / (2 * kPi * ((u1 - u0) * (fmaxf(a, b) - fminf(a, b))));
}

__device__ Vec3 env_sample(const Scene& S, float u, float v, float w, float* pdf) {
    const Env& env = S.env;
    if (env.type == ATRC_ENV_NATIVE_SKY) return uniform_on_sphere(u, v, pdf);
    const int n = env.pw * env.ph;
    const int idx = alias_sample(env.alias_prob, env.alias_idx, n, u);
    const int py = idx / env.pw, px = idx % env.pw;
    const float pp = env.probs[idx];
    const float u0 = float(px) / env.pw, u1 = float(px + 1) / env.pw;
    const float a = cosf(kPi * float(py + 1) / env.ph), b = cosf(kPi * float(py) / env.ph);
    const float cmin = fminf(a, b), cmax = fmaxf(a, b);
    const float ct = cmin + w * (cmax - cmin);
    const float st = cos_2_sin(ct);
    float s, c;
    sincosf(2 * kPi * (u0 * (1 - v) + u1 * v), &s, &c);
    *pdf = pp / (2 * kPi * ((u1 - u0) * (cmax - cmin)));
    return Vec3(st * c, st * s, ct);
}

// IBL::emit_pos (ibl.cpp:103-131)
__device__ Vec3 env_emit_pos(const Scene& S, Vec3 ref, Vec3 to_light) {
    const Coord c = coord_from_z(to_light);
    const float R = S.env.radius;
    const Vec3 a = R * c.x, b = R * c.y, cc = -c.z;
    const Vec3 m = ref - Vec3(S.env.centre[0], S.env.centre[1], S.env.centre[2]) - R * c.z;
    const float D0 = a.y * b.z - a.z * b.y, D1 = a.x * b.z - a.z * b.x, D2 = a.x * b.y - a.y * b.x;
    const float det = cc.x * D0 - cc.y * D1 + cc.z * D2;
    const float tdet = m.x * D0 - m.y * D1 + m.z * D2;
    return ref + (tdet / det) * c.z;
}

// =================================================================== media
struct Phase {
    float g;
    Vec3 albedo;
};

__device__ __forceinline__ float hg_value(float g, float u) {
    const float g2 = g * g;
    const float dem = 1 + g2 - 2 * g * u;
    return (1 - g2) / (4 * kPi * dem * sqrtf(dem));
}
__device__ __forceinline__ float hg_pdf(const Phase& ph, Vec3 wi, Vec3 wo) { return hg_value(ph.g, -cosv(wi, wo)); }
__device__ BSDFSample hg_sample(const Phase& ph, Vec3 wo, float u0, float u1) {
    const float s = 2 * u0 - 1;
    float u;
    if (fabsf(ph.g) < 0.001f) {
        u = s;
    } else {
        const float g2 = ph.g * ph.g;
        u = (1 + g2 - sqrf((1 - g2) / (1 + ph.g * s))) / (2 * ph.g);
    }
    const float ct = -u, st = cos_2_sin(ct);
    float sp, cp;
    sincosf(2 * kPi * u1, &sp, &cp);
    const Vec3 lwi(st * sp, st * cp, ct);
    const float pv = hg_value(ph.g, u);
    BSDFSample r;
    r.dir = coord_from_z(wo).local_to_global(lwi);
    r.f = Vec3(pv);
    r.pdf = pv;
    r.delta = false;
    return r;
}

// Transmittance (ratio tracking for grids); `cap` bounds the loop.
__device__ Vec3 medium_tr(const Scene& S, int mi, Vec3 a, Vec3 b, Rng& rng, int* watchdog) {
    const Medium& m = S.media[mi];
    if (m.type == ATRC_MED_HOMOGENEOUS) {
        const float d = length(a - b);
        return Vec3(__expf(-m.sigma_t[0] * d), __expf(-m.sigma_t[1] * d), __expf(-m.sigma_t[2] * d));
    }
    if (m.type == ATRC_MED_HETEROGENEOUS) {
        float result = 1, t = 0;
        const float t_max = length(a - b);
        for (int it = 0;; ++it) {
            if (it >= (1 << 16)) { *watchdog = 3; break; }
            t += -logf(1 - rng.u()) * m.inv_max_density;
            if (t >= t_max) break;
            const Vec3 p = a + (b - a) * (t / t_max);
            const float dens = tex3d_sample<true>(S, m.density, apply_point_rn(m.inv, p)).x;
            result *= 1 - dens / m.max_density;
        }
        return Vec3(result);
    }
    return Vec3(1.0f);
}

__device__ Vec3 medium_ab(const Scene& S, int mi, Vec3 a, Vec3 b, Rng& rng, int* watchdog) {
    const Medium& m = S.media[mi];
    if (m.type == ATRC_MED_HOMOGENEOUS) {
        const float d = length(a - b);
        return Vec3(__expf(-m.sigma_a[0] * d), __expf(-m.sigma_a[1] * d), __expf(-m.sigma_a[2] * d));
    }
    return medium_tr(S, mi, a, b, rng, watchdog);
}

// sample_scattering on the segment a -> b; true if scattered.
__device__ bool medium_sample(const Scene& S, int mi, Vec3 a, Vec3 b, bool indirect, Rng& rng, Vec3* tp,
                              Vec3* pos, Vec3* wr, Phase* ph, int* watchdog) {
    const Medium& m = S.media[mi];
    if (m.type == ATRC_MED_HOMOGENEOUS) {  // homogeneous.cpp:66-109
        const float u = rng.u();
        const Vec3 ss(m.sigma_s[0], m.sigma_s[1], m.sigma_s[2]), st(m.sigma_t[0], m.sigma_t[1], m.sigma_t[2]);
        if (black(ss)) { *tp = medium_tr(S, mi, a, b, rng, watchdog); return false; }
        const float t_max = length(b - a);
        const int ch = min(int(u * 3), 2);
        const float nu = u * 3 - ch;
        const float sampled = -logf(nu) / st[ch];
        const bool in_medium = sampled < t_max;
        const float dd = fminf(sampled, t_max);
        const Vec3 tr(__expf(-st.x * dd), __expf(-st.y * dd), __expf(-st.z * dd));
        const Vec3 dens = in_medium ? st * tr : tr;
        const float pdf = fmaxf((dens.x + dens.y + dens.z) / 3, S.eps);
        Vec3 t = tr / pdf;
        if (in_medium) t = t * ss;
        *tp = t;
        if (in_medium) {
            *pos = a + (b - a) * (sampled / t_max);
            *wr = (a - b) / t_max;
            ph->g = m.g;
            ph->albedo = ss / st;
            return true;
        }
        return false;
    }
    if (m.type == ATRC_MED_HETEROGENEOUS) {  // heterogeneous.cpp:83-123
        const float t_max = length(b - a);
        float t = 0;
        for (int it = 0;; ++it) {
            if (it >= (1 << 16)) { *watchdog = 3; break; }
            t += -logf(1 - rng.u()) * m.inv_max_density;
            if (t >= t_max) break;
            const Vec3 p = a + (b - a) * (t / t_max);
            const Vec3 unit = apply_point_rn(m.inv, p);
            const float dens = tex3d_sample<true>(S, m.density, unit).x;
            if (rng.u() < dens / m.max_density) {
                const Vec3 alb = m.white_for_indirect && indirect ? Vec3(1.0f) : tex3d_sample<false>(S, m.albedo, unit);
                ph->g = tex3d_sample<true>(S, m.g_tex, unit).x;
                ph->albedo = alb;
                *pos = p;
                *wr = (a - b) / t_max;
                *tp = alb;
                return true;
            }
        }
        *tp = Vec3(1.0f);
        return false;
    }
    *tp = Vec3(1.0f);
    return false;
}

}  // namespace dev
}  // namespace atrc
