// Learned directional guiding: encodings and the von Mises-Fisher mixture.
//
// The guide maps a surface vertex (position, normal, outgoing direction,
// roughness) to a mixture of kGuideLobes vMF lobes over world directions plus
// a probability c of sampling the mixture instead of the BSDF.  It has no
// counterpart in the reference: `pt` samples the BSDF only
// (path_tracing.cpp:150-169).  Sampling is one-sample MIS between the
// mixture and the BSDF, so the pdf of a direction is c q(w) + (1 - c) p(w)
// and the estimator stays unbiased wherever the BSDF sampler has support
// (c <= kGuideMaxSelect keeps that support).
//
// Network input (kGuideIn = 112 features, padded with zeros):
//   [0, 32)    multiresolution hash grid: 16 levels x 2 features, trilinear
//              (Mueller et al. 2022, "Instant neural graphics primitives"),
//              position normalised to the scene bound;
//   [32, 64)   one-blob of the shading normal: 16 bins of (cos theta + 1) / 2
//              and 16 bins of (phi + pi) / 2 pi, tent kernel of one bin;
//   [64, 96)   the same for the outgoing direction;
//   [96]       roughness (0 for non-Disney materials).
// Output (kGuideOut = 48 raw values, 41 used): per lobe k the unnormalised
// mean direction o[5k..5k+2], log kappa o[5k+3] and mixture logit o[5k+4];
// o[40] is the selection logit (c = max_select sigmoid(o[40] - 2)).
#pragma once

#include <cstdint>

#include "dev_math.cuh"

namespace atrc {
namespace dev {

constexpr int kGuideLobes = 8;
constexpr int kGuideIn = 112;
constexpr int kGuideHidden = 64;
constexpr int kGuideOut = 48;
constexpr int kGuideUsed = 5 * kGuideLobes + 1;
constexpr int kHashLevels = 16;
constexpr int kHashFeatures = 2;
// Default cap: c = max_select * sigmoid(o[40] + kSelectOffset).  The weight
// of a vertex is at most 1 / (1 - c) times the BSDF sampler's, so the cap
// bounds the variance a guide that is still learning can add: on the indoor
// room's equal-time protocol (5 seeds) caps of 0.9 / 0.5 / 0.3 / 0.25 / 0.15
// gave time ratios of 1.13 / 0.74 / 0.63-0.73 / 0.56 / 0.61 with guided
// depth 3; with depth 5, caps of 0.2 / 0.15 / 0.125 / 0.1 averaged 0.50 /
// 0.48 / 0.47 / 0.49 over runs on two seed sets (run-to-run spread about
// +-0.05).
constexpr float kGuideMaxSelect = 0.15f;
constexpr float kSelectOffset = -2.0f;    // an untrained guide (o ~ 0) is picked with c ~ 0.12 max_select
constexpr float kLogKappaMin = -6.9f;     // kappa in [1e-3, 1e4]
constexpr float kLogKappaMax = 9.2f;

// One query of the guide (48 bytes).
struct GuideQuery {
    float pos[3], nrm[3], wo[3], rough;
    int32_t slot;   // path slot the result belongs to (-1: no query)
    int32_t pad;
};

// Decoded mixture of one vertex.
struct GuideMix {
    float mu[kGuideLobes][3];
    float kappa[kGuideLobes];
    float w[kGuideLobes];
    float c;
};

// Hash-grid geometry shared by every kernel that encodes positions.
struct HashGrid {
    int32_t log2_table;          // entries per level = 1 << log2_table
    int32_t res[kHashLevels];    // cells per axis of level l: floor(base * growth^l), computed on the host
    float lo[3], inv_ext[3];     // position normalisation to [0, 1]^3
};

__device__ __forceinline__ int hash_res(const HashGrid& g, int level) { return g.res[level]; }

// Table slot of a grid vertex: dense while the level fits the table, else
// the spatial hash of Teschner et al. as used by instant-ngp.
__device__ __forceinline__ uint32_t hash_slot(const HashGrid& g, int res, uint32_t x, uint32_t y, uint32_t z) {
    const uint32_t n = uint32_t(res) + 1;
    const uint32_t mask = (1u << g.log2_table) - 1u;
    if (uint64_t(n) * n * n <= (uint64_t(1) << g.log2_table)) return x + n * (y + n * z);
    return (x * 1u ^ y * 2654435761u ^ z * 805459861u) & mask;
}

// Corners and trilinear weights of one level.
struct HashCell {
    uint32_t slot[8];
    float w[8];
};

__device__ __forceinline__ void hash_cell(const HashGrid& g, int level, const float p01[3], HashCell* c) {
    const int res = hash_res(g, level);
    float f[3];
    uint32_t i0[3];
    for (int a = 0; a < 3; ++a) {
        const float x = fminf(fmaxf(p01[a], 0.0f), 1.0f) * float(res);
        const float fl = fminf(floorf(x), float(res - 1));
        i0[a] = uint32_t(fl);
        f[a] = x - fl;
    }
    for (int k = 0; k < 8; ++k) {
        const uint32_t dx = k & 1, dy = (k >> 1) & 1, dz = k >> 2;
        c->slot[k] = hash_slot(g, res, i0[0] + dx, i0[1] + dy, i0[2] + dz);
        c->w[k] = (dx ? f[0] : 1 - f[0]) * (dy ? f[1] : 1 - f[1]) * (dz ? f[2] : 1 - f[2]);
    }
}

__device__ __forceinline__ void normalise_pos(const HashGrid& g, const float pos[3], float p01[3]) {
    for (int a = 0; a < 3; ++a) p01[a] = (pos[a] - g.lo[a]) * g.inv_ext[a];
}

// Tent one-blob of s in [0, 1] into 16 bins.
__device__ __forceinline__ void one_blob16(float s, float* out) {
    const float x = fminf(fmaxf(s, 0.0f), 1.0f) * 16.0f;
    for (int i = 0; i < 16; ++i) out[i] = fmaxf(0.0f, 1.0f - fabsf(x - (float(i) + 0.5f)));
}

__device__ __forceinline__ void dir_blob(const float d[3], float* out) {
    one_blob16(0.5f * (fminf(fmaxf(d[2], -1.0f), 1.0f) + 1.0f), out);
    one_blob16((atan2f(d[1], d[0]) + kPi) * (0.5f / kPi), out + 16);
}

// The non-hash part of the input: features [32, 112).
__device__ __forceinline__ void guide_dense_features(const GuideQuery& q, float* out80) {
    dir_blob(q.nrm, out80);
    dir_blob(q.wo, out80 + 32);
    out80[64] = q.rough;
    for (int i = 65; i < 80; ++i) out80[i] = 0.0f;
}

__device__ __forceinline__ float sigmoidf_(float x) { return 1.0f / (1.0f + __expf(-x)); }

// vMF lobe density: kappa / (2 pi (1 - e^{-2 kappa})) exp(kappa (cos - 1)).
__device__ __forceinline__ float vmf_norm(float kappa) { return kappa / (2.0f * kPi * -expm1f(-2.0f * kappa)); }

// max_select: the cap on the selection probability (AtrcGuideDesc.max_select).
__device__ __forceinline__ void guide_decode(const float* o, GuideMix* m, float max_select = kGuideMaxSelect) {
    float mx = -1e30f;
    for (int k = 0; k < kGuideLobes; ++k) mx = fmaxf(mx, o[5 * k + 4]);
    float sum = 0;
    for (int k = 0; k < kGuideLobes; ++k) {
        const float x = o[5 * k], y = o[5 * k + 1], z = o[5 * k + 2];
        const float n2 = x * x + y * y + z * z;
        const float inv = n2 > 1e-20f ? rsqrtf(n2) : 0.0f;
        m->mu[k][0] = n2 > 1e-20f ? x * inv : 0.0f;
        m->mu[k][1] = n2 > 1e-20f ? y * inv : 0.0f;
        m->mu[k][2] = n2 > 1e-20f ? z * inv : 1.0f;
        m->kappa[k] = __expf(fminf(fmaxf(o[5 * k + 3], kLogKappaMin), kLogKappaMax));
        m->w[k] = __expf(o[5 * k + 4] - mx);
        sum += m->w[k];
    }
    for (int k = 0; k < kGuideLobes; ++k) m->w[k] /= sum;
    m->c = max_select * sigmoidf_(o[5 * kGuideLobes] + kSelectOffset);
}

__device__ __forceinline__ float guide_pdf(const GuideMix& m, Vec3 d) {
    float p = 0;
    for (int k = 0; k < kGuideLobes; ++k) {
        const float cs = m.mu[k][0] * d.x + m.mu[k][1] * d.y + m.mu[k][2] * d.z;
        p += m.w[k] * vmf_norm(m.kappa[k]) * __expf(m.kappa[k] * (cs - 1.0f));
    }
    return p;
}

// Sample the mixture: u0 picks the lobe, (u1, u2) the direction in it
// (inversion of the vMF cosine distribution, Jakob 2012).
__device__ __forceinline__ Vec3 guide_sample(const GuideMix& m, float u0, float u1, float u2) {
    int k = 0;
    float acc = m.w[0];
    while (k + 1 < kGuideLobes && u0 >= acc) acc += m.w[++k];
    const float kap = m.kappa[k];
    const float w = 1.0f + logf(u1 + (1.0f - u1) * __expf(-2.0f * kap)) / kap;
    const float wc = fminf(fmaxf(w, -1.0f), 1.0f);
    const float v = sqrtf(fmaxf(0.0f, 1.0f - wc * wc));
    float sp, cp;
    __sincosf(2.0f * kPi * u2, &sp, &cp);
    const Vec3 mu(m.mu[k][0], m.mu[k][1], m.mu[k][2]);
    const Coord c = coord_from_z(mu);
    return normalize(c.x * (v * cp) + c.y * (v * sp) + mu * wc);
}

}  // namespace dev
}  // namespace atrc
