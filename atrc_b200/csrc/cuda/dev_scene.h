// Device scene layout (structure of arrays in HBM).
//
// One flat triangle pool holds every triangle of every leaf geometry; each
// leaf geometry owns a bottom-level BVH over its slice of the pool, and a
// top-level BVH spans the entities.  Triangles are split into a hot part
// (three float4: A, B-A, C-A, 48 bytes, read by traversal) and a cold part
// (shading data, read once per hit).
#pragma once

#include <cstdint>

#include "../host/bvh_build.h"
#include "../host/vecmath.h"

namespace atrc {
namespace dev {

constexpr int kMaxLights = 256;

enum EntityFlags : uint32_t {
    ENT_WRAP = 1u,          // transform_wrapper present
    ENT_LOCAL = 2u,         // geometry's own transform moves rays to local space
    ENT_DOUBLE_SIDED = 4u,
    ENT_LIGHT = 8u,
    ENT_NO_DENOISE = 16u,
};

enum LeafKind : int32_t { LEAF_TRIANGLES = 0, LEAF_SPHERE = 1, LEAF_DISK = 2 };

struct Entity {
    int32_t kind;          // LeafKind
    int32_t blas_root;     // root link of the leaf geometry's BVH
    uint32_t flags;        // EntityFlags
    int32_t material;
    int32_t med_in, med_out;
    int32_t tri_first;     // first triangle of the leaf in the pool
    int32_t tri_count;
    float wrap_m[12], wrap_inv[12];
    float local_m[12], local_inv[12];
    float emit[3];
    float radius;          // sphere / disk radius (local)
    float area;            // world surface area (for light pdfs)
    float world_radius;    // sphere
    float wrap_scale;      // |wrap * (0,0,1)| (transform_wrapper.cpp:13)
    int32_t alias_first;   // triangle-area alias table of the leaf
    int32_t geom_type;     // AtrcGeometryType of the leaf
    float quad_abc_prob;   // quad: probability of sampling ABC
    float leaf_area;       // leaf surface area before wrapper scaling
};

// Cold per-triangle data (96 bytes).
struct TriShade {
    float x[3], z[3];        // geometric frame (x = dpdu, z = face normal)
    float n_a[3], n_ba[3], n_ca[3];
    float t_a[2], t_ba[2], t_ca[2];
    float pad[3];
};

struct Texture2D {
    int32_t type, width, height, nearest;
    float texel[3];
    float inv_gamma;
    float texel2[3];         // checker board: second colour
    float grid_size;         // checker board: 1 / grid_count
    float uv[6];
    int32_t wrap_u, wrap_v;
    int64_t data_offset;     // float offset into the texel pool
    int32_t tex3d;           // solid image: the 3D texture behind it
    int32_t pad_;
};

struct Texture3D {
    int32_t type, width, height, depth;
    int32_t channels, nearest;
    int32_t wrap[3];
    float texel[3];
    float inv_gamma;
    float max_real;
    float uvw[12];
    int64_t data_offset;
};

// Material with every constant texture folded into `c`.
struct Material {
    int32_t type;
    int32_t all_constant;    // 1 if every texture slot is constant
    int32_t tex[13];
    int32_t normal_map;
    float c[16];             // constant values: base_color rgb, metallic, roughness,
                             // transmission, trans_rough, ior, spec_scale rgb,
                             // spec_tint, aniso, sheen, sheen_tint, clearcoat
    float cc_gloss;
    int32_t bssrdf[3];       // subsurface A, dmfp, eta textures (-1: none)
};

struct Medium {
    int32_t type;
    int32_t max_scattering_count;
    float sigma_a[3], sigma_s[3], sigma_t[3];
    float g;
    float inv[12];
    int32_t density, albedo, g_tex;
    int32_t white_for_indirect;
    float max_density, inv_max_density;
};

struct Env {
    int32_t type;
    int32_t tex;
    int32_t pw, ph;          // patch grid of the importance sampler
    float top[3], bottom[3];
    float centre[3];
    float radius;
    const float* probs;      // pw * ph normalised patch probabilities
    const float* alias_prob; // alias table
    const int32_t* alias_idx;
};

struct Scene {
    const Bvh4Node* nodes;          // all 4-wide BVH nodes (every BLAS + the TLAS)
    const float* tris;              // 12 floats per triangle: A,_, B-A,_, C-A,_
    const float* tri_bc;            // 8 floats per triangle: the exact vertices B,_, C,_ (watertight test)
    const TriShade* tri_shade;
    const uint32_t* tri_orig;       // original index per pool triangle
    const Entity* entities;
    const uint32_t* tlas_order;     // TLAS leaf slot -> entity index
    int32_t tlas_root;
    int32_t entity_count;
    const Material* materials;
    int32_t material_count;
    const Texture2D* tex2d;
    const Texture3D* tex3d;
    const float* texels;
    const Medium* media;
    int32_t medium_count;
    int32_t has_media;              // any non-void medium referenced
    int32_t has_subsurface;         // any material with subsurface scattering
    const float* alias_prob;        // triangle-area alias tables (all leaves)
    const int32_t* alias_idx;
    int32_t light_count;            // lights: env first (if any), then areas
    int32_t light_entity[kMaxLights]; // -1 for the environment light
    Env env;
    float eps;
    int32_t disney_fixed;           // sample the Disney diffuse lobe (render option)
    float scene_lo[3], scene_hi[3];
};

}  // namespace dev
}  // namespace atrc
