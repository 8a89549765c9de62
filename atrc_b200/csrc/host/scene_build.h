// Host-side flattening of an AtrcSceneDesc into the device scene layout
// (dev_scene.h): triangle pool, per-leaf bottom-level BVHs, a top-level BVH
// over entities, folded material constants, texel pools and the sampling
// tables (triangle-area alias tables, environment patch alias table).
#pragma once

#include <string>
#include <vector>

#include "../../../include/atrc_cuda.h"
#include "../cuda/dev_scene.h"

namespace atrc {

struct HostScene {
    std::vector<Bvh4Node> nodes;  // every 4-wide node (each BLAS, then the TLAS)
    std::vector<float> tris;          // 12 per triangle
    std::vector<float> tri_bc;        // 8 per triangle: exact B and C
    std::vector<dev::TriShade> tri_shade;
    std::vector<uint32_t> tri_orig;
    std::vector<dev::Entity> entities;
    std::vector<uint32_t> tlas_order;
    std::vector<dev::Material> materials;
    std::vector<dev::Texture2D> tex2d;
    std::vector<dev::Texture3D> tex3d;
    std::vector<float> texels;
    std::vector<dev::Medium> media;
    std::vector<float> alias_prob;
    std::vector<int32_t> alias_idx;
    std::vector<float> env_probs, env_alias_prob;
    std::vector<int32_t> env_alias_idx;
    dev::Scene scene{};               // pointers left null; filled on upload
    int max_blas_depth = 0, tlas_depth = 0;
};

// Throws std::runtime_error with a message on unsupported or invalid input.
// `device` runs the PLOC builder where the description asks for it (-1:
// build every tree on the host with the SAH builder).
void build_host_scene(const AtrcSceneDesc& desc, HostScene* out, int device = -1);

}  // namespace atrc
