// Binned-SAH BVH builder for the device acceleration structure.
//
// The reference builds a binary midpoint/median BVH per mesh
// (src/tracer/src/core/geometry/triangle_bvh.cpp:122-304) and a median-split
// BVH over entities (src/tracer/src/core/aggregate/entity_bvh.cpp:46-116).
// The device uses its own layout instead: a binary SAH tree whose nodes hold
// both children's boxes (64 bytes, four 128-bit loads), so a traversal step
// tests two boxes per node fetch.  Hit results do not depend on the tree shape.
#pragma once

#include <cstdint>
#include <vector>

namespace atrc {

struct BuildPrim {
    float lo[3], hi[3];
};

// Device node: child boxes + child links.  A link >= 0 is an interior node
// index; a negative link encodes a leaf: ~((first << 4) | (count - 1)).
struct alignas(16) BvhNode {
    float c0lo_x, c0hi_x, c0lo_y, c0hi_y;
    float c1lo_x, c1hi_x, c1lo_y, c1hi_y;
    float c0lo_z, c0hi_z, c1lo_z, c1hi_z;
    int32_t link0, link1, pad0, pad1;
};
static_assert(sizeof(BvhNode) == 64, "node must be 64 bytes");

struct BvhResult {
    std::vector<BvhNode> nodes;   // node 0 is the root (if any interior node)
    std::vector<uint32_t> order;  // leaf order -> primitive index
    int32_t root_link = 0;        // link of the root (leaf if the tree is one leaf)
    float bound_lo[3], bound_hi[3];
    int max_depth = 0;
};

// max_leaf: largest primitive count per leaf (<= 16).
BvhResult build_bvh(const std::vector<BuildPrim>& prims, int max_leaf, float traversal_cost = 1.0f,
                    float intersect_cost = 1.0f);

inline int32_t leaf_link(uint32_t first, uint32_t count) { return ~int32_t((first << 4) | (count - 1)); }

}  // namespace atrc
