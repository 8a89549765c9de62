// Binned-SAH BVH builder for the device acceleration structure.
//
// The reference builds a binary midpoint/median BVH per mesh
// (src/tracer/src/core/geometry/triangle_bvh.cpp:122-304) and a median-split
// BVH over entities (src/tracer/src/core/aggregate/entity_bvh.cpp:46-116).
// The device uses its own layout instead: a binary SAH tree (nodes hold both
// children's boxes) collapsed into a 4-wide tree whose 128-byte nodes hold
// the four children's boxes as structure of arrays, so one traversal step
// tests four boxes with seven 128-bit loads.  Hit results do not depend on
// the tree shape.
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

// 4-wide device node: child boxes (x, y, z bounds of the four children) and
// child links in the encoding of BvhNode; unused slots hold kEmptyLink.
struct alignas(16) Bvh4Node {
    float lo_x[4], hi_x[4], lo_y[4], hi_y[4], lo_z[4], hi_z[4];
    int32_t link[4];
    int32_t pad[4];
};
static_assert(sizeof(Bvh4Node) == 128, "node must be 128 bytes");
constexpr int32_t kEmptyLink = int32_t(0x80000002u);  // INT_MIN + 2: no child

// Collapse a binary tree into 4-wide nodes appended to `out` (depth-first,
// interior links are indices into `out`, leaf links keep the binary tree's
// encoding): each wide node opens the widest (largest surface area)
// interior child until it has four children.  Returns the root link.
int32_t collapse_bvh4(const BvhResult& b, std::vector<Bvh4Node>* out);

// Structural check of a 4-wide tree below `root`: links in range, every
// node reached once (no cycle or sharing), leaves covering primitive slots
// [0, prim_count) exactly once (leaf firsts relative to prim_first).
// Throws std::runtime_error.
void validate_bvh4(const std::vector<Bvh4Node>& nodes, int32_t root, uint32_t prim_first, uint32_t prim_count);

// max_leaf: largest primitive count per leaf (<= 16).
BvhResult build_bvh(const std::vector<BuildPrim>& prims, int max_leaf, float traversal_cost = 1.0f,
                    float intersect_cost = 1.0f);

inline int32_t leaf_link(uint32_t first, uint32_t count) { return ~int32_t((first << 4) | (count - 1)); }

}  // namespace atrc
