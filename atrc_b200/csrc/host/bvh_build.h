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

// ------------------------------------------------------------- PLOC
// Parallel locally-ordered clustering (Meister and Bittner 2018, "Parallel
// Locally-Ordered Clustering for Bounding Volume Hierarchy Construction"):
// primitives sorted by the 63-bit Morton code of their box centres start as
// clusters; every round, each cluster finds the cluster within `radius`
// positions whose union box has the smallest surface area, mutual nearest
// neighbours merge (the new cluster keeps the lower position) and the list
// is compacted, until one cluster is left.  Ties are broken by the pair of
// positions, so the nearest-neighbour relation has a strict order, every
// round merges at least one pair, and the tree does not depend on thread
// timing: the device build (bvh_gpu.cu) and the serial build below give the
// same tree bit for bit.
//
// The binary cluster tree: node i < n is the leaf of sorted primitive i,
// node n + k is the k-th merge (children created before their parent).
struct ClusterTree {
    uint32_t n = 0;
    int32_t root = -1;
    std::vector<uint32_t> order;       // sorted position -> primitive index
    std::vector<int32_t> left, right;  // children of internal node n + k
    std::vector<BuildPrim> box;        // box of internal node n + k
    int rounds = 0;
};

constexpr int kPlocRadius = 16;

// Box centre quantised to 21 bits per axis, bits interleaved x-y-z (x in
// the lowest position); lo / inv_ext map the centre bound to [0, 1].
uint64_t morton63(const BuildPrim& p, const float lo[3], const float inv_ext[3]);

// Surface-area measure of the union of two boxes, as the cluster distance.
float union_area(const BuildPrim& a, const BuildPrim& b);

// Serial PLOC (the specification of the device build; O(n radius) per round).
ClusterTree ploc_build_host(const std::vector<BuildPrim>& prims, int radius = kPlocRadius);

// Device PLOC on `device` (bvh_gpu.cu); throws std::runtime_error.
ClusterTree ploc_build_device(const std::vector<BuildPrim>& prims, int device, int radius = kPlocRadius);

// A finished 4-wide tree: interior links index `nodes`, leaf links encode
// (first, count) into `order` (leaf position -> primitive index).
struct WideBvh {
    std::vector<Bvh4Node> nodes;
    std::vector<uint32_t> order;
    int32_t root = 0;
    float bound_lo[3] = {0, 0, 0}, bound_hi[3] = {0, 0, 0};
    int rounds = 0;
};

// The whole mesh-tree build on `device`: PLOC, the surface-area leaves of
// bvh_from_clusters (decided as the clusters merge) and the 4-wide collapse
// of collapse_bvh4 (walked from the root round by round), so only the result
// comes back.  The same tree as collapse_bvh4(bvh_from_clusters(
// ploc_build_host(prims))) up to the numbering of its nodes.
WideBvh ploc_wide_device(const std::vector<BuildPrim>& prims, int device, int max_leaf = 4,
                         float traversal_cost = 1.0f, float intersect_cost = 1.0f);

// A cluster tree as a binary BVH with leaves of up to max_leaf primitives:
// a subtree becomes a leaf where that is cheaper under the surface-area
// heuristic (leaf: count * intersect_cost; split: traversal_cost + the
// children's costs weighted by their area over the parent's).
BvhResult bvh_from_clusters(const ClusterTree& t, const std::vector<BuildPrim>& prims, int max_leaf,
                            float traversal_cost = 1.0f, float intersect_cost = 1.0f);

// Surface-area cost of a 4-wide tree (interior visits weighted by area over
// the root's area, plus leaf primitives likewise), for comparing builders.
double bvh4_sah_cost(const std::vector<Bvh4Node>& nodes, int32_t root, float traversal_cost = 1.0f,
                     float intersect_cost = 1.0f);

// Depth of a 4-wide tree (a leaf root has depth 0).
int bvh4_depth(const std::vector<Bvh4Node>& nodes, int32_t root);

}  // namespace atrc
