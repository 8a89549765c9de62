// Binned SAH build (32 bins per axis, centroid bounds), iterative with an
// explicit task stack; large ranges are split across threads.
#include "bvh_build.h"

#include <algorithm>
#include <atomic>
#include <cstdint>
#include <cmath>
#include <cstring>
#include <future>
#include <limits>
#include <mutex>
#include <stdexcept>
#include <thread>

namespace atrc {

namespace {

struct Box {
    float lo[3] = {std::numeric_limits<float>::max(), std::numeric_limits<float>::max(),
                   std::numeric_limits<float>::max()};
    float hi[3] = {-std::numeric_limits<float>::max(), -std::numeric_limits<float>::max(),
                   -std::numeric_limits<float>::max()};
    void grow(const float* l, const float* h) {
        for (int k = 0; k < 3; ++k) {
            lo[k] = std::min(lo[k], l[k]);
            hi[k] = std::max(hi[k], h[k]);
        }
    }
    void grow(const Box& b) { grow(b.lo, b.hi); }
    float area() const {
        float d[3];
        for (int k = 0; k < 3; ++k) d[k] = std::max(0.0f, hi[k] - lo[k]);
        return 2.0f * (d[0] * d[1] + d[1] * d[2] + d[2] * d[0]);
    }
    bool valid() const { return lo[0] <= hi[0]; }
};

constexpr int kBins = 32;

struct Builder {
    const std::vector<BuildPrim>& prims;
    std::vector<uint32_t>& idx;
    std::vector<float> cen;  // 3 per prim
    int max_leaf;
    float ct, ci;
    std::mutex mtx;
    std::vector<BvhNode>& nodes;
    std::atomic<int> max_depth{0};

    Builder(const std::vector<BuildPrim>& p, std::vector<uint32_t>& i, std::vector<BvhNode>& n, int ml, float t,
            float c)
        : prims(p), idx(i), max_leaf(ml), ct(t), ci(c), nodes(n) {
        cen.resize(p.size() * 3);
        for (size_t k = 0; k < p.size(); ++k)
            for (int a = 0; a < 3; ++a) cen[k * 3 + a] = 0.5f * (p[k].lo[a] + p[k].hi[a]);
    }

    int alloc_node() {
        std::lock_guard<std::mutex> lk(mtx);
        nodes.push_back(BvhNode{});
        return int(nodes.size() - 1);
    }

    Box range_box(uint32_t b, uint32_t e) const {
        Box r;
        for (uint32_t i = b; i < e; ++i) r.grow(prims[idx[i]].lo, prims[idx[i]].hi);
        return r;
    }

    // Split [b, e) and return the split position, or e if a leaf is better.
    uint32_t split(uint32_t b, uint32_t e, const Box& box) {
        const uint32_t n = e - b;
        if (n <= 1) return e;
        Box cb;
        for (uint32_t i = b; i < e; ++i) {
            const float* c = &cen[size_t(idx[i]) * 3];
            cb.grow(c, c);
        }
        float best_cost = std::numeric_limits<float>::max();
        int best_axis = -1, best_bin = -1;
        for (int a = 0; a < 3; ++a) {
            const float ext = cb.hi[a] - cb.lo[a];
            if (!(ext > 0)) continue;
            Box bb[kBins];
            uint32_t cnt[kBins] = {0};
            const float scale = kBins / ext;
            for (uint32_t i = b; i < e; ++i) {
                const uint32_t p = idx[i];
                int k = int((cen[size_t(p) * 3 + a] - cb.lo[a]) * scale);
                k = std::min(std::max(k, 0), kBins - 1);
                cnt[k]++;
                bb[k].grow(prims[p].lo, prims[p].hi);
            }
            float right_area[kBins];
            uint32_t right_cnt[kBins];
            Box acc;
            uint32_t c = 0;
            for (int k = kBins - 1; k > 0; --k) {
                acc.grow(bb[k]);
                c += cnt[k];
                right_area[k] = acc.valid() ? acc.area() : 0;
                right_cnt[k] = c;
            }
            Box lacc;
            uint32_t lc = 0;
            for (int k = 0; k < kBins - 1; ++k) {
                lacc.grow(bb[k]);
                lc += cnt[k];
                if (lc == 0 || right_cnt[k + 1] == 0) continue;
                const float cost = (lacc.valid() ? lacc.area() : 0) * lc + right_area[k + 1] * right_cnt[k + 1];
                if (cost < best_cost) {
                    best_cost = cost;
                    best_axis = a;
                    best_bin = k;
                }
            }
        }
        const float parent_area = std::max(box.area(), 1e-30f);
        const float leaf_cost = ci * n;
        const float split_cost = ct + ci * best_cost / parent_area;
        if (best_axis < 0) {
            // all centroids coincide: median split if the range is too large
            if (n <= uint32_t(max_leaf)) return e;
            return b + n / 2;
        }
        if (n <= uint32_t(max_leaf) && leaf_cost <= split_cost) return e;
        const float ext = cb.hi[best_axis] - cb.lo[best_axis];
        const float scale = kBins / ext;
        auto mid_it = std::partition(idx.begin() + b, idx.begin() + e, [&](uint32_t p) {
            int k = int((cen[size_t(p) * 3 + best_axis] - cb.lo[best_axis]) * scale);
            k = std::min(std::max(k, 0), kBins - 1);
            return k <= best_bin;
        });
        uint32_t mid = uint32_t(mid_it - idx.begin());
        if (mid == b || mid == e) mid = b + n / 2;
        return mid;
    }

    // Builds the subtree of [b, e) and returns its link.
    int32_t build(uint32_t b, uint32_t e, const Box& box, int depth) {
        int md = max_depth.load();
        while (depth > md && !max_depth.compare_exchange_weak(md, depth)) {}
        const uint32_t mid = split(b, e, box);
        if (mid == e) return leaf_link(b, e - b);
        const int node = alloc_node();
        Box lb = range_box(b, mid), rb = range_box(mid, e);
        int32_t l, r;
        if (e - b > 200000 && depth < 6) {
            auto fut = std::async(std::launch::async, [&] { return build(b, mid, lb, depth + 1); });
            r = build(mid, e, rb, depth + 1);
            l = fut.get();
        } else {
            l = build(b, mid, lb, depth + 1);
            r = build(mid, e, rb, depth + 1);
        }
        std::lock_guard<std::mutex> lk(mtx);
        BvhNode& nd = nodes[node];
        nd.c0lo_x = lb.lo[0]; nd.c0hi_x = lb.hi[0]; nd.c0lo_y = lb.lo[1]; nd.c0hi_y = lb.hi[1];
        nd.c1lo_x = rb.lo[0]; nd.c1hi_x = rb.hi[0]; nd.c1lo_y = rb.lo[1]; nd.c1hi_y = rb.hi[1];
        nd.c0lo_z = lb.lo[2]; nd.c0hi_z = lb.hi[2]; nd.c1lo_z = rb.lo[2]; nd.c1hi_z = rb.hi[2];
        nd.link0 = l;
        nd.link1 = r;
        return node;
    }
};

}  // namespace

BvhResult build_bvh(const std::vector<BuildPrim>& prims, int max_leaf, float traversal_cost, float intersect_cost) {
    BvhResult res;
    if (max_leaf < 1 || max_leaf > 16) throw std::runtime_error("max_leaf must be in [1, 16]");
    if (prims.size() >= (1u << 27)) throw std::runtime_error("too many primitives for one BVH");
    res.order.resize(prims.size());
    for (size_t i = 0; i < prims.size(); ++i) res.order[i] = uint32_t(i);
    if (prims.empty()) {
        res.root_link = 0;
        for (int k = 0; k < 3; ++k) { res.bound_lo[k] = 0; res.bound_hi[k] = 0; }
        return res;
    }
    res.nodes.reserve(prims.size() / 2 + 1);
    Builder b(prims, res.order, res.nodes, max_leaf, traversal_cost, intersect_cost);
    Box box = b.range_box(0, uint32_t(prims.size()));
    // reserve the root slot so that an interior root is node 0
    res.root_link = b.build(0, uint32_t(prims.size()), box, 0);
    res.max_depth = b.max_depth.load();
    for (int k = 0; k < 3; ++k) { res.bound_lo[k] = box.lo[k]; res.bound_hi[k] = box.hi[k]; }
    return res;
}

int32_t collapse_bvh4(const BvhResult& b, std::vector<Bvh4Node>* out) {
    if (b.root_link < 0) return b.root_link;  // a single leaf
    struct Child {
        int32_t link;  // binary-tree link (node index or leaf)
        float lo[3], hi[3];
        float area() const {
            const float dx = std::max(0.0f, hi[0] - lo[0]), dy = std::max(0.0f, hi[1] - lo[1]),
                        dz = std::max(0.0f, hi[2] - lo[2]);
            return dx * dy + dy * dz + dz * dx;
        }
    };
    auto children_of = [&](int32_t n, Child* c) {
        const BvhNode& nd = b.nodes[size_t(n)];
        c[0] = Child{nd.link0, {nd.c0lo_x, nd.c0lo_y, nd.c0lo_z}, {nd.c0hi_x, nd.c0hi_y, nd.c0hi_z}};
        c[1] = Child{nd.link1, {nd.c1lo_x, nd.c1lo_y, nd.c1lo_z}, {nd.c1hi_x, nd.c1hi_y, nd.c1hi_z}};
    };
    // iterative depth-first build: (binary node, wide parent and slot to patch)
    struct Pending {
        int32_t bin;
        size_t parent;
        int slot;
    };
    std::vector<Pending> stack;
    out->reserve(out->size() + b.nodes.size() / 2 + 1);
    const size_t root = out->size();
    stack.push_back({0, SIZE_MAX, 0});
    while (!stack.empty()) {
        const Pending pd = stack.back();
        stack.pop_back();
        Child kids[4];
        int n = 2;
        children_of(pd.bin, kids);
        while (n < 4) {  // open the widest interior child
            int best = -1;
            float best_a = -1.0f;
            for (int k = 0; k < n; ++k)
                if (kids[k].link >= 0 && kids[k].area() > best_a) { best_a = kids[k].area(); best = k; }
            if (best < 0) break;
            Child two[2];
            children_of(kids[best].link, two);
            kids[best] = two[0];
            kids[n++] = two[1];
        }
        const size_t me = out->size();
        out->push_back(Bvh4Node{});
        if (pd.parent != SIZE_MAX) (*out)[pd.parent].link[pd.slot] = int32_t(me);
        Bvh4Node& w = (*out)[me];
        for (int k = 0; k < 4; ++k) {
            if (k < n) {
                w.lo_x[k] = kids[k].lo[0]; w.hi_x[k] = kids[k].hi[0];
                w.lo_y[k] = kids[k].lo[1]; w.hi_y[k] = kids[k].hi[1];
                w.lo_z[k] = kids[k].lo[2]; w.hi_z[k] = kids[k].hi[2];
                w.link[k] = kids[k].link;  // leaves keep their encoding; interior links patched below
            } else {
                w.lo_x[k] = w.lo_y[k] = w.lo_z[k] = 1.0f;
                w.hi_x[k] = w.hi_y[k] = w.hi_z[k] = -1.0f;
                w.link[k] = kEmptyLink;
            }
            w.pad[k] = 0;
        }
        for (int k = n - 1; k >= 0; --k)
            if (kids[k].link >= 0) stack.push_back({kids[k].link, me, k});
    }
    return int32_t(root);
}

void validate_bvh4(const std::vector<Bvh4Node>& nodes, int32_t root, uint32_t prim_first, uint32_t prim_count) {
    std::vector<uint8_t> covered(prim_count, 0);
    std::vector<uint8_t> seen;
    std::vector<int32_t> stack{root};
    size_t visits = 0;
    auto leaf = [&](int32_t link) {
        const uint32_t enc = uint32_t(~link);
        const uint32_t first = enc >> 4, count = (enc & 15) + 1;
        if (first < prim_first || first - prim_first + count > prim_count)
            throw std::runtime_error("BVH leaf outside its primitive range");
        for (uint32_t k = 0; k < count; ++k) {
            if (covered[first - prim_first + k]) throw std::runtime_error("BVH primitive in two leaves");
            covered[first - prim_first + k] = 1;
        }
    };
    while (!stack.empty()) {
        const int32_t l = stack.back();
        stack.pop_back();
        if (l == kEmptyLink) continue;
        if (l < 0) {
            leaf(l);
            continue;
        }
        if (size_t(l) >= nodes.size()) throw std::runtime_error("BVH node link out of range");
        if (seen.size() < nodes.size()) seen.resize(nodes.size(), 0);
        if (seen[size_t(l)]) throw std::runtime_error("BVH node reached twice");
        seen[size_t(l)] = 1;
        if (++visits > nodes.size()) throw std::runtime_error("BVH has a cycle");
        bool any = false;
        for (int k = 0; k < 4; ++k) {
            if (nodes[size_t(l)].link[k] != kEmptyLink) any = true;
            stack.push_back(nodes[size_t(l)].link[k]);
        }
        if (!any) throw std::runtime_error("BVH node without children");
    }
    for (uint32_t k = 0; k < prim_count; ++k)
        if (!covered[k]) throw std::runtime_error("BVH primitive in no leaf");
}

// ------------------------------------------------------------------- PLOC

namespace {

uint64_t spread21(uint32_t v) {
    uint64_t x = v & 0x1fffffu;
    x = (x | x << 32) & 0x1f00000000ffffULL;
    x = (x | x << 16) & 0x1f0000ff0000ffULL;
    x = (x | x << 8) & 0x100f00f00f00f00fULL;
    x = (x | x << 4) & 0x10c30c30c30c30c3ULL;
    x = (x | x << 2) & 0x1249249249249249ULL;
    return x;
}

float box_area(const BuildPrim& b) {
    const float dx = b.hi[0] - b.lo[0], dy = b.hi[1] - b.lo[1], dz = b.hi[2] - b.lo[2];
    return dx * dy + dy * dz + dz * dx;
}

BuildPrim box_union(const BuildPrim& a, const BuildPrim& b) {
    BuildPrim u;
    for (int k = 0; k < 3; ++k) {
        u.lo[k] = std::min(a.lo[k], b.lo[k]);
        u.hi[k] = std::max(a.hi[k], b.hi[k]);
    }
    return u;
}

// (min, max) of the position pair, compared lexicographically
bool pair_before(uint32_t i, uint32_t j1, uint32_t j2) {
    const uint32_t a1 = std::min(i, j1), b1 = std::max(i, j1), a2 = std::min(i, j2), b2 = std::max(i, j2);
    return a1 != a2 ? a1 < a2 : b1 < b2;
}

}  // namespace

uint64_t morton63(const BuildPrim& p, const float lo[3], const float inv_ext[3]) {
    uint32_t q[3];
    for (int a = 0; a < 3; ++a) {
        const float c = 0.5f * (p.lo[a] + p.hi[a]);
        float t = (c - lo[a]) * inv_ext[a];
        if (!(t >= 0.0f)) t = 0.0f;
        if (t > 1.0f) t = 1.0f;
        q[a] = uint32_t(t * 2097151.0f);
    }
    return spread21(q[0]) | spread21(q[1]) << 1 | spread21(q[2]) << 2;
}

float union_area(const BuildPrim& a, const BuildPrim& b) {
    const float dx = std::max(a.hi[0], b.hi[0]) - std::min(a.lo[0], b.lo[0]);
    const float dy = std::max(a.hi[1], b.hi[1]) - std::min(a.lo[1], b.lo[1]);
    const float dz = std::max(a.hi[2], b.hi[2]) - std::min(a.lo[2], b.lo[2]);
    return dx * dy + dy * dz + dz * dx;
}

ClusterTree ploc_build_host(const std::vector<BuildPrim>& prims, int radius) {
    ClusterTree t;
    const uint32_t n = uint32_t(prims.size());
    t.n = n;
    if (n == 0) return t;
    if (radius < 1) throw std::runtime_error("PLOC radius must be positive");
    float clo[3], chi[3], inv[3];
    for (int a = 0; a < 3; ++a) {
        clo[a] = std::numeric_limits<float>::infinity();
        chi[a] = -std::numeric_limits<float>::infinity();
    }
    for (const BuildPrim& p : prims)
        for (int a = 0; a < 3; ++a) {
            if (!std::isfinite(p.lo[a]) || !std::isfinite(p.hi[a])) throw std::runtime_error("non-finite primitive bound");
            const float c = 0.5f * (p.lo[a] + p.hi[a]);
            clo[a] = std::min(clo[a], c);
            chi[a] = std::max(chi[a], c);
        }
    for (int a = 0; a < 3; ++a) inv[a] = chi[a] > clo[a] ? 1.0f / (chi[a] - clo[a]) : 0.0f;
    std::vector<std::pair<uint64_t, uint32_t>> keys(n);
    for (uint32_t i = 0; i < n; ++i) keys[i] = {morton63(prims[i], clo, inv), i};
    std::sort(keys.begin(), keys.end());
    t.order.resize(n);
    std::vector<BuildPrim> box(size_t(2) * n - 1);
    for (uint32_t i = 0; i < n; ++i) {
        t.order[i] = keys[i].second;
        box[i] = prims[keys[i].second];
    }
    std::vector<int32_t> C(n), next_c(n), nn(n);
    for (uint32_t i = 0; i < n; ++i) C[i] = int32_t(i);
    t.left.reserve(n - 1);
    t.right.reserve(n - 1);
    t.box.reserve(n - 1);
    uint32_t m = n, next = n;
    while (m > 1) {
        for (uint32_t i = 0; i < m; ++i) {
            const uint32_t j0 = i > uint32_t(radius) ? i - uint32_t(radius) : 0;
            const uint32_t j1 = std::min(m - 1, i + uint32_t(radius));
            int32_t best = -1;
            float best_a = 0.0f;
            for (uint32_t j = j0; j <= j1; ++j) {
                if (j == i) continue;
                const float a = union_area(box[size_t(C[i])], box[size_t(C[j])]);
                if (best < 0 || a < best_a || (a == best_a && pair_before(i, j, uint32_t(best)))) {
                    best = int32_t(j);
                    best_a = a;
                }
            }
            nn[i] = best;
        }
        uint32_t merges = 0, w = 0;
        for (uint32_t i = 0; i < m; ++i) {
            const uint32_t j = uint32_t(nn[i]);
            if (uint32_t(nn[j]) == i && i < j) {
                const uint32_t k = next++;
                t.left.push_back(C[i]);
                t.right.push_back(C[j]);
                box[k] = box_union(box[size_t(C[i])], box[size_t(C[j])]);
                t.box.push_back(box[k]);
                next_c[i] = int32_t(k);
                ++merges;
            } else {
                next_c[i] = C[i];
            }
        }
        if (merges == 0) throw std::runtime_error("PLOC made no progress");
        for (uint32_t i = 0; i < m; ++i) {
            const uint32_t j = uint32_t(nn[i]);
            if (uint32_t(nn[j]) == i && j < i) continue;  // merged into position j
            C[w++] = next_c[i];
        }
        m = w;
        ++t.rounds;
    }
    t.root = C[0];
    return t;
}

BvhResult bvh_from_clusters(const ClusterTree& t, const std::vector<BuildPrim>& prims, int max_leaf,
                            float traversal_cost, float intersect_cost) {
    BvhResult res;
    const uint32_t n = t.n;
    if (max_leaf < 1 || max_leaf > 16) throw std::runtime_error("max_leaf must be in [1, 16]");
    if (n != prims.size() || t.order.size() != n || t.left.size() + 1 != std::max<size_t>(n, 1) ||
        t.right.size() != t.left.size() || t.box.size() != t.left.size())
        throw std::runtime_error("cluster tree does not match its primitives");
    if (n == 0) {
        res.root_link = 0;
        for (int k = 0; k < 3; ++k) res.bound_lo[k] = res.bound_hi[k] = 0;
        return res;
    }
    if (n >= (1u << 27)) throw std::runtime_error("too many primitives for one BVH");
    const size_t total = size_t(2) * n - 1;
    if (t.root < 0 || size_t(t.root) >= total) throw std::runtime_error("cluster tree root out of range");
    auto box_of = [&](int32_t node) -> const BuildPrim& {
        return uint32_t(node) < n ? prims[t.order[size_t(node)]] : t.box[size_t(node) - n];
    };
    // bottom-up: children are created before their parents
    std::vector<uint32_t> count(total, 1);
    std::vector<float> cost(total, intersect_cost);
    std::vector<uint8_t> leaf(total, 1);
    for (uint32_t k = 0; k + 1 < n; ++k) {
        const size_t node = size_t(n) + k;
        const int32_t l = t.left[k], r = t.right[k];
        if (l < 0 || r < 0 || size_t(l) >= node || size_t(r) >= node)
            throw std::runtime_error("cluster tree child out of order");
        count[node] = count[size_t(l)] + count[size_t(r)];
        const float A = box_area(t.box[k]);
        const float cl = cost[size_t(l)], cr = cost[size_t(r)];
        const float split = A > 0.0f ? traversal_cost + (box_area(box_of(l)) * cl + box_area(box_of(r)) * cr) / A
                                     : traversal_cost + cl + cr;
        const bool as_leaf = count[node] <= uint32_t(max_leaf) && float(count[node]) * intersect_cost <= split;
        leaf[node] = as_leaf;
        cost[node] = as_leaf ? float(count[node]) * intersect_cost : split;
    }
    res.order.reserve(n);
    std::vector<int32_t> walk;
    auto emit_leaf = [&](int32_t node) -> int32_t {
        const uint32_t first = uint32_t(res.order.size());
        walk.assign(1, node);
        while (!walk.empty()) {
            const int32_t x = walk.back();
            walk.pop_back();
            if (uint32_t(x) < n) {
                res.order.push_back(t.order[size_t(x)]);
            } else {
                walk.push_back(t.right[size_t(x) - n]);
                walk.push_back(t.left[size_t(x) - n]);
            }
        }
        return leaf_link(first, uint32_t(res.order.size()) - first);
    };
    const BuildPrim& rb = box_of(t.root);
    for (int k = 0; k < 3; ++k) {
        res.bound_lo[k] = rb.lo[k];
        res.bound_hi[k] = rb.hi[k];
    }
    if (leaf[size_t(t.root)]) {
        res.root_link = emit_leaf(t.root);
        return res;
    }
    struct Item {
        int32_t node;
        int32_t bin;
        int depth;
    };
    std::vector<Item> stack{{t.root, 0, 1}};
    res.nodes.reserve(n / 2 + 1);
    res.nodes.push_back(BvhNode{});
    res.root_link = 0;
    while (!stack.empty()) {
        const Item it = stack.back();
        stack.pop_back();
        res.max_depth = std::max(res.max_depth, it.depth);
        const int32_t kids[2] = {t.left[size_t(it.node) - n], t.right[size_t(it.node) - n]};
        int32_t links[2];
        for (int c = 0; c < 2; ++c) {
            if (leaf[size_t(kids[c])]) {
                links[c] = emit_leaf(kids[c]);
            } else {
                links[c] = int32_t(res.nodes.size());
                res.nodes.push_back(BvhNode{});
                stack.push_back({kids[c], links[c], it.depth + 1});
            }
        }
        BvhNode& nd = res.nodes[size_t(it.bin)];
        const BuildPrim& lb = box_of(kids[0]);
        const BuildPrim& rb2 = box_of(kids[1]);
        nd.c0lo_x = lb.lo[0]; nd.c0hi_x = lb.hi[0]; nd.c0lo_y = lb.lo[1]; nd.c0hi_y = lb.hi[1];
        nd.c1lo_x = rb2.lo[0]; nd.c1hi_x = rb2.hi[0]; nd.c1lo_y = rb2.lo[1]; nd.c1hi_y = rb2.hi[1];
        nd.c0lo_z = lb.lo[2]; nd.c0hi_z = lb.hi[2]; nd.c1lo_z = rb2.lo[2]; nd.c1hi_z = rb2.hi[2];
        nd.link0 = links[0];
        nd.link1 = links[1];
        nd.pad0 = nd.pad1 = 0;
    }
    if (res.order.size() != n) throw std::runtime_error("cluster tree leaves do not cover the primitives");
    return res;
}

double bvh4_sah_cost(const std::vector<Bvh4Node>& nodes, int32_t root, float traversal_cost, float intersect_cost) {
    auto slot_area = [](const Bvh4Node& w, int k) {
        const double dx = double(w.hi_x[k]) - w.lo_x[k], dy = double(w.hi_y[k]) - w.lo_y[k],
                     dz = double(w.hi_z[k]) - w.lo_z[k];
        return dx * dy + dy * dz + dz * dx;
    };
    if (root < 0) return intersect_cost * double((uint32_t(~root) & 15) + 1);
    const Bvh4Node& r = nodes[size_t(root)];
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (int k = 0; k < 4; ++k) {
        if (r.link[k] == kEmptyLink) continue;
        lo[0] = std::min(lo[0], double(r.lo_x[k])); hi[0] = std::max(hi[0], double(r.hi_x[k]));
        lo[1] = std::min(lo[1], double(r.lo_y[k])); hi[1] = std::max(hi[1], double(r.hi_y[k]));
        lo[2] = std::min(lo[2], double(r.lo_z[k])); hi[2] = std::max(hi[2], double(r.hi_z[k]));
    }
    const double a0 = std::max(1e-300, (hi[0] - lo[0]) * (hi[1] - lo[1]) + (hi[1] - lo[1]) * (hi[2] - lo[2]) +
                                           (hi[2] - lo[2]) * (hi[0] - lo[0]));
    double cost = 0;
    std::vector<std::pair<int32_t, double>> stack{{root, a0}};
    while (!stack.empty()) {
        const auto [link, area] = stack.back();
        stack.pop_back();
        cost += traversal_cost * area / a0;
        const Bvh4Node& w = nodes[size_t(link)];
        for (int k = 0; k < 4; ++k) {
            const int32_t l = w.link[k];
            if (l == kEmptyLink) continue;
            if (l < 0) cost += intersect_cost * double((uint32_t(~l) & 15) + 1) * slot_area(w, k) / a0;
            else stack.push_back({l, slot_area(w, k)});
        }
    }
    return cost;
}

int bvh4_depth(const std::vector<Bvh4Node>& nodes, int32_t root) {
    if (root < 0) return 0;
    int depth = 0;
    std::vector<std::pair<int32_t, int>> stack{{root, 1}};
    while (!stack.empty()) {
        const auto [link, d] = stack.back();
        stack.pop_back();
        depth = std::max(depth, d);
        for (int k = 0; k < 4; ++k)
            if (nodes[size_t(link)].link[k] >= 0) stack.push_back({nodes[size_t(link)].link[k], d + 1});
    }
    return depth;
}

}  // namespace atrc
