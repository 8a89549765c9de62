// Device BVH construction: parallel locally-ordered clustering (PLOC).
//
// Scene ingestion for large meshes: the reference builds its triangle BVH on
// the CPU (triangle_bvh.cpp:122-304), as does the library's binned-SAH
// builder (bvh_build.cpp), at about a microsecond per triangle on one core.
// Here the primitives are sorted by Morton code and clustered on the GPU,
// one round per launch group:
//   k_morton   63-bit Morton key of each box centre (HBM-bound, 32 B / prim)
//   sort       CUB radix sort of (key, index) pairs (stable: equal keys keep
//              the input order)
//   k_leaves   leaf boxes in sorted order, cluster list = leaves
//   per round: k_nearest   nearest neighbour within kPlocRadius positions,
//                          the window's boxes staged in shared memory
//              k_flags     mutual pairs, lower position merges
//              scan        merge slots (node n + scan) in position order
//              k_merge     union boxes of the new nodes
//              scan        surviving positions
//              k_compact   the next round's cluster list
// The topology, boxes and leaf order come back to the host, where the tree
// gets SAH leaves (bvh_from_clusters), its 4-wide collapse and its
// structural validation like every other tree.  Every float operation is
// written with round-to-nearest intrinsics and no contraction, so the result
// equals ploc_build_host's bit for bit (checked by the GPU tests).
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <limits>
#include <vector>

#include "../host/bvh_build.h"
#include "cuda_util.h"

namespace atrc {
namespace {

constexpr int kPlocBlock = 256;

__device__ __forceinline__ uint64_t spread21_dev(uint32_t v) {
    uint64_t x = v & 0x1fffffu;
    x = (x | x << 32) & 0x1f00000000ffffULL;
    x = (x | x << 16) & 0x1f0000ff0000ffULL;
    x = (x | x << 8) & 0x100f00f00f00f00fULL;
    x = (x | x << 4) & 0x10c30c30c30c30c3ULL;
    x = (x | x << 2) & 0x1249249249249249ULL;
    return x;
}

__device__ __forceinline__ uint32_t quantise21(float lo, float hi, float clo, float inv) {
    const float c = __fmul_rn(0.5f, __fadd_rn(lo, hi));
    float t = __fmul_rn(__fsub_rn(c, clo), inv);
    if (!(t >= 0.0f)) t = 0.0f;
    if (t > 1.0f) t = 1.0f;
    return __float2uint_rz(__fmul_rn(t, 2097151.0f));
}

__global__ void k_morton(const BuildPrim* __restrict__ prims, uint32_t n, float3 clo, float3 inv,
                         uint64_t* __restrict__ keys, uint32_t* __restrict__ idx) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const BuildPrim p = prims[i];
    const uint32_t qx = quantise21(p.lo[0], p.hi[0], clo.x, inv.x);
    const uint32_t qy = quantise21(p.lo[1], p.hi[1], clo.y, inv.y);
    const uint32_t qz = quantise21(p.lo[2], p.hi[2], clo.z, inv.z);
    keys[i] = spread21_dev(qx) | spread21_dev(qy) << 1 | spread21_dev(qz) << 2;
    idx[i] = i;
}

// Per-node data of the cluster tree besides boxes and children: primitive
// count, surface-area cost and whether the subtree is emitted as one leaf
// (bvh_from_clusters' rule).
struct NodeCost {
    uint32_t* count;
    float* cost;
    uint8_t* leaf;
    int max_leaf;
    float ct, ci;
};

__global__ void k_leaves(const BuildPrim* __restrict__ prims, const uint32_t* __restrict__ order, uint32_t n,
                         float4* __restrict__ blo, float4* __restrict__ bhi, int32_t* __restrict__ C, NodeCost nc) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const BuildPrim p = prims[order[i]];
    blo[i] = make_float4(p.lo[0], p.lo[1], p.lo[2], 0.0f);
    bhi[i] = make_float4(p.hi[0], p.hi[1], p.hi[2], 0.0f);
    C[i] = int32_t(i);
    nc.count[i] = 1;
    nc.cost[i] = nc.ci;
    nc.leaf[i] = 1;
}

// dx dy + dy dz + dz dx of a box (bvh_build.cpp box_area)
__device__ __forceinline__ float box_area_dev(float4 lo, float4 hi) {
    const float dx = __fsub_rn(hi.x, lo.x), dy = __fsub_rn(hi.y, lo.y), dz = __fsub_rn(hi.z, lo.z);
    return __fadd_rn(__fadd_rn(__fmul_rn(dx, dy), __fmul_rn(dy, dz)), __fmul_rn(dz, dx));
}

__device__ __forceinline__ float union_area_dev(float4 alo, float4 ahi, float4 blo, float4 bhi) {
    const float dx = __fsub_rn(fmaxf(ahi.x, bhi.x), fminf(alo.x, blo.x));
    const float dy = __fsub_rn(fmaxf(ahi.y, bhi.y), fminf(alo.y, blo.y));
    const float dz = __fsub_rn(fmaxf(ahi.z, bhi.z), fminf(alo.z, blo.z));
    return __fadd_rn(__fadd_rn(__fmul_rn(dx, dy), __fmul_rn(dy, dz)), __fmul_rn(dz, dx));
}

// (min, max) of the position pair, compared lexicographically
__device__ __forceinline__ bool pair_before_dev(uint32_t i, uint32_t j1, uint32_t j2) {
    const uint32_t a1 = min(i, j1), b1 = max(i, j1), a2 = min(i, j2), b2 = max(i, j2);
    return a1 != a2 ? a1 < a2 : b1 < b2;
}

template <int R>
__global__ void __launch_bounds__(kPlocBlock) k_nearest(const int32_t* __restrict__ C, uint32_t m,
                                                        const float4* __restrict__ blo,
                                                        const float4* __restrict__ bhi, int32_t* __restrict__ nn) {
    __shared__ float4 slo[kPlocBlock + 2 * R], shi[kPlocBlock + 2 * R];
    const int64_t b0 = int64_t(blockIdx.x) * kPlocBlock;
    for (int s = threadIdx.x; s < kPlocBlock + 2 * R; s += blockDim.x) {
        const int64_t j = b0 - R + s;
        if (j >= 0 && j < int64_t(m)) {
            const int32_t c = C[j];
            slo[s] = blo[c];
            shi[s] = bhi[c];
        }
    }
    __syncthreads();
    const int64_t i = b0 + threadIdx.x;
    if (i >= int64_t(m)) return;
    const float4 ilo = slo[threadIdx.x + R], ihi = shi[threadIdx.x + R];
    const int64_t j0 = i > R ? i - R : 0, j1 = min(i + R, int64_t(m) - 1);
    int32_t best = -1;
    float best_a = 0.0f;
    for (int64_t j = j0; j <= j1; ++j) {
        if (j == i) continue;
        const int sj = int(j - b0) + R;
        const float a = union_area_dev(ilo, ihi, slo[sj], shi[sj]);
        if (best < 0 || a < best_a || (a == best_a && pair_before_dev(uint32_t(i), uint32_t(j), uint32_t(best)))) {
            best = int32_t(j);
            best_a = a;
        }
    }
    nn[i] = best;
}

__global__ void k_flags(const int32_t* __restrict__ nn, uint32_t m, int32_t* __restrict__ flag) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i > m) return;
    if (i == m) {
        flag[i] = 0;
        return;
    }
    const uint32_t j = uint32_t(nn[i]);
    flag[i] = (uint32_t(nn[j]) == i && i < j) ? 1 : 0;
}

__global__ void k_merge(const int32_t* __restrict__ C, const int32_t* __restrict__ nn, const int32_t* __restrict__ offs,
                        uint32_t m, uint32_t n, uint32_t base, float4* __restrict__ blo, float4* __restrict__ bhi,
                        int32_t* __restrict__ left, int32_t* __restrict__ right, int32_t* __restrict__ Cn,
                        int32_t* __restrict__ keep, NodeCost nc) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i > m) return;
    if (i == m) {
        keep[i] = 0;
        return;
    }
    const uint32_t j = uint32_t(nn[i]);
    const bool mutual = uint32_t(nn[j]) == i;
    if (mutual && i < j) {
        const uint32_t k = base + uint32_t(offs[i]);
        const int32_t a = C[i], b = C[j];
        left[k - n] = a;
        right[k - n] = b;
        const float4 alo = blo[a], ahi = bhi[a], clo = blo[b], chi = bhi[b];
        const float4 ulo = make_float4(fminf(alo.x, clo.x), fminf(alo.y, clo.y), fminf(alo.z, clo.z), 0.0f);
        const float4 uhi = make_float4(fmaxf(ahi.x, chi.x), fmaxf(ahi.y, chi.y), fmaxf(ahi.z, chi.z), 0.0f);
        blo[k] = ulo;
        bhi[k] = uhi;
        // surface-area leaf decision (bvh_from_clusters): children are final
        const uint32_t cnt = nc.count[a] + nc.count[b];
        const float A = box_area_dev(ulo, uhi);
        const float ca = nc.cost[a], cb = nc.cost[b];
        const float split =
            A > 0.0f ? __fadd_rn(nc.ct, __fdiv_rn(__fadd_rn(__fmul_rn(box_area_dev(alo, ahi), ca),
                                                             __fmul_rn(box_area_dev(clo, chi), cb)), A))
                     : __fadd_rn(__fadd_rn(nc.ct, ca), cb);
        const float as_leaf_cost = __fmul_rn(float(cnt), nc.ci);
        const bool as_leaf = cnt <= uint32_t(nc.max_leaf) && as_leaf_cost <= split;
        nc.count[k] = cnt;
        nc.cost[k] = as_leaf ? as_leaf_cost : split;
        nc.leaf[k] = as_leaf ? 1 : 0;
        Cn[i] = int32_t(k);
        keep[i] = 1;
    } else if (mutual) {
        keep[i] = 0;  // merged into position j
    } else {
        Cn[i] = C[i];
        keep[i] = 1;
    }
}

__global__ void k_compact(const int32_t* __restrict__ Cn, const int32_t* __restrict__ keep,
                          const int32_t* __restrict__ pos, uint32_t m, int32_t* __restrict__ C) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m && keep[i]) C[pos[i]] = Cn[i];
}

// ------------------------------------------------- 4-wide emission

// Children of a 4-wide node made from binary node k: open the widest
// interior child until there are four (collapse_bvh4's greedy rule, the
// opened child's second half appended).  Returns the child count.
__device__ __forceinline__ float slot_area_dev(float4 lo, float4 hi) {
    const float dx = fmaxf(0.0f, __fsub_rn(hi.x, lo.x)), dy = fmaxf(0.0f, __fsub_rn(hi.y, lo.y)),
                dz = fmaxf(0.0f, __fsub_rn(hi.z, lo.z));
    return __fadd_rn(__fadd_rn(__fmul_rn(dx, dy), __fmul_rn(dy, dz)), __fmul_rn(dz, dx));
}

__device__ __forceinline__ int wide_kids(uint32_t k, uint32_t n, const int32_t* __restrict__ left,
                                         const int32_t* __restrict__ right, const uint8_t* __restrict__ leaf,
                                         const float4* __restrict__ blo, const float4* __restrict__ bhi,
                                         uint32_t kids[4]) {
    kids[0] = uint32_t(left[k - n]);
    kids[1] = uint32_t(right[k - n]);
    int nk = 2;
    while (nk < 4) {
        int best = -1;
        float best_a = -1.0f;
        for (int q = 0; q < nk; ++q) {
            const uint32_t c = kids[q];
            if (leaf[c]) continue;
            const float a = slot_area_dev(blo[c], bhi[c]);
            if (a > best_a) {
                best_a = a;
                best = q;
            }
        }
        if (best < 0) break;
        const uint32_t c = kids[best];
        kids[best] = uint32_t(left[c - n]);
        kids[nk++] = uint32_t(right[c - n]);
    }
    return nk;
}

// One merge round, walked from the root down (rounds in reverse order):
// leaf-order offsets of the children, and which interior nodes head a
// 4-wide node.
__global__ void k_topdown(uint32_t b, uint32_t e, uint32_t n, const int32_t* __restrict__ left,
                          const int32_t* __restrict__ right, const uint32_t* __restrict__ count,
                          const uint8_t* __restrict__ leaf, const float4* __restrict__ blo,
                          const float4* __restrict__ bhi, uint32_t* __restrict__ first, int32_t* __restrict__ wide) {
    const uint32_t k = b + blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= e) return;
    const uint32_t l = uint32_t(left[k - n]), r = uint32_t(right[k - n]);
    const uint32_t f = first[k];
    first[l] = f;
    first[r] = f + count[l];
    if (wide[k]) {
        uint32_t kids[4];
        const int nk = wide_kids(k, n, left, right, leaf, blo, bhi, kids);
        for (int q = 0; q < nk; ++q)
            if (!leaf[kids[q]]) wide[kids[q]] = 1;
    }
}

__global__ void k_leaf_order(const uint32_t* __restrict__ order, const uint32_t* __restrict__ first, uint32_t n,
                             uint32_t* __restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[first[i]] = order[i];
}

__global__ void k_emit(uint32_t n, uint32_t total, const int32_t* __restrict__ left, const int32_t* __restrict__ right,
                       const uint32_t* __restrict__ count, const uint8_t* __restrict__ leaf,
                       const float4* __restrict__ blo, const float4* __restrict__ bhi,
                       const uint32_t* __restrict__ first, const int32_t* __restrict__ wide,
                       const int32_t* __restrict__ widx, Bvh4Node* __restrict__ out) {
    const uint32_t k = n + blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= total || !wide[k]) return;
    uint32_t kids[4];
    const int nk = wide_kids(k, n, left, right, leaf, blo, bhi, kids);
    Bvh4Node w;
    for (int q = 0; q < 4; ++q) {
        if (q < nk) {
            const uint32_t c = kids[q];
            const float4 lo = blo[c], hi = bhi[c];
            w.lo_x[q] = lo.x; w.hi_x[q] = hi.x;
            w.lo_y[q] = lo.y; w.hi_y[q] = hi.y;
            w.lo_z[q] = lo.z; w.hi_z[q] = hi.z;
            w.link[q] = leaf[c] ? ~int32_t((first[c] << 4) | (count[c] - 1)) : widx[c];
        } else {
            w.lo_x[q] = w.lo_y[q] = w.lo_z[q] = 1.0f;
            w.hi_x[q] = w.hi_y[q] = w.hi_z[q] = -1.0f;
            w.link[q] = kEmptyLink;
        }
        w.pad[q] = 0;
    }
    out[widx[k]] = w;
}

struct StreamGuard {
    cudaStream_t s = nullptr;
    StreamGuard() { CK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking)); }
    ~StreamGuard() {
        if (s) cudaStreamDestroy(s);
    }
};

inline unsigned blocks_for(size_t n, int threads) { return unsigned((n + threads - 1) / threads); }

// Device buffers of one PLOC build and the node range of each merge round.
struct Ploc {
    uint32_t n = 0;
    size_t total = 0;
    int rounds = 0;
    std::vector<uint32_t> round_begin;  // first node of each round (+ total at the end)
    DevBuf prims, keys, keys2, idx, idx2, lo, hi, left, right, C, Cn, nn, flag, offs, keep, pos, tmp;
    DevBuf count, cost, leaf;
    const uint32_t* order() const { return idx2.as<uint32_t>(); }
};

void centre_bound(const std::vector<BuildPrim>& prims, float clo[3], float inv[3]) {
    float chi[3];
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
}

// Sort and cluster on the device; leaves the tree in P's buffers.
void run_ploc(const std::vector<BuildPrim>& prims, int max_leaf, float ct, float ci, cudaStream_t s, Ploc* P) {
    static_assert(sizeof(BuildPrim) == 24, "BuildPrim layout");
    const uint32_t n = uint32_t(prims.size());
    if (n == 0) throw std::runtime_error("PLOC over no primitives");
    if (prims.size() >= (size_t(1) << 27)) throw std::runtime_error("too many primitives for one BVH");
    if (max_leaf < 1 || max_leaf > 16) throw std::runtime_error("max_leaf must be in [1, 16]");
    float clo[3], inv[3];
    centre_bound(prims, clo, inv);
    P->n = n;
    P->total = size_t(2) * n - 1;
    const size_t total = P->total;
    P->prims.alloc(size_t(n) * sizeof(BuildPrim));
    CK(cudaMemcpyAsync(P->prims.p, prims.data(), size_t(n) * sizeof(BuildPrim), cudaMemcpyHostToDevice, s));
    P->keys.alloc(size_t(n) * 8);
    P->keys2.alloc(size_t(n) * 8);
    P->idx.alloc(size_t(n) * 4);
    P->idx2.alloc(size_t(n) * 4);
    P->lo.alloc(total * sizeof(float4));
    P->hi.alloc(total * sizeof(float4));
    P->left.alloc(std::max<size_t>(n - 1, 1) * 4);
    P->right.alloc(std::max<size_t>(n - 1, 1) * 4);
    P->C.alloc(size_t(n) * 4);
    P->Cn.alloc(size_t(n) * 4);
    P->nn.alloc(size_t(n) * 4);
    P->flag.alloc((size_t(n) + 1) * 4);
    P->offs.alloc((size_t(n) + 1) * 4);
    P->keep.alloc((size_t(n) + 1) * 4);
    P->pos.alloc((size_t(n) + 1) * 4);
    P->count.alloc(total * 4);
    P->cost.alloc(total * 4);
    P->leaf.alloc(total);
    NodeCost nc{P->count.as<uint32_t>(), P->cost.as<float>(), P->leaf.as<uint8_t>(), max_leaf, ct, ci};
    size_t sort_bytes = 0, scan_bytes = 0;
    CK(cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, P->keys.as<uint64_t>(), P->keys2.as<uint64_t>(),
                                       P->idx.as<uint32_t>(), P->idx2.as<uint32_t>(), int(n), 0, 63, s));
    CK(cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, P->flag.as<int32_t>(), P->offs.as<int32_t>(),
                                     int(total) + 1, s));
    P->tmp.alloc(std::max<size_t>(std::max(sort_bytes, scan_bytes), 16));

    k_morton<<<blocks_for(n, 256), 256, 0, s>>>(P->prims.as<BuildPrim>(), n, make_float3(clo[0], clo[1], clo[2]),
                                                make_float3(inv[0], inv[1], inv[2]), P->keys.as<uint64_t>(),
                                                P->idx.as<uint32_t>());
    CK(cudaGetLastError());
    size_t tb = P->tmp.bytes;
    CK(cub::DeviceRadixSort::SortPairs(P->tmp.p, tb, P->keys.as<uint64_t>(), P->keys2.as<uint64_t>(),
                                       P->idx.as<uint32_t>(), P->idx2.as<uint32_t>(), int(n), 0, 63, s));
    float4* blo = P->lo.as<float4>();
    float4* bhi = P->hi.as<float4>();
    k_leaves<<<blocks_for(n, 256), 256, 0, s>>>(P->prims.as<BuildPrim>(), P->order(), n, blo, bhi,
                                                P->C.as<int32_t>(), nc);
    CK(cudaGetLastError());

    int32_t* C = P->C.as<int32_t>();
    int32_t* nn = P->nn.as<int32_t>();
    int32_t* flag = P->flag.as<int32_t>();
    int32_t* offs = P->offs.as<int32_t>();
    int32_t* keep = P->keep.as<int32_t>();
    int32_t* pos = P->pos.as<int32_t>();
    uint32_t m = n, next = n;
    int32_t merges_h = 0;
    P->round_begin.clear();
    // every round merges at least one pair (the pair with the least key is
    // mutual), so n - 1 rounds bound the loop; real inputs need tens
    while (m > 1) {
        if (P->rounds >= int(n)) throw std::runtime_error("PLOC did not converge");
        k_nearest<kPlocRadius><<<blocks_for(m, kPlocBlock), kPlocBlock, 0, s>>>(C, m, blo, bhi, nn);
        k_flags<<<blocks_for(size_t(m) + 1, 256), 256, 0, s>>>(nn, m, flag);
        tb = P->tmp.bytes;
        CK(cub::DeviceScan::ExclusiveSum(P->tmp.p, tb, flag, offs, int(m) + 1, s));
        CK(cudaMemcpyAsync(&merges_h, offs + m, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        if (merges_h <= 0 || uint32_t(merges_h) > m / 2) throw std::runtime_error("PLOC made no progress");
        k_merge<<<blocks_for(size_t(m) + 1, 256), 256, 0, s>>>(C, nn, offs, m, n, next, blo, bhi,
                                                               P->left.as<int32_t>(), P->right.as<int32_t>(),
                                                               P->Cn.as<int32_t>(), keep, nc);
        tb = P->tmp.bytes;
        CK(cub::DeviceScan::ExclusiveSum(P->tmp.p, tb, keep, pos, int(m) + 1, s));
        k_compact<<<blocks_for(m, 256), 256, 0, s>>>(P->Cn.as<int32_t>(), keep, pos, m, C);
        CK(cudaGetLastError());
        P->round_begin.push_back(next);
        next += uint32_t(merges_h);
        m -= uint32_t(merges_h);
        ++P->rounds;
    }
    P->round_begin.push_back(next);
    if (next != uint32_t(total)) throw std::runtime_error("PLOC merge count mismatch");
}

}  // namespace

ClusterTree ploc_build_device(const std::vector<BuildPrim>& prims, int device, int radius) {
    if (radius != kPlocRadius) throw std::runtime_error("the device PLOC build is compiled for one search radius");
    ClusterTree t;
    const uint32_t n = uint32_t(prims.size());
    t.n = n;
    if (n == 0) return t;
    CK(cudaSetDevice(device));
    StreamGuard sg;
    cudaStream_t s = sg.s;
    Ploc P;
    run_ploc(prims, 4, 1.0f, 1.0f, s, &P);
    t.rounds = P.rounds;
    t.order.resize(n);
    CK(cudaMemcpyAsync(t.order.data(), P.order(), size_t(n) * 4, cudaMemcpyDeviceToHost, s));
    t.root = int32_t(P.total - 1);  // the last merge makes the root
    std::vector<float4> lo4(n - 1), hi4(n - 1);
    t.left.resize(n - 1);
    t.right.resize(n - 1);
    if (n > 1) {
        CK(cudaMemcpyAsync(t.left.data(), P.left.p, size_t(n - 1) * 4, cudaMemcpyDeviceToHost, s));
        CK(cudaMemcpyAsync(t.right.data(), P.right.p, size_t(n - 1) * 4, cudaMemcpyDeviceToHost, s));
        CK(cudaMemcpyAsync(lo4.data(), P.lo.as<float4>() + n, size_t(n - 1) * sizeof(float4), cudaMemcpyDeviceToHost, s));
        CK(cudaMemcpyAsync(hi4.data(), P.hi.as<float4>() + n, size_t(n - 1) * sizeof(float4), cudaMemcpyDeviceToHost, s));
    }
    CK(cudaStreamSynchronize(s));
    t.box.resize(n - 1);
    for (uint32_t k = 0; k + 1 < n; ++k) {
        BuildPrim& b = t.box[k];
        b.lo[0] = lo4[k].x; b.lo[1] = lo4[k].y; b.lo[2] = lo4[k].z;
        b.hi[0] = hi4[k].x; b.hi[1] = hi4[k].y; b.hi[2] = hi4[k].z;
    }
    return t;
}

WideBvh ploc_wide_device(const std::vector<BuildPrim>& prims, int device, int max_leaf, float traversal_cost,
                         float intersect_cost) {
    WideBvh w;
    const uint32_t n = uint32_t(prims.size());
    if (n == 0) throw std::runtime_error("BVH over no primitives");
    if (n == 1) {
        w.order = {0};
        w.root = leaf_link(0, 1);
        for (int a = 0; a < 3; ++a) {
            w.bound_lo[a] = prims[0].lo[a];
            w.bound_hi[a] = prims[0].hi[a];
        }
        return w;
    }
    CK(cudaSetDevice(device));
    StreamGuard sg;
    cudaStream_t s = sg.s;
    Ploc P;
    run_ploc(prims, max_leaf, traversal_cost, intersect_cost, s, &P);
    w.rounds = P.rounds;
    const size_t total = P.total;
    const uint32_t root = uint32_t(total - 1);
    DevBuf first, wide, widx, order_out;
    first.alloc(total * 4);
    wide.alloc((total + 1) * 4);
    widx.alloc((total + 1) * 4);
    order_out.alloc(size_t(n) * 4);
    CK(cudaMemsetAsync(wide.p, 0, (total + 1) * 4, s));
    CK(cudaMemsetAsync(first.as<uint32_t>() + root, 0, 4, s));
    uint8_t root_leaf = 0;
    CK(cudaMemcpyAsync(&root_leaf, P.leaf.as<uint8_t>() + root, 1, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    const int32_t one = 1;
    if (!root_leaf) CK(cudaMemcpyAsync(wide.as<int32_t>() + root, &one, 4, cudaMemcpyHostToDevice, s));
    const float4* blo = P.lo.as<float4>();
    const float4* bhi = P.hi.as<float4>();
    // root to leaves: round r's nodes have their parents in later rounds
    for (int r = P.rounds - 1; r >= 0; --r) {
        const uint32_t b = P.round_begin[size_t(r)], e = P.round_begin[size_t(r) + 1];
        k_topdown<<<blocks_for(e - b, 256), 256, 0, s>>>(b, e, n, P.left.as<int32_t>(), P.right.as<int32_t>(),
                                                         P.count.as<uint32_t>(), P.leaf.as<uint8_t>(), blo, bhi,
                                                         first.as<uint32_t>(), wide.as<int32_t>());
    }
    k_leaf_order<<<blocks_for(n, 256), 256, 0, s>>>(P.order(), first.as<uint32_t>(), n, order_out.as<uint32_t>());
    CK(cudaGetLastError());
    size_t tb = P.tmp.bytes;
    CK(cub::DeviceScan::ExclusiveSum(P.tmp.p, tb, wide.as<int32_t>(), widx.as<int32_t>(), int(total) + 1, s));
    int32_t nwide = 0;
    CK(cudaMemcpyAsync(&nwide, widx.as<int32_t>() + total, 4, cudaMemcpyDeviceToHost, s));
    w.order.resize(n);
    CK(cudaMemcpyAsync(w.order.data(), order_out.p, size_t(n) * 4, cudaMemcpyDeviceToHost, s));
    float4 rlo, rhi;
    CK(cudaMemcpyAsync(&rlo, blo + root, sizeof(float4), cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(&rhi, bhi + root, sizeof(float4), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    w.bound_lo[0] = rlo.x; w.bound_lo[1] = rlo.y; w.bound_lo[2] = rlo.z;
    w.bound_hi[0] = rhi.x; w.bound_hi[1] = rhi.y; w.bound_hi[2] = rhi.z;
    if (root_leaf) {
        w.root = leaf_link(0, n);
        return w;
    }
    if (nwide <= 0 || size_t(nwide) > total) throw std::runtime_error("4-wide node count out of range");
    DevBuf nodes;
    nodes.alloc(size_t(nwide) * sizeof(Bvh4Node));
    k_emit<<<blocks_for(n - 1, 256), 256, 0, s>>>(n, uint32_t(total), P.left.as<int32_t>(), P.right.as<int32_t>(),
                                                  P.count.as<uint32_t>(), P.leaf.as<uint8_t>(), blo, bhi,
                                                  first.as<uint32_t>(), wide.as<int32_t>(), widx.as<int32_t>(),
                                                  nodes.as<Bvh4Node>());
    CK(cudaGetLastError());
    w.nodes.resize(size_t(nwide));
    CK(cudaMemcpyAsync(w.nodes.data(), nodes.p, size_t(nwide) * sizeof(Bvh4Node), cudaMemcpyDeviceToHost, s));
    int32_t root_idx = 0;
    CK(cudaMemcpyAsync(&root_idx, widx.as<int32_t>() + root, 4, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    w.root = root_idx;
    return w;
}

}  // namespace atrc


// ------------------------------------------------------------------ C ABI

#include <chrono>
#include <cstring>

#include "../../../include/atrc_cuda.h"

namespace {

std::vector<atrc::BuildPrim> prims_from(const float* boxes, uint64_t n) {
    std::vector<atrc::BuildPrim> prims(n);
    std::memcpy(prims.data(), boxes, n * sizeof(atrc::BuildPrim));
    return prims;
}

template <class F>
int guarded_bvh(F&& f) {
    try {
        return f();
    } catch (const atrc::CudaError& e) {
        atrc::set_last_error(e.what());
        return ATRC_ERR_CUDA;
    } catch (const std::bad_alloc&) {
        atrc::set_last_error("host allocation failed");
        return ATRC_ERR_OUT_OF_MEMORY;
    } catch (const std::exception& e) {
        atrc::set_last_error(e.what());
        return ATRC_ERR_INVALID_ARG;
    }
}

}  // namespace

extern "C" {

int atrc_bvh_build(int32_t builder, int32_t device, const float* boxes, uint64_t n, AtrcBvhBuildInfo* info) {
    if (!boxes || !info || n == 0) {
        atrc::set_last_error("atrc_bvh_build: null argument or no boxes");
        return ATRC_ERR_INVALID_ARG;
    }
    if (builder != ATRC_BVH_SAH && builder != ATRC_BVH_PLOC) {
        atrc::set_last_error("atrc_bvh_build: builder must be ATRC_BVH_SAH or ATRC_BVH_PLOC");
        return ATRC_ERR_INVALID_ARG;
    }
    return guarded_bvh([&] {
        const std::vector<atrc::BuildPrim> prims = prims_from(boxes, n);
        const auto t0 = std::chrono::steady_clock::now();
        atrc::WideBvh w;
        if (builder == ATRC_BVH_PLOC && device >= 0) {
            w = atrc::ploc_wide_device(prims, device);
        } else {
            atrc::BvhResult b = builder == ATRC_BVH_PLOC
                                    ? atrc::bvh_from_clusters(atrc::ploc_build_host(prims), prims, 4)
                                    : atrc::build_bvh(prims, 4);
            w.rounds = 0;
            w.root = atrc::collapse_bvh4(b, &w.nodes);
            w.order = std::move(b.order);
        }
        atrc::validate_bvh4(w.nodes, w.root, 0, uint32_t(n));
        info->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        info->sah_cost = atrc::bvh4_sah_cost(w.nodes, w.root);
        info->nodes = w.nodes.size();
        info->rounds = w.rounds;
        info->max_depth = atrc::bvh4_depth(w.nodes, w.root);
        return int(ATRC_OK);
    });
}

int atrc_bvh_cluster_tree(int32_t device, const float* boxes, uint64_t n, uint32_t* order, int32_t* left,
                          int32_t* right, float* node_boxes, int32_t* root, int32_t* rounds) {
    if (!boxes || !order || !root || !rounds || n == 0 || (n > 1 && (!left || !right || !node_boxes))) {
        atrc::set_last_error("atrc_bvh_cluster_tree: null argument or no boxes");
        return ATRC_ERR_INVALID_ARG;
    }
    return guarded_bvh([&] {
        const std::vector<atrc::BuildPrim> prims = prims_from(boxes, n);
        const atrc::ClusterTree t = device < 0 ? atrc::ploc_build_host(prims) : atrc::ploc_build_device(prims, device);
        std::memcpy(order, t.order.data(), n * sizeof(uint32_t));
        if (n > 1) {
            std::memcpy(left, t.left.data(), (n - 1) * sizeof(int32_t));
            std::memcpy(right, t.right.data(), (n - 1) * sizeof(int32_t));
            std::memcpy(node_boxes, t.box.data(), (n - 1) * sizeof(atrc::BuildPrim));
        }
        *root = t.root;
        *rounds = t.rounds;
        return int(ATRC_OK);
    });
}

}  // extern "C"
