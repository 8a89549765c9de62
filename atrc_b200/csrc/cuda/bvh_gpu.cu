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

__global__ void k_leaves(const BuildPrim* __restrict__ prims, const uint32_t* __restrict__ order, uint32_t n,
                         float4* __restrict__ blo, float4* __restrict__ bhi, int32_t* __restrict__ C) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const BuildPrim p = prims[order[i]];
    blo[i] = make_float4(p.lo[0], p.lo[1], p.lo[2], 0.0f);
    bhi[i] = make_float4(p.hi[0], p.hi[1], p.hi[2], 0.0f);
    C[i] = int32_t(i);
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
                        int32_t* __restrict__ keep) {
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
        blo[k] = make_float4(fminf(alo.x, clo.x), fminf(alo.y, clo.y), fminf(alo.z, clo.z), 0.0f);
        bhi[k] = make_float4(fmaxf(ahi.x, chi.x), fmaxf(ahi.y, chi.y), fmaxf(ahi.z, chi.z), 0.0f);
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

struct StreamGuard {
    cudaStream_t s = nullptr;
    StreamGuard() { CK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking)); }
    ~StreamGuard() {
        if (s) cudaStreamDestroy(s);
    }
};

inline unsigned blocks_for(size_t n, int threads) { return unsigned((n + threads - 1) / threads); }

}  // namespace

ClusterTree ploc_build_device(const std::vector<BuildPrim>& prims, int device, int radius) {
    static_assert(sizeof(BuildPrim) == 24, "BuildPrim layout");
    if (radius != kPlocRadius) throw std::runtime_error("the device PLOC build is compiled for one search radius");
    ClusterTree t;
    const uint32_t n = uint32_t(prims.size());
    t.n = n;
    if (n == 0) return t;
    if (prims.size() >= (size_t(1) << 30)) throw std::runtime_error("too many primitives for the device BVH build");
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

    CK(cudaSetDevice(device));
    StreamGuard sg;
    cudaStream_t s = sg.s;
    const size_t total = size_t(2) * n - 1;
    DevBuf d_prims, d_keys, d_keys2, d_idx, d_idx2, d_lo, d_hi, d_left, d_right, d_C, d_Cn, d_nn, d_flag, d_offs,
        d_keep, d_pos, d_tmp;
    d_prims.alloc(size_t(n) * sizeof(BuildPrim));
    CK(cudaMemcpyAsync(d_prims.p, prims.data(), size_t(n) * sizeof(BuildPrim), cudaMemcpyHostToDevice, s));
    d_keys.alloc(size_t(n) * 8);
    d_keys2.alloc(size_t(n) * 8);
    d_idx.alloc(size_t(n) * 4);
    d_idx2.alloc(size_t(n) * 4);
    d_lo.alloc(total * sizeof(float4));
    d_hi.alloc(total * sizeof(float4));
    d_left.alloc(std::max<size_t>(n - 1, 1) * 4);
    d_right.alloc(std::max<size_t>(n - 1, 1) * 4);
    d_C.alloc(size_t(n) * 4);
    d_Cn.alloc(size_t(n) * 4);
    d_nn.alloc(size_t(n) * 4);
    d_flag.alloc((size_t(n) + 1) * 4);
    d_offs.alloc((size_t(n) + 1) * 4);
    d_keep.alloc((size_t(n) + 1) * 4);
    d_pos.alloc((size_t(n) + 1) * 4);
    size_t sort_bytes = 0, scan_bytes = 0;
    CK(cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, d_keys.as<uint64_t>(), d_keys2.as<uint64_t>(),
                                       d_idx.as<uint32_t>(), d_idx2.as<uint32_t>(), int(n), 0, 63, s));
    CK(cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, d_flag.as<int32_t>(), d_offs.as<int32_t>(), int(n) + 1, s));
    d_tmp.alloc(std::max<size_t>(std::max(sort_bytes, scan_bytes), 16));

    k_morton<<<blocks_for(n, 256), 256, 0, s>>>(d_prims.as<BuildPrim>(), n, make_float3(clo[0], clo[1], clo[2]),
                                                make_float3(inv[0], inv[1], inv[2]), d_keys.as<uint64_t>(),
                                                d_idx.as<uint32_t>());
    CK(cudaGetLastError());
    size_t tb = d_tmp.bytes;
    CK(cub::DeviceRadixSort::SortPairs(d_tmp.p, tb, d_keys.as<uint64_t>(), d_keys2.as<uint64_t>(),
                                       d_idx.as<uint32_t>(), d_idx2.as<uint32_t>(), int(n), 0, 63, s));
    const uint32_t* order = d_idx2.as<uint32_t>();
    float4* blo = d_lo.as<float4>();
    float4* bhi = d_hi.as<float4>();
    k_leaves<<<blocks_for(n, 256), 256, 0, s>>>(d_prims.as<BuildPrim>(), order, n, blo, bhi, d_C.as<int32_t>());
    CK(cudaGetLastError());

    int32_t* C = d_C.as<int32_t>();
    int32_t* nn = d_nn.as<int32_t>();
    int32_t* flag = d_flag.as<int32_t>();
    int32_t* offs = d_offs.as<int32_t>();
    int32_t* keep = d_keep.as<int32_t>();
    int32_t* pos = d_pos.as<int32_t>();
    uint32_t m = n, next = n;
    int32_t merges_h = 0;
    // every round merges at least one pair (the pair with the least key is
    // mutual), so n - 1 rounds bound the loop; real inputs need tens
    while (m > 1) {
        if (t.rounds >= int(n)) throw std::runtime_error("PLOC did not converge");
        k_nearest<kPlocRadius><<<blocks_for(m, kPlocBlock), kPlocBlock, 0, s>>>(C, m, blo, bhi, nn);
        k_flags<<<blocks_for(size_t(m) + 1, 256), 256, 0, s>>>(nn, m, flag);
        tb = d_tmp.bytes;
        CK(cub::DeviceScan::ExclusiveSum(d_tmp.p, tb, flag, offs, int(m) + 1, s));
        CK(cudaMemcpyAsync(&merges_h, offs + m, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        if (merges_h <= 0 || uint32_t(merges_h) > m / 2) throw std::runtime_error("PLOC made no progress");
        k_merge<<<blocks_for(size_t(m) + 1, 256), 256, 0, s>>>(C, nn, offs, m, n, next, blo, bhi, d_left.as<int32_t>(),
                                                               d_right.as<int32_t>(), d_Cn.as<int32_t>(), keep);
        tb = d_tmp.bytes;
        CK(cub::DeviceScan::ExclusiveSum(d_tmp.p, tb, keep, pos, int(m) + 1, s));
        k_compact<<<blocks_for(m, 256), 256, 0, s>>>(d_Cn.as<int32_t>(), keep, pos, m, C);
        CK(cudaGetLastError());
        next += uint32_t(merges_h);
        m -= uint32_t(merges_h);
        ++t.rounds;
    }
    if (next != uint32_t(total)) throw std::runtime_error("PLOC merge count mismatch");
    // results back to the host
    t.order.resize(n);
    CK(cudaMemcpyAsync(t.order.data(), order, size_t(n) * 4, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(&t.root, C, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    std::vector<float4> lo4(n - 1), hi4(n - 1);
    t.left.resize(n - 1);
    t.right.resize(n - 1);
    if (n > 1) {
        CK(cudaMemcpyAsync(t.left.data(), d_left.p, size_t(n - 1) * 4, cudaMemcpyDeviceToHost, s));
        CK(cudaMemcpyAsync(t.right.data(), d_right.p, size_t(n - 1) * 4, cudaMemcpyDeviceToHost, s));
        CK(cudaMemcpyAsync(lo4.data(), blo + n, size_t(n - 1) * sizeof(float4), cudaMemcpyDeviceToHost, s));
        CK(cudaMemcpyAsync(hi4.data(), bhi + n, size_t(n - 1) * sizeof(float4), cudaMemcpyDeviceToHost, s));
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
        atrc::BvhResult b;
        int rounds = 0;
        if (builder == ATRC_BVH_PLOC) {
            atrc::ClusterTree t = atrc::ploc_build_device(prims, device);
            rounds = t.rounds;
            b = atrc::bvh_from_clusters(t, prims, 4);
        } else {
            b = atrc::build_bvh(prims, 4);
        }
        std::vector<atrc::Bvh4Node> nodes;
        const int32_t root = atrc::collapse_bvh4(b, &nodes);
        atrc::validate_bvh4(nodes, root, 0, uint32_t(n));
        info->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        info->sah_cost = atrc::bvh4_sah_cost(nodes, root);
        info->nodes = nodes.size();
        info->rounds = rounds;
        info->max_depth = b.max_depth;
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
