// Encoding of guide queries into the network's input rows, written straight
// into the K-major tile layout of the tensor-core operands (dev_tc.cuh), in
// shared or global memory.  Shared by the training kernel and by the
// wavefront's feature kernel, which encodes each query once into a global
// staging buffer of 128-row tiles that the inference kernel copies whole.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "dev_guide.cuh"
#include "dev_tc.cuh"

namespace atrc {
namespace dev {

constexpr int kGuideTile = 128;                                 // rows per MMA tile
constexpr int kGuideTileBytes = kGuideTile * kGuideIn * 2;      // one encoded input tile
constexpr int kHashIn = kHashLevels * kHashFeatures;            // 32 inputs from the grid

template <class T>
__device__ __forceinline__ float2 table_pair(const T* t, size_t i);
template <>
__device__ __forceinline__ float2 table_pair<float>(const float* t, size_t i) {
    return *reinterpret_cast<const float2*>(t + 2 * i);
}
template <>
__device__ __forceinline__ float2 table_pair<__half>(const __half* t, size_t i) {
    return __half22float2(__ldg(reinterpret_cast<const __half2*>(t + 2 * i)));
}

// Hash features of one level.
template <class T>
__device__ __forceinline__ float2 hash_level(const HashGrid& g, const T* table, int level, const float p01[3]) {
    HashCell c;
    hash_cell(g, level, p01, &c);
    const size_t base = size_t(level) << g.log2_table;
    float2 acc = make_float2(0, 0);
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const float2 v = table_pair(table, base + c.slot[k]);
        acc.x += c.w[k] * v.x;
        acc.y += c.w[k] * v.y;
    }
    return acc;
}

__device__ __forceinline__ uint32_t pack_bf16x2(float a, float b) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<const uint32_t*>(&h);
}

// Write 8 consecutive values of row `row` (k0 a multiple of 8) of a K-major
// operand with K columns.
__device__ __forceinline__ void store_row8(uint8_t* buf, int K, int row, int k0, const float* v) {
    uint4 q;
    q.x = pack_bf16x2(v[0], v[1]);
    q.y = pack_bf16x2(v[2], v[3]);
    q.z = pack_bf16x2(v[4], v[5]);
    q.w = pack_bf16x2(v[6], v[7]);
    *reinterpret_cast<uint4*>(buf + tc::kmajor_offset(K, row, k0)) = q;
}
__device__ __forceinline__ void store_one(uint8_t* buf, int K, int row, int k, float v) {
    *reinterpret_cast<__nv_bfloat16*>(buf + tc::kmajor_offset(K, row, k)) = __float2bfloat16_rn(v);
}

// The 112 input features of query q as row `row` of X (K = 112) and, when
// xt != null, as column `row` of X^T (112 rows, K = 128).
template <class T>
__device__ __forceinline__ void write_inputs(const HashGrid& g, const T* table, const GuideQuery& q, int row, uint8_t* x,
                             uint8_t* xt) {
    float p01[3];
    normalise_pos(g, q.pos, p01);
    float v[16];
#pragma unroll
    for (int l = 0; l < kHashLevels; l += 4) {
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const float2 f = hash_level(g, table, l + j, p01);
            v[2 * j] = f.x;
            v[2 * j + 1] = f.y;
        }
        store_row8(x, kGuideIn, row, 2 * l, v);
        if (xt) for (int j = 0; j < 8; ++j) store_one(xt, kGuideTile, 2 * l + j, row, v[j]);
    }
    float d[80];
    guide_dense_features(q, d);
    for (int k = 0; k < 80; k += 8) {
        store_row8(x, kGuideIn, row, kHashIn + k, d + k);
        if (xt) for (int j = 0; j < 8; ++j) store_one(xt, kGuideTile, kHashIn + k + j, row, d[k + j]);
    }
}

}  // namespace dev
}  // namespace atrc
