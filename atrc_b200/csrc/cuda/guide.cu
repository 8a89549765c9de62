// Learned path guiding on sm_100a: a hash-grid-encoded MLP whose output is a
// von Mises-Fisher mixture (dev_guide.cuh), evaluated and trained with
// hand-written tcgen05 kernels (BF16 operands in shared memory, FP32
// accumulators in tensor memory) and updated with Adam.
//
// Network: 112 inputs -> 64 -> 64 -> 64 -> 48 outputs, ReLU between layers,
// no biases.  Weights are kept as FP32 masters (Adam state beside them) and
// copied to BF16 for the tensor cores; the hash table (levels x 2^log2 x 2
// features) is kept as FP32 master and FP16 copy.
//
// Kernels:
//  - k_guide_encode (and the wavefront's feature kernel) encode queries into
//    128-row input tiles in global memory, in the operand layout;
//  - k_guide_mlp: one CTA of 128 threads per tile (persistent over tiles)
//    copies a tile to shared memory; thread t owns row t and TMEM lane t.
//    The four layers run as four MMA groups on the same 64 TMEM columns.
//  - k_guide_train: forward as above, keeping activations and their
//    transposes in shared memory, then the loss gradient of every record
//    (thread-local), the backward pass (dA = dZ W on the tensor core) and the
//    weight gradients dW^T += A^T dZ accumulated in TMEM across all tiles of
//    the CTA; hash-table gradients are scattered with FP32 atomics.
//  - k_guide_adam: Adam over every parameter, refreshing the BF16 / FP16
//    copies.
// The reference has no learned guiding: `pt` samples the BSDF only
// (path_tracing.cpp:150-169).
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <memory>
#include <random>
#include <string>
#include <type_traits>
#include <vector>

#include "../../../include/atrc_cuda.h"
#include "cuda_util.h"
#include "dev_guide.cuh"
#include "dev_guide_enc.cuh"
#include "dev_tc.cuh"
#include "guide.h"

namespace atrc {

using namespace dev;

namespace {

// packed MLP weights, row-major [out][in] per layer
constexpr int kOffW1 = 0;
constexpr int kOffW2 = kOffW1 + kGuideHidden * kGuideIn;
constexpr int kOffW3 = kOffW2 + kGuideHidden * kGuideHidden;
constexpr int kOffW4 = kOffW3 + kGuideHidden * kGuideHidden;
constexpr int kWeights = kOffW4 + kGuideOut * kGuideHidden;  // 18,432
constexpr int kTile = kGuideTile;

struct NetView {
    const __nv_bfloat16* w;   // BF16 weights
    const __half* table_h;    // FP16 table (inference)
    const float* table_f;     // FP32 table (training)
    HashGrid grid;
    float max_select;         // cap on the selection probability
};

// Copy W (rows x cols, row-major, BF16 in global) into a K-major operand in
// shared memory: as is (operand rows = out, K = in) or transposed (rows = in,
// K = out), taking only rows [0, take) of the result.
__device__ void load_weights(uint8_t* dst, const __nv_bfloat16* w, int out, int in, bool transpose, int take) {
    const int rows = transpose ? in : out, K = transpose ? out : in;
    const int n = min(rows, take) * K;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const int r = i / K, k = i % K;
        const __nv_bfloat16 v = transpose ? w[size_t(k) * in + r] : w[size_t(r) * in + k];
        *reinterpret_cast<__nv_bfloat16*>(dst + tc::kmajor_offset(K, r, k)) = v;
    }
}

// Load this warp's 32 lanes x `n` (multiple of 16) columns from TMEM.
__device__ __forceinline__ void tmem_row(uint32_t tbase, int col0, int n, float* v) {
    const int lane0 = (threadIdx.x >> 5) * 32;
    for (int c = 0; c < n; c += 16) tc::tmem_ld16(tc::tmem_at(tbase, lane0, col0 + c), v + c);
}

// ------------------------------------------------------------ inference
// shared memory of k_guide_mlp (bytes): two input buffers (each holds an
// encoded tile, then H2, then the tile's outputs), H1 / H3, the weights and
// the barriers (MMA completion, one per input buffer)
constexpr int kInfX = 0;                                  // X[0], X[1]: 128 x 112 each
constexpr int kInfH = kInfX + 2 * kGuideTileBytes;        // H1 / H3 128 x 64
constexpr int kInfW1 = kInfH + kTile * kGuideHidden * 2;
constexpr int kInfW2 = kInfW1 + kGuideHidden * kGuideIn * 2;
constexpr int kInfW3 = kInfW2 + kGuideHidden * kGuideHidden * 2;
constexpr int kInfW4 = kInfW3 + kGuideHidden * kGuideHidden * 2;
constexpr int kInfBar = kInfW4 + kGuideOut * kGuideHidden * 2;
constexpr int kInfSmem = kInfBar + 64;
constexpr uint32_t kInfTmemCols = 64;
static_assert(kGuideTileBytes == kTile * kGuideIn * 2 && kGuideTileBytes % 16 == 0, "an encoded tile fills X");
static_assert(kTile * kGuideOut * 4 <= kGuideTileBytes, "a tile's outputs fit its input buffer");
static_assert(2 * (kInfSmem + 1024) <= 228 * 1024, "two CTAs per SM");

// One MMA group: thread 0 issues, all wait.  Returns false (uniformly) when
// the wait gave up.
__device__ __forceinline__ bool run_mma(uint64_t* bar, uint32_t* phase, int* err, uint32_t tmem_d, uint32_t a,
                                        uint32_t b, int k, int n, bool acc) {
    tc::fence_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    if (threadIdx.x == 0) {
        tc::fence_after_sync();
        tc::mma_tile(tmem_d, a, b, k, n, acc);
        tc::mma_commit(bar);
    }
    const bool ok = tc::mbar_wait(bar, *phase, err);
    *phase ^= 1u;
    tc::fence_after_sync();
    return __syncthreads_and(ok) != 0;
}

// ReLU of this thread's 64 accumulator columns into row t of dst (K = 64),
// 16 columns at a time.
__device__ __forceinline__ void relu_row(uint32_t tmem, uint8_t* dst, int t) {
    const int lane0 = (threadIdx.x >> 5) * 32;
    for (int c = 0; c < kGuideHidden; c += 16) {
        float v[16];
        tc::tmem_ld16(tc::tmem_at(tmem, lane0, c), v);
        for (int j = 0; j < 16; ++j) v[j] = fmaxf(v[j], 0.0f);
        store_row8(dst, kGuideHidden, t, c, v);
        store_row8(dst, kGuideHidden, t, c + 8, v + 8);
    }
}

// Encode queries into 128-row input tiles (one thread per query).
template <class T>
__global__ void k_guide_encode(HashGrid grid, const T* __restrict__ table, const GuideQuery* __restrict__ q, int n,
                               uint8_t* __restrict__ xtiles) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        write_inputs<T>(grid, table, q[i], i % kTile, xtiles + size_t(i / kTile) * kGuideTileBytes, nullptr);
}

// The MLP over encoded tiles: *n_dev rows.  DECODE writes the decoded
// mixture (GuideMix order, kGuideOut floats per row), else the raw outputs.
// Persistent CTAs of 128 threads, two per SM; thread t owns row t and TMEM
// lane t, and the four layers run on the same 64 TMEM columns.  While a
// tile runs through the tensor core, the CTA's next tile streams into the
// other input buffer (one bulk copy, completion counted on that buffer's
// mbarrier); the finished tile's outputs are staged in its input buffer and
// leave in coalesced 16-byte stores.
template <bool DECODE>
__global__ void __launch_bounds__(kTile, 2) k_guide_mlp(NetView net, const uint8_t* __restrict__ xtiles,
                                                       const int* __restrict__ n_dev, float* __restrict__ out,
                                                       int* err) {
    extern __shared__ __align__(1024) uint8_t smem[];
    uint8_t* H = smem + kInfH;
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + kInfBar);       // MMA completion
    uint64_t* bar_in = reinterpret_cast<uint64_t*>(smem + kInfBar + 8);  // [2] input copies
    uint32_t* tslot = reinterpret_cast<uint32_t*>(smem + kInfBar + 24);
    const int n = *n_dev;
    const int ntiles = (n + kTile - 1) / kTile;
    if (int(blockIdx.x) >= ntiles) return;  // uniform per CTA, before any TMEM use
    const int t = threadIdx.x;
    if (t == 0) {
        tc::mbar_init(bar, 1);
        tc::mbar_init(bar_in, 1);
        tc::mbar_init(bar_in + 1, 1);
        // the first tile starts streaming before the weights are staged
        tc::mbar_arrive_expect_tx(bar_in, kGuideTileBytes);
        tc::bulk_g2s(smem + kInfX, xtiles + size_t(blockIdx.x) * kGuideTileBytes, kGuideTileBytes, bar_in);
    }
    load_weights(smem + kInfW1, net.w + kOffW1, kGuideHidden, kGuideIn, false, kGuideHidden);
    load_weights(smem + kInfW2, net.w + kOffW2, kGuideHidden, kGuideHidden, false, kGuideHidden);
    load_weights(smem + kInfW3, net.w + kOffW3, kGuideHidden, kGuideHidden, false, kGuideHidden);
    load_weights(smem + kInfW4, net.w + kOffW4, kGuideOut, kGuideHidden, false, kGuideOut);
    if (t < 32) tc::tmem_alloc(tslot, kInfTmemCols);
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = *tslot;
    const uint32_t sH = tc::smem_addr(H);
    uint32_t phase = 0, phase_in[2] = {0, 0};
    bool pending[2] = {true, false};  // a copy into the buffer not waited for yet
    int it = 0;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++it) {
        const int buf = it & 1;
        uint8_t* X = smem + kInfX + buf * kGuideTileBytes;
        const uint32_t sX = tc::smem_addr(X);
        // the next tile into the other buffer (its last use, the previous
        // tile's output staging, ended at the barrier closing that tile)
        const int next = tile + int(gridDim.x);
        if (next < ntiles) {
            if (t == 0) {
                uint8_t* Xn = smem + kInfX + (buf ^ 1) * kGuideTileBytes;
                tc::fence_async_smem();
                tc::mbar_arrive_expect_tx(bar_in + (buf ^ 1), kGuideTileBytes);
                tc::bulk_g2s(Xn, xtiles + size_t(next) * kGuideTileBytes, kGuideTileBytes, bar_in + (buf ^ 1));
            }
            pending[buf ^ 1] = true;
        }
        // this tile's inputs (rows past n hold stale values; every output row
        // depends on its own input row only, and is not written)
        const bool ok = tc::mbar_wait(bar_in + buf, phase_in[buf], err);
        if (!__syncthreads_and(ok)) break;
        phase_in[buf] ^= 1u;
        pending[buf] = false;
        if (!run_mma(bar, &phase, err, tmem, sX, tc::smem_addr(smem + kInfW1), kGuideIn, kGuideHidden, false)) break;
        relu_row(tmem, H, t);
        if (!run_mma(bar, &phase, err, tmem, sH, tc::smem_addr(smem + kInfW2), kGuideHidden, kGuideHidden, false)) break;
        relu_row(tmem, X, t);
        if (!run_mma(bar, &phase, err, tmem, sX, tc::smem_addr(smem + kInfW3), kGuideHidden, kGuideHidden, false)) break;
        relu_row(tmem, H, t);
        if (!run_mma(bar, &phase, err, tmem, sH, tc::smem_addr(smem + kInfW4), kGuideHidden, kGuideOut, false)) break;
        float v[kGuideOut];
        tmem_row(tmem, 0, kGuideOut, v);
        // stage row t (H2 in X was read by the layer-3 MMA, complete now)
        float* o = reinterpret_cast<float*>(X) + t * kGuideOut;
        if (DECODE) {
            GuideMix m;
            guide_decode(v, &m, net.max_select);
            for (int k = 0; k < kGuideLobes; ++k) {
                o[5 * k] = m.mu[k][0];
                o[5 * k + 1] = m.mu[k][1];
                o[5 * k + 2] = m.mu[k][2];
                o[5 * k + 3] = m.kappa[k];
                o[5 * k + 4] = m.w[k];
            }
            o[kGuideUsed - 1] = m.c;
            for (int k = kGuideUsed; k < kGuideOut; ++k) o[k] = 0.0f;
        } else {
            for (int k = 0; k < kGuideOut; ++k) o[k] = v[k];
        }
        __syncthreads();
        // the tile's valid rows leave as one contiguous block
        const int rows = min(kTile, n - tile * kTile);
        const uint4* src = reinterpret_cast<const uint4*>(X);
        uint4* dst = reinterpret_cast<uint4*>(out + size_t(tile) * kTile * kGuideOut);
        for (int k = t; k < rows * kGuideOut / 4; k += kTile) dst[k] = src[k];
        __syncthreads();
    }
    // copies still in flight (the loop left early) land before the CTA
    // exits; these waits are bounded like the others
    if (t == 0)
        for (int b = 0; b < 2; ++b)
            if (pending[b]) tc::mbar_wait(bar_in + b, phase_in[b], err, 1u << 16);
    tc::fence_before_sync();
    __syncthreads();
    if (t < 32) tc::tmem_dealloc(tmem, kInfTmemCols);
}

// ------------------------------------------------------------- training
// shared memory of k_guide_train (bytes); row groups outermost everywhere,
// so the M = 128 reads of the 112- and 64-row transposes run into the next
// buffer (their extra TMEM lanes are ignored)
constexpr int kTrW1 = 0;                                          // W1 64 x 112
constexpr int kTrW2 = kTrW1 + kGuideHidden * kGuideIn * 2;        // W2 64 x 64
constexpr int kTrW3 = kTrW2 + kGuideHidden * kGuideHidden * 2;    // W3 64 x 64
constexpr int kTrW4 = kTrW3 + kGuideHidden * kGuideHidden * 2;    // W4 48 x 64
constexpr int kTrB1 = kTrW4 + kGuideOut * kGuideHidden * 2;       // W1^T rows 0..31: 32 x 64
constexpr int kTrB2 = kTrB1 + kHashIn * kGuideHidden * 2;         // W2^T 64 x 64
constexpr int kTrB3 = kTrB2 + kGuideHidden * kGuideHidden * 2;    // W3^T 64 x 64
constexpr int kTrB4 = kTrB3 + kGuideHidden * kGuideHidden * 2;    // W4^T 64 x 48
constexpr int kTrP0 = kTrB4 + kGuideHidden * kGuideOut * 2;       // X 128 x 112 / H2 128 x 64
constexpr int kTrP1 = kTrP0 + kTile * kGuideIn * 2;               // H1 / H3 128 x 64
constexpr int kTrXT = kTrP1 + kTile * kGuideHidden * 2;           // X^T 112 x 128
constexpr int kTrHT1 = kTrXT + kGuideIn * kTile * 2;              // H1^T 64 x 128
constexpr int kTrHT2 = kTrHT1 + kGuideHidden * kTile * 2;
constexpr int kTrHT3 = kTrHT2 + kGuideHidden * kTile * 2;
constexpr int kTrDZ = kTrHT3 + kGuideHidden * kTile * 2;          // dZ 128 x 64 (48)
constexpr int kTrDZT = kTrDZ + kTile * kGuideHidden * 2;          // dZ^T 64 (48) x 128
constexpr int kTrBar = kTrDZT + kGuideHidden * kTile * 2;
constexpr int kTrSmem = kTrBar + 64;
static_assert(kTrSmem <= 227 * 1024, "training kernel shared memory");
// the padded reads stay inside the allocation
static_assert(kTrXT + (kTile / 8) * (kTile / 8) * 128 <= kTrSmem, "X^T overread");
static_assert(kTrHT3 + (kTile / 8) * (kTile / 8) * 128 <= kTrSmem, "H3^T overread");
// TMEM columns
constexpr int kColF = 0, kColB = 64, kColW1 = 128, kColW2 = 192, kColW3 = 256, kColW4 = 320;
constexpr uint32_t kTrTmemCols = 512;

struct TrainArgs {
    const GuideRecord* rec;
    int n;                     // records in this batch
    const float* weight_sum;   // sum of the batch's targets (device)
    float* grad_w;             // FP32 gradients of the packed weights
    float* grad_table;         // FP32 gradients of the table
    float* loss;               // sum of the batch's loss terms
    float target_clamp;        // > 0: record targets capped at this multiple of the batch mean
};

// Gradient of loss = -w log(c g + (1 - c) b) with respect to the raw outputs.
__device__ void loss_grad(const float* o, const GuideRecord& r, float w, float max_select, float* d, float* loss) {
    for (int k = 0; k < kGuideOut; ++k) d[k] = 0.0f;
    *loss = 0.0f;
    if (!(w > 0.0f)) return;
    GuideMix m;
    guide_decode(o, &m, max_select);
    const Vec3 wi(r.wi[0], r.wi[1], r.wi[2]);
    float v[kGuideLobes], dots[kGuideLobes];
    float g = 0.0f;
    for (int k = 0; k < kGuideLobes; ++k) {
        dots[k] = m.mu[k][0] * wi.x + m.mu[k][1] * wi.y + m.mu[k][2] * wi.z;
        v[k] = vmf_norm(m.kappa[k]) * __expf(m.kappa[k] * (dots[k] - 1.0f));
        g += m.w[k] * v[k];
    }
    const float b = r.pdf_bsdf;
    const float q = m.c * g + (1.0f - m.c) * b;
    if (!(q > 1e-20f)) return;
    *loss = -w * logf(q);
    const float dq = -w / q;
    // selection: c = cmax sigmoid(s), dc/ds = c (1 - sigmoid(s))
    const float sg = m.c / max_select;
    d[5 * kGuideLobes] = dq * (g - b) * m.c * (1.0f - sg);
    const float dg = dq * m.c;
    for (int k = 0; k < kGuideLobes; ++k) {
        const float wv = m.w[k] * v[k];
        // mixture logit (softmax)
        d[5 * k + 4] = dg * m.w[k] * (v[k] - g);
        // log kappa (zero where clamped)
        const float lk = o[5 * k + 3];
        if (lk > kLogKappaMin && lk < kLogKappaMax) {
            const float kap = m.kappa[k];
            const float corr = kap < 1e-3f ? 1.0f : 2.0f * kap / expm1f(2.0f * kap);
            d[5 * k + 3] = dg * wv * (1.0f - corr + kap * (dots[k] - 1.0f));
        }
        // mean direction through the normalisation
        const float x = o[5 * k], y = o[5 * k + 1], z = o[5 * k + 2];
        const float len = sqrtf(x * x + y * y + z * z);
        if (len > 1e-10f) {
            const float s = dg * wv * m.kappa[k] / len;
            d[5 * k] = s * (wi.x - dots[k] * m.mu[k][0]);
            d[5 * k + 1] = s * (wi.y - dots[k] * m.mu[k][1]);
            d[5 * k + 2] = s * (wi.z - dots[k] * m.mu[k][2]);
        }
    }
}

// ReLU layer output into a row of P (K = 64) and a column of HT; returns the mask.
__device__ __forceinline__ uint64_t relu_store(const float* v, uint8_t* P, uint8_t* HT, int t) {
    uint64_t mask = 0;
    for (int k = 0; k < kGuideHidden; k += 8) {
        float r[8];
        for (int j = 0; j < 8; ++j) {
            r[j] = fmaxf(v[k + j], 0.0f);
            if (v[k + j] > 0.0f) mask |= uint64_t(1) << (k + j);
        }
        store_row8(P, kGuideHidden, t, k, r);
        for (int j = 0; j < 8; ++j) store_one(HT, kTile, k + j, t, r[j]);
    }
    return mask;
}

// Gradient row of width n into DZ (row t, K = n) and DZT (column t, n rows).
__device__ __forceinline__ void dz_store(const float* d, int n, uint8_t* DZ, uint8_t* DZT, int t) {
    for (int k = 0; k < n; k += 8) {
        store_row8(DZ, n, t, k, d + k);
        for (int j = 0; j < 8; ++j) store_one(DZT, kTile, k + j, t, d[k + j]);
    }
}

__global__ void __launch_bounds__(kTile, 1) k_guide_train(NetView net, TrainArgs a, int* err) {
    extern __shared__ __align__(1024) uint8_t smem[];
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + kTrBar);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(smem + kTrBar + 8);
    const int ntiles = (a.n + kTile - 1) / kTile;
    if (int(blockIdx.x) >= ntiles) return;
    load_weights(smem + kTrW1, net.w + kOffW1, kGuideHidden, kGuideIn, false, kGuideHidden);
    load_weights(smem + kTrW2, net.w + kOffW2, kGuideHidden, kGuideHidden, false, kGuideHidden);
    load_weights(smem + kTrW3, net.w + kOffW3, kGuideHidden, kGuideHidden, false, kGuideHidden);
    load_weights(smem + kTrW4, net.w + kOffW4, kGuideOut, kGuideHidden, false, kGuideOut);
    load_weights(smem + kTrB1, net.w + kOffW1, kGuideHidden, kGuideIn, true, kHashIn);
    load_weights(smem + kTrB2, net.w + kOffW2, kGuideHidden, kGuideHidden, true, kGuideHidden);
    load_weights(smem + kTrB3, net.w + kOffW3, kGuideHidden, kGuideHidden, true, kGuideHidden);
    load_weights(smem + kTrB4, net.w + kOffW4, kGuideOut, kGuideHidden, true, kGuideHidden);
    if (threadIdx.x == 0) tc::mbar_init(bar, 1);
    if (threadIdx.x < 32) tc::tmem_alloc(tslot, kTrTmemCols);
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tm = *tslot;
    auto S = [&](int off) { return tc::smem_addr(smem + off); };
    const float inv_wsum = *a.weight_sum > 0 ? 1.0f / *a.weight_sum : 0.0f;
    // a few records of a batch can carry most of its weight (a path that found
    // the light): capping the targets keeps one step from following them alone
    const float tcap = a.target_clamp > 0.0f ? a.target_clamp * *a.weight_sum / float(max(a.n, 1)) : INFINITY;
    uint32_t phase = 0;
    const int t = threadIdx.x;
    bool first = true, ok = true;
    float loss_acc = 0.0f;
    for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
        const int i = tile * kTile + t;
        GuideRecord r;
        if (i < a.n) r = a.rec[i];
        else memset(&r, 0, sizeof(r));
        GuideQuery q;
        for (int j = 0; j < 3; ++j) { q.pos[j] = r.pos[j]; q.nrm[j] = r.nrm[j]; q.wo[j] = r.wo[j]; }
        q.rough = r.rough;
        q.slot = 0;
        const float w = i < a.n ? fminf(r.target, tcap) * inv_wsum : 0.0f;
        // ---- forward
        write_inputs<float>(net.grid, net.table_f, q, t, smem + kTrP0, smem + kTrXT);
        float v[kGuideHidden];
        if (!(ok = run_mma(bar, &phase, err, tm + kColF, S(kTrP0), S(kTrW1), kGuideIn, kGuideHidden, false))) break;
        tmem_row(tm, kColF, kGuideHidden, v);
        const uint64_t m1 = relu_store(v, smem + kTrP1, smem + kTrHT1, t);
        if (!(ok = run_mma(bar, &phase, err, tm + kColF, S(kTrP1), S(kTrW2), kGuideHidden, kGuideHidden, false))) break;
        tmem_row(tm, kColF, kGuideHidden, v);
        const uint64_t m2 = relu_store(v, smem + kTrP0, smem + kTrHT2, t);
        if (!(ok = run_mma(bar, &phase, err, tm + kColF, S(kTrP0), S(kTrW3), kGuideHidden, kGuideHidden, false))) break;
        tmem_row(tm, kColF, kGuideHidden, v);
        const uint64_t m3 = relu_store(v, smem + kTrP1, smem + kTrHT3, t);
        if (!(ok = run_mma(bar, &phase, err, tm + kColF, S(kTrP1), S(kTrW4), kGuideHidden, kGuideOut, false))) break;
        tmem_row(tm, kColF, kGuideOut, v);
        // ---- loss gradient of this thread's record
        float d[kGuideHidden];
        float lo;
        loss_grad(v, r, w, net.max_select, d, &lo);
        loss_acc += lo;
        dz_store(d, kGuideOut, smem + kTrDZ, smem + kTrDZT, t);
        // ---- backward: dA3 = dZ4 W4, dW4^T += H3^T dZ4
        tc::fence_async_smem();
        tc::fence_before_sync();
        __syncthreads();
        if (t == 0) {
            tc::fence_after_sync();
            tc::mma_tile(tm + kColB, S(kTrDZ), S(kTrB4), kGuideOut, kGuideHidden, false);
            tc::mma_tile(tm + kColW4, S(kTrHT3), S(kTrDZT), kTile, kGuideOut, !first);
            tc::mma_commit(bar);
        }
        ok = tc::mbar_wait(bar, phase, err);
        phase ^= 1u;
        tc::fence_after_sync();
        if (!(ok = __syncthreads_and(ok) != 0)) break;
        // layers 3 and 2
        const uint64_t masks[2] = {m3, m2};
        const int bw[2] = {kTrB3, kTrB2}, ht[2] = {kTrHT2, kTrHT1}, cw[2] = {kColW3, kColW2};
        for (int L = 0; L < 2 && ok; ++L) {
            tmem_row(tm, kColB, kGuideHidden, v);
            for (int k = 0; k < kGuideHidden; ++k) d[k] = (masks[L] >> k) & 1 ? v[k] : 0.0f;
            dz_store(d, kGuideHidden, smem + kTrDZ, smem + kTrDZT, t);
            tc::fence_async_smem();
            tc::fence_before_sync();
            __syncthreads();
            if (t == 0) {
                tc::fence_after_sync();
                tc::mma_tile(tm + kColB, S(kTrDZ), S(bw[L]), kGuideHidden, kGuideHidden, false);
                tc::mma_tile(tm + cw[L], S(ht[L]), S(kTrDZT), kTile, kGuideHidden, !first);
                tc::mma_commit(bar);
            }
            ok = tc::mbar_wait(bar, phase, err);
            phase ^= 1u;
            tc::fence_after_sync();
            ok = __syncthreads_and(ok) != 0;
        }
        if (!ok) break;
        // layer 1: dX[:, 0:32] = dZ1 W1[:, 0:32], dW1^T += X^T dZ1
        tmem_row(tm, kColB, kGuideHidden, v);
        for (int k = 0; k < kGuideHidden; ++k) d[k] = (m1 >> k) & 1 ? v[k] : 0.0f;
        dz_store(d, kGuideHidden, smem + kTrDZ, smem + kTrDZT, t);
        tc::fence_async_smem();
        tc::fence_before_sync();
        __syncthreads();
        if (t == 0) {
            tc::fence_after_sync();
            tc::mma_tile(tm + kColB, S(kTrDZ), S(kTrB1), kGuideHidden, kHashIn, false);
            tc::mma_tile(tm + kColW1, S(kTrXT), S(kTrDZT), kTile, kGuideHidden, !first);
            tc::mma_commit(bar);
        }
        ok = tc::mbar_wait(bar, phase, err);
        phase ^= 1u;
        tc::fence_after_sync();
        if (!(ok = __syncthreads_and(ok) != 0)) break;
        // hash-table gradients
        tmem_row(tm, kColB, kHashIn, v);
        if (i < a.n && w > 0.0f) {
            float p01[3];
            normalise_pos(net.grid, q.pos, p01);
            for (int l = 0; l < kHashLevels; ++l) {
                HashCell c;
                hash_cell(net.grid, l, p01, &c);
                const size_t base = size_t(l) << net.grid.log2_table;
                for (int k = 0; k < 8; ++k) {
                    float* gp = a.grad_table + 2 * (base + c.slot[k]);
                    atomicAdd(reinterpret_cast<float2*>(gp), make_float2(c.w[k] * v[2 * l], c.w[k] * v[2 * l + 1]));
                }
            }
        }
        first = false;
    }
    // ---- weight gradients out of TMEM (lane = input feature)
    if (ok && !first) {
        tc::fence_before_sync();
        __syncthreads();
        tc::fence_after_sync();
        float v[kGuideHidden];
        tmem_row(tm, kColW1, kGuideHidden, v);
        if (t < kGuideIn) for (int o = 0; o < kGuideHidden; ++o) atomicAdd(a.grad_w + kOffW1 + o * kGuideIn + t, v[o]);
        tmem_row(tm, kColW2, kGuideHidden, v);
        if (t < kGuideHidden) for (int o = 0; o < kGuideHidden; ++o) atomicAdd(a.grad_w + kOffW2 + o * kGuideHidden + t, v[o]);
        tmem_row(tm, kColW3, kGuideHidden, v);
        if (t < kGuideHidden) for (int o = 0; o < kGuideHidden; ++o) atomicAdd(a.grad_w + kOffW3 + o * kGuideHidden + t, v[o]);
        tmem_row(tm, kColW4, kGuideOut, v);
        if (t < kGuideHidden) for (int o = 0; o < kGuideOut; ++o) atomicAdd(a.grad_w + kOffW4 + o * kGuideHidden + t, v[o]);
    }
    for (int o = 16; o > 0; o >>= 1) loss_acc += __shfl_down_sync(0xffffffffu, loss_acc, o);
    if ((t & 31) == 0) atomicAdd(a.loss, loss_acc);
    tc::fence_before_sync();
    __syncthreads();
    if (threadIdx.x < 32) tc::tmem_dealloc(tm, kTrTmemCols);
}

// Mixture pdf of directions from decoded mixtures (tests and tools).
__global__ void k_mix_pdf(const float* __restrict__ mixes, const float* __restrict__ dirs, int n, float* __restrict__ pdf,
                          float* __restrict__ select) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float* gm = mixes + size_t(i) * kGuideOut;
        GuideMix m;
        for (int k = 0; k < kGuideLobes; ++k) {
            m.mu[k][0] = gm[5 * k]; m.mu[k][1] = gm[5 * k + 1]; m.mu[k][2] = gm[5 * k + 2];
            m.kappa[k] = gm[5 * k + 3];
            m.w[k] = gm[5 * k + 4];
        }
        m.c = gm[kGuideUsed - 1];
        pdf[i] = guide_pdf(m, Vec3(dirs[3 * i], dirs[3 * i + 1], dirs[3 * i + 2]));
        select[i] = m.c;
    }
}

__global__ void k_target_sum(const GuideRecord* rec, int n, float* sum) {
    float s = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) s += rec[i].target;
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(sum, s);
}

// The records of a pass whose target is positive, compacted into `out`: a
// zero-target record adds nothing to the loss or to its gradient, so the
// training batches carry only records that do (order not kept).
__global__ void k_live_records(const GuideRecord* __restrict__ rec, int n, GuideRecord* __restrict__ out,
                               int* count) {
    const int lane = threadIdx.x & 31;
    for (int i0 = blockIdx.x * blockDim.x; i0 < n; i0 += gridDim.x * blockDim.x) {
        const int i = i0 + threadIdx.x;
        const bool live = i < n && rec[i].target > 0.0f;
        const unsigned m = __ballot_sync(0xffffffffu, live);
        int base = 0;
        if (lane == 0 && m) base = atomicAdd(count, __popc(m));
        base = __shfl_sync(0xffffffffu, base, 0);
        if (live) out[base + __popc(m & ((1u << lane) - 1u))] = rec[i];
    }
}

struct AdamArgs {
    float lr, b1, b2, eps, c1, c2;  // c1 = 1 / (1 - b1^t), c2 = 1 / (1 - b2^t)
};

template <class Copy>
__global__ void k_guide_adam(float* __restrict__ p, float* __restrict__ g, float* __restrict__ m,
                             float* __restrict__ v, Copy* __restrict__ copy, size_t n, AdamArgs a) {
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) {
        const float gi = g[i];
        const float mi = a.b1 * m[i] + (1.0f - a.b1) * gi;
        const float vi = a.b2 * v[i] + (1.0f - a.b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float pi = p[i] - a.lr * (mi * a.c1) / (sqrtf(vi * a.c2) + a.eps);
        p[i] = pi;
        g[i] = 0.0f;
        if constexpr (std::is_same<Copy, __half>::value) copy[i] = __float2half_rn(pi);
        else copy[i] = __float2bfloat16_rn(pi);
    }
}

template <class Copy>
__global__ void k_copy_params(const float* __restrict__ p, Copy* __restrict__ copy, size_t n) {
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) {
        if constexpr (std::is_same<Copy, __half>::value) copy[i] = __float2half_rn(p[i]);
        else copy[i] = __float2bfloat16_rn(p[i]);
    }
}

}  // namespace

// ====================================================================== guide
struct GuideImpl {
    int device = 0;
    int sm_count = 148;
    cudaStream_t stream = nullptr;
    AtrcGuideDesc desc{};
    HashGrid grid{};
    size_t table_n = 0;  // floats in the table
    DevBuf w_f, w_g, w_m, w_v, w_bf;          // weights: master, grad, Adam m / v, BF16 copy
    DevBuf t_f, t_g, t_m, t_v, t_h;           // table: master, grad, m, v, FP16 copy
    DevBuf records, rec_count, rec_last, queries, mixes, gidx, xtiles, scratch, err;
    DevBuf live;          // the records of a pass with a non-zero target, compacted for training
    size_t slots = 0;
    int steps = 0;
    float record_keep = 1.0f;  // recording probability of the next pass (from the last one's vertex count)
    NetView view() const {
        NetView v;
        v.w = w_bf.as<__nv_bfloat16>();
        v.table_h = t_h.as<__half>();
        v.table_f = t_f.as<float>();
        v.grid = grid;
        v.max_select = desc.max_select;
        return v;
    }
    ~GuideImpl() {
        if (stream) cudaStreamDestroy(stream);
    }
};

GuideFrame guide_frame(GuideImpl* g, size_t cap, bool record, cudaStream_t s) {
    if (g->slots < cap) {
        g->queries.alloc(cap * sizeof(GuideQuery));
        g->mixes.alloc(cap * kGuideOut * sizeof(float));
        g->rec_last.alloc(cap * sizeof(int));
        g->gidx.alloc(cap * sizeof(int));
        g->xtiles.alloc((cap + kTile - 1) / kTile * kGuideTileBytes);
        g->slots = cap;
    }
    GuideFrame f{};
    f.queries = g->queries.as<GuideQuery>();
    f.mixes = g->mixes.as<float>();
    f.gidx = g->gidx.as<int>();
    f.max_depth = g->desc.max_depth;
    f.xtiles = g->xtiles.as<uint8_t>();
    f.table_h = g->t_h.as<__half>();
    f.grid = g->grid;
    if (record) {
        CK(cudaMemsetAsync(g->rec_count.p, 0, 2 * sizeof(int), s));
        CK(cudaMemsetAsync(g->rec_last.p, 0xff, cap * sizeof(int), s));
        f.records = g->records.as<GuideRecord>();
        f.record_count = g->rec_count.as<int>();
        f.record_cap = int(g->desc.record_capacity);
        f.record_keep = g->record_keep;
        f.record_last = g->rec_last.as<int>();
    }
    return f;
}

void guide_infer(GuideImpl* g, const int* n_dev, cudaStream_t s) {
    k_guide_mlp<true><<<g->sm_count * 2, kTile, kInfSmem, s>>>(g->view(), g->xtiles.as<uint8_t>(), n_dev,
                                                              g->mixes.as<float>(), g->err.as<int>());
}

int guide_device(const GuideImpl* g) { return g->device; }

}  // namespace atrc

// ====================================================================== C ABI
using namespace atrc;

struct AtrcGuide {
    GuideImpl impl;
};

namespace atrc {
GuideImpl* guide_impl(AtrcGuide* g) { return &g->impl; }
}  // namespace atrc

namespace {

int gfail(int code, const std::string& msg) {
    set_last_error(msg);
    return code;
}

template <class F>
int gguarded(F&& f) {
    try {
        return f();
    } catch (const CudaError& e) {
        return gfail(ATRC_ERR_CUDA, e.what());
    } catch (const std::bad_alloc&) {
        return gfail(ATRC_ERR_OUT_OF_MEMORY, "host allocation failed");
    } catch (const std::exception& e) {
        return gfail(ATRC_ERR_UNSUPPORTED, e.what());
    }
}

void check_err(GuideImpl& g, const char* what) {
    int e = 0;
    CK(cudaMemcpyAsync(&e, g.err.p, sizeof(int), cudaMemcpyDeviceToHost, g.stream));
    CK(cudaStreamSynchronize(g.stream));
    if (e) {
        CK(cudaMemsetAsync(g.err.p, 0, sizeof(int), g.stream));
        throw CudaError(std::string(what) + ": a tensor-core completion wait reached its limit");
    }
}

// dynamic shared memory above 48 KB (set on the current device)
void set_smem_limits() {
    CK(cudaFuncSetAttribute(k_guide_mlp<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kInfSmem));
    CK(cudaFuncSetAttribute(k_guide_mlp<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, kInfSmem));
    CK(cudaFuncSetAttribute(k_guide_train, cudaFuncAttributeMaxDynamicSharedMemorySize, kTrSmem));
}

}  // namespace

extern "C" {

int atrc_guide_default_desc(AtrcGuideDesc* d) {
    if (!d) return gfail(ATRC_ERR_INVALID_ARG, "atrc_guide_default_desc: null argument");
    std::memset(d, 0, sizeof(*d));
    d->log2_table = 19;
    // guiding needs a smooth field: finer levels memorise single records
    // (the training loss falls below the achievable optimum)
    d->base_resolution = 4;
    d->max_resolution = 64;
    // vertices past depth 3 carry little of the image's variance on the
    // indoor workload but cost inference (best time to relMSE 1e-3 of
    // depths 2, 3, 4 and all)
    d->max_depth = 5;
    d->learning_rate = 1e-2f;
    d->max_select = kGuideMaxSelect;
    d->target_clamp = 0.0f;
    d->batch = 1 << 18;
    d->record_capacity = 1 << 20;
    d->seed = 7;
    return ATRC_OK;
}

int atrc_guide_create(int device, const float scene_lo[3], const float scene_hi[3], const AtrcGuideDesc* desc,
                      AtrcGuide** out) {
    if (!desc || !out || !scene_lo || !scene_hi) return gfail(ATRC_ERR_INVALID_ARG, "atrc_guide_create: null argument");
    *out = nullptr;
    if (desc->log2_table < 8 || desc->log2_table > 22 || desc->base_resolution < 2 ||
        desc->max_resolution < desc->base_resolution || desc->batch < kTile || desc->record_capacity < kTile ||
        !(desc->learning_rate > 0) || desc->max_depth < 0 || !(desc->max_select > 0 && desc->max_select <= 0.99f) ||
        !(desc->target_clamp >= 0))
        return gfail(ATRC_ERR_INVALID_ARG, "atrc_guide_create: parameter out of range");
    return gguarded([&] {
        auto g = std::make_unique<AtrcGuide>();
        GuideImpl& G = g->impl;
        G.device = device;
        CK(cudaSetDevice(device));
        int sms = 0;
        CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
        G.sm_count = sms;
        CK(cudaStreamCreateWithFlags(&G.stream, cudaStreamNonBlocking));
        G.desc = *desc;
        HashGrid& hg = G.grid;
        hg.log2_table = desc->log2_table;
        const double growth = std::exp((std::log(double(desc->max_resolution)) - std::log(double(desc->base_resolution))) /
                                       double(kHashLevels - 1));
        for (int l = 0; l < kHashLevels; ++l)
            hg.res[l] = std::max(1, int(std::floor(double(desc->base_resolution) * std::pow(growth, l) + 1e-9)));
        for (int a = 0; a < 3; ++a) {
            const float ext = std::max(scene_hi[a] - scene_lo[a], 1e-6f);
            hg.lo[a] = scene_lo[a] - 1e-3f * ext;
            hg.inv_ext[a] = 1.0f / (ext * 1.002f);
        }
        G.table_n = size_t(kHashLevels) << desc->log2_table;
        G.table_n *= kHashFeatures;
        // initial parameters (seeded): Glorot-uniform weights, the output
        // layer scaled down so that the first mixtures are broad; table
        // entries U(-1e-4, 1e-4)
        std::mt19937_64 rng(desc->seed);
        std::uniform_real_distribution<float> U(-1.0f, 1.0f);
        std::vector<float> w(kWeights);
        auto fill = [&](int off, int out_, int in_, float scale) {
            const float s = std::sqrt(6.0f / float(in_ + out_)) * scale;
            for (int i = 0; i < out_ * in_; ++i) w[off + i] = s * U(rng);
        };
        fill(kOffW1, kGuideHidden, kGuideIn, 1.0f);
        fill(kOffW2, kGuideHidden, kGuideHidden, 1.0f);
        fill(kOffW3, kGuideHidden, kGuideHidden, 1.0f);
        fill(kOffW4, kGuideOut, kGuideHidden, 0.1f);
        std::vector<float> tab(G.table_n);
        for (auto& x : tab) x = 1e-4f * U(rng);
        G.w_f.alloc(kWeights * 4); G.w_g.alloc(kWeights * 4); G.w_m.alloc(kWeights * 4); G.w_v.alloc(kWeights * 4);
        G.w_bf.alloc(kWeights * 2);
        G.t_f.alloc(G.table_n * 4); G.t_g.alloc(G.table_n * 4); G.t_m.alloc(G.table_n * 4); G.t_v.alloc(G.table_n * 4);
        G.t_h.alloc(G.table_n * 2);
        G.records.alloc(size_t(desc->record_capacity) * sizeof(GuideRecord));
        G.live.alloc(size_t(desc->record_capacity) * sizeof(GuideRecord));
        G.rec_count.alloc(2 * sizeof(int));
        G.scratch.alloc(64);
        G.err.alloc(sizeof(int));
        cudaStream_t s = G.stream;
        CK(cudaMemcpyAsync(G.w_f.p, w.data(), kWeights * 4, cudaMemcpyHostToDevice, s));
        CK(cudaMemcpyAsync(G.t_f.p, tab.data(), G.table_n * 4, cudaMemcpyHostToDevice, s));
        for (DevBuf* b : {&G.w_g, &G.w_m, &G.w_v, &G.t_g, &G.t_m, &G.t_v, &G.err, &G.rec_count})
            CK(cudaMemsetAsync(b->p, 0, b->bytes, s));
        k_copy_params<__nv_bfloat16><<<64, 256, 0, s>>>(G.w_f.as<float>(), G.w_bf.as<__nv_bfloat16>(), kWeights);
        k_copy_params<__half><<<G.sm_count * 4, 256, 0, s>>>(G.t_f.as<float>(), G.t_h.as<__half>(), G.table_n);
        CK(cudaGetLastError());
        set_smem_limits();
        CK(cudaStreamSynchronize(s));
        *out = g.release();
        return int(ATRC_OK);
    });
}

void atrc_guide_destroy(AtrcGuide* g) {
    if (!g) return;
    cudaSetDevice(g->impl.device);
    cudaStreamSynchronize(g->impl.stream);
    delete g;
}

int atrc_guide_params(AtrcGuide* g, float* weights, float* table, int set) {
    if (!g) return gfail(ATRC_ERR_INVALID_ARG, "atrc_guide_params: null guide");
    return gguarded([&] {
        GuideImpl& G = g->impl;
        CK(cudaSetDevice(G.device));
        cudaStream_t s = G.stream;
        if (set) {
            if (weights) CK(cudaMemcpyAsync(G.w_f.p, weights, kWeights * 4, cudaMemcpyHostToDevice, s));
            if (table) CK(cudaMemcpyAsync(G.t_f.p, table, G.table_n * 4, cudaMemcpyHostToDevice, s));
            k_copy_params<__nv_bfloat16><<<64, 256, 0, s>>>(G.w_f.as<float>(), G.w_bf.as<__nv_bfloat16>(), kWeights);
            k_copy_params<__half><<<G.sm_count * 4, 256, 0, s>>>(G.t_f.as<float>(), G.t_h.as<__half>(), G.table_n);
            CK(cudaGetLastError());
        } else {
            if (weights) CK(cudaMemcpyAsync(weights, G.w_f.p, kWeights * 4, cudaMemcpyDeviceToHost, s));
            if (table) CK(cudaMemcpyAsync(table, G.t_f.p, G.table_n * 4, cudaMemcpyDeviceToHost, s));
        }
        CK(cudaStreamSynchronize(s));
        return int(ATRC_OK);
    });
}

int atrc_guide_set_max_select(AtrcGuide* g, float max_select) {
    if (!g || !(max_select > 0 && max_select <= 0.99f))
        return gfail(ATRC_ERR_INVALID_ARG, "atrc_guide_set_max_select: max_select must be in (0, 0.99]");
    g->impl.desc.max_select = max_select;
    return int(ATRC_OK);
}

int atrc_guide_info(AtrcGuide* g, AtrcGuideInfo* info) {
    if (!g || !info) return gfail(ATRC_ERR_INVALID_ARG, "atrc_guide_info: null argument");
    const GuideImpl& G = g->impl;
    std::memset(info, 0, sizeof(*info));
    info->weights = kWeights;
    info->table_floats = G.table_n;
    info->levels = kHashLevels;
    info->inputs = kGuideIn;
    info->hidden = kGuideHidden;
    info->outputs = kGuideOut;
    info->lobes = kGuideLobes;
    info->steps = G.steps;
    for (int a = 0; a < 3; ++a) { info->grid_lo[a] = G.grid.lo[a]; info->grid_inv_extent[a] = G.grid.inv_ext[a]; }
    for (int l = 0; l < kHashLevels; ++l) info->grid_res[l] = G.grid.res[l];
    info->log2_table = G.grid.log2_table;
    info->max_select = G.desc.max_select;
    return ATRC_OK;
}

// queries: n x 10 floats (pos, normal, wo, roughness); raw: n x 48 outputs
int atrc_guide_eval(AtrcGuide* g, const float* queries, size_t n, float* raw) {
    if (!g || (n && (!queries || !raw))) return gfail(ATRC_ERR_INVALID_ARG, "atrc_guide_eval: null argument");
    if (n > (size_t(1) << 26)) return gfail(ATRC_ERR_INVALID_ARG, "atrc_guide_eval: too many queries");
    if (n == 0) return ATRC_OK;
    return gguarded([&] {
        GuideImpl& G = g->impl;
        CK(cudaSetDevice(G.device));
        cudaStream_t s = G.stream;
        std::vector<GuideQuery> q(n);
        for (size_t i = 0; i < n; ++i) {
            const float* a = queries + 10 * i;
            std::memcpy(q[i].pos, a, 3 * 4);
            std::memcpy(q[i].nrm, a + 3, 3 * 4);
            std::memcpy(q[i].wo, a + 6, 3 * 4);
            q[i].rough = a[9];
            q[i].slot = 0;
            q[i].pad = 0;
        }
        DevBuf dq, dr, dx, dn;
        const size_t tiles = (n + kTile - 1) / kTile;
        dq.alloc(n * sizeof(GuideQuery));
        dr.alloc(n * kGuideOut * 4);
        dx.alloc(tiles * kGuideTileBytes);
        dn.alloc(sizeof(int));
        const int ni = int(n);
        CK(cudaMemcpyAsync(dq.p, q.data(), n * sizeof(GuideQuery), cudaMemcpyHostToDevice, s));
        CK(cudaMemcpyAsync(dn.p, &ni, sizeof(int), cudaMemcpyHostToDevice, s));
        // the FP32 master table, so that the check needs no FP16 rounding
        k_guide_encode<float><<<G.sm_count * 4, 128, 0, s>>>(G.grid, G.t_f.as<float>(), dq.as<GuideQuery>(), ni,
                                                            dx.as<uint8_t>());
        k_guide_mlp<false><<<G.sm_count * 2, kTile, kInfSmem, s>>>(G.view(), dx.as<uint8_t>(), dn.as<int>(),
                                                                  dr.as<float>(), G.err.as<int>());
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(raw, dr.p, n * kGuideOut * 4, cudaMemcpyDeviceToHost, s));
        check_err(G, "atrc_guide_eval");
        return int(ATRC_OK);
    });
}

// Guide pdf of (query, direction) pairs and the selection probability,
// through the inference kernel and the device decoding.
int atrc_guide_pdf(AtrcGuide* g, const float* queries, const float* dirs, size_t n, float* pdf, float* select) {
    if (!g || (n && (!queries || !dirs || !pdf || !select))) return gfail(ATRC_ERR_INVALID_ARG, "atrc_guide_pdf: null argument");
    if (n > (size_t(1) << 26)) return gfail(ATRC_ERR_INVALID_ARG, "atrc_guide_pdf: too many queries");
    if (n == 0) return ATRC_OK;
    return gguarded([&] {
        GuideImpl& G = g->impl;
        CK(cudaSetDevice(G.device));
        cudaStream_t s = G.stream;
        std::vector<GuideQuery> q(n);
        for (size_t i = 0; i < n; ++i) {
            const float* a = queries + 10 * i;
            std::memcpy(q[i].pos, a, 3 * 4);
            std::memcpy(q[i].nrm, a + 3, 3 * 4);
            std::memcpy(q[i].wo, a + 6, 3 * 4);
            q[i].rough = a[9];
            q[i].slot = 0;
            q[i].pad = 0;
        }
        DevBuf dq, dm, dd, dout, dn, dx;
        dx.alloc((n + kTile - 1) / kTile * kGuideTileBytes);
        dq.alloc(n * sizeof(GuideQuery));
        dm.alloc(n * kGuideOut * 4);
        dd.alloc(n * 3 * 4);
        dout.alloc(n * 2 * 4);
        dn.alloc(sizeof(int));
        const int ni = int(n);
        CK(cudaMemcpyAsync(dq.p, q.data(), n * sizeof(GuideQuery), cudaMemcpyHostToDevice, s));
        CK(cudaMemcpyAsync(dd.p, dirs, n * 3 * 4, cudaMemcpyHostToDevice, s));
        CK(cudaMemcpyAsync(dn.p, &ni, sizeof(int), cudaMemcpyHostToDevice, s));
        k_guide_encode<__half><<<G.sm_count * 4, 128, 0, s>>>(G.grid, G.t_h.as<__half>(), dq.as<GuideQuery>(), ni,
                                                             dx.as<uint8_t>());
        k_guide_mlp<true><<<G.sm_count * 2, kTile, kInfSmem, s>>>(G.view(), dx.as<uint8_t>(), dn.as<int>(),
                                                                 dm.as<float>(), G.err.as<int>());
        k_mix_pdf<<<G.sm_count * 4, 128, 0, s>>>(dm.as<float>(), dd.as<float>(), ni, dout.as<float>(),
                                                dout.as<float>() + n);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(pdf, dout.p, n * 4, cudaMemcpyDeviceToHost, s));
        CK(cudaMemcpyAsync(select, dout.as<float>() + n, n * 4, cudaMemcpyDeviceToHost, s));
        check_err(G, "atrc_guide_pdf");
        return int(ATRC_OK);
    });
}

// One Adam step on `n` records at `records` (device) -- internal helper.
static void train_step(GuideImpl& G, const GuideRecord* rec, int n, float* loss_out) {
    cudaStream_t s = G.stream;
    float* sc = G.scratch.as<float>();  // [0] target sum, [1] loss
    CK(cudaMemsetAsync(sc, 0, 2 * sizeof(float), s));
    k_target_sum<<<G.sm_count * 2, 256, 0, s>>>(rec, n, sc);
    TrainArgs a;
    a.rec = rec;
    a.n = n;
    a.weight_sum = sc;
    a.grad_w = G.w_g.as<float>();
    a.grad_table = G.t_g.as<float>();
    a.loss = sc + 1;
    a.target_clamp = G.desc.target_clamp;
    const int tiles = (n + kTile - 1) / kTile;
    k_guide_train<<<std::min(tiles, G.sm_count), kTile, kTrSmem, s>>>(G.view(), a, G.err.as<int>());
    ++G.steps;
    AdamArgs ad;
    ad.lr = G.desc.learning_rate;
    ad.b1 = 0.9f;
    ad.b2 = 0.99f;
    ad.eps = 1e-15f;
    ad.c1 = float(1.0 / (1.0 - std::pow(0.9, G.steps)));
    ad.c2 = float(1.0 / (1.0 - std::pow(0.99, G.steps)));
    k_guide_adam<__nv_bfloat16><<<64, 256, 0, s>>>(G.w_f.as<float>(), G.w_g.as<float>(), G.w_m.as<float>(),
                                                   G.w_v.as<float>(), G.w_bf.as<__nv_bfloat16>(), kWeights, ad);
    k_guide_adam<__half><<<G.sm_count * 8, 256, 0, s>>>(G.t_f.as<float>(), G.t_g.as<float>(), G.t_m.as<float>(),
                                                        G.t_v.as<float>(), G.t_h.as<__half>(), G.table_n, ad);
    CK(cudaGetLastError());
    if (loss_out) CK(cudaMemcpyAsync(loss_out, sc + 1, sizeof(float), cudaMemcpyDeviceToHost, s));
}

int atrc_guide_train(AtrcGuide* g, int steps, float* last_loss) {
    if (!g || steps < 0) return gfail(ATRC_ERR_INVALID_ARG, "atrc_guide_train: invalid argument");
    return gguarded([&] {
        GuideImpl& G = g->impl;
        CK(cudaSetDevice(G.device));
        cudaStream_t s = G.stream;
        int counts[2] = {0, 0};  // records stored, guided vertices seen
        CK(cudaMemcpyAsync(counts, G.rec_count.p, 2 * sizeof(int), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        const int cap = int(G.desc.record_capacity);
        const int stored = std::min(counts[0], cap);
        // the next recording pass keeps about 0.95 cap of its guided vertices
        // (this pass's count stands in for the next one's)
        if (counts[1] > 0)
            G.record_keep = std::min(1.0f, std::max(1.0f / 4096.0f, 0.95f * float(cap) / float(counts[1])));
        if (last_loss) *last_loss = 0;
        if (stored < kTile) return int(ATRC_OK);
        int* live_n = reinterpret_cast<int*>(G.scratch.as<float>() + 4);
        CK(cudaMemsetAsync(live_n, 0, sizeof(int), s));
        k_live_records<<<G.sm_count * 4, 256, 0, s>>>(G.records.as<GuideRecord>(), stored,
                                                     G.live.as<GuideRecord>(), live_n);
        CK(cudaGetLastError());
        int n = 0;
        CK(cudaMemcpyAsync(&n, live_n, sizeof(int), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        if (n < kTile) return int(ATRC_OK);
        const int batch = std::min(n, int(G.desc.batch));
        float loss = 0;
        for (int k = 0; k < steps; ++k) {
            // consecutive batches through the live records (wrapping)
            const int start = int((size_t(k) * batch) % size_t(n));
            const int cnt = std::min(batch, n - start);
            train_step(G, G.live.as<GuideRecord>() + start, cnt, &loss);
        }
        check_err(G, "atrc_guide_train");
        if (last_loss) *last_loss = loss;
        return int(ATRC_OK);
    });
}

// Train on host-provided records (n x 24 floats in GuideRecord layout).
int atrc_guide_train_records(AtrcGuide* g, const float* records, size_t n, int steps, float* last_loss) {
    if (!g || !records || n < kTile || steps < 0)
        return gfail(ATRC_ERR_INVALID_ARG, "atrc_guide_train_records: invalid argument");
    return gguarded([&] {
        GuideImpl& G = g->impl;
        CK(cudaSetDevice(G.device));
        if (n > size_t(G.desc.record_capacity)) throw std::runtime_error("more records than the guide's capacity");
        CK(cudaMemcpyAsync(G.records.p, records, n * sizeof(GuideRecord), cudaMemcpyHostToDevice, G.stream));
        const int cnt = int(n);
        CK(cudaMemcpyAsync(G.rec_count.p, &cnt, sizeof(int), cudaMemcpyHostToDevice, G.stream));
        CK(cudaStreamSynchronize(G.stream));
        const int batch = std::min(cnt, int(G.desc.batch));
        float loss = 0;
        for (int k = 0; k < steps; ++k) {
            const int start = int((size_t(k) * batch) % size_t(cnt));
            train_step(G, G.records.as<GuideRecord>() + start, std::min(batch, cnt - start), &loss);
        }
        check_err(G, "atrc_guide_train_records");
        if (last_loss) *last_loss = loss;
        return int(ATRC_OK);
    });
}

// The loss gradients of one batch of host records (n x 24 floats, at most
// the record capacity) at the current parameters: the training kernel
// without the Adam step.  The gradient buffers are read back and cleared, so
// the parameters and the optimiser state are untouched.
int atrc_guide_gradients(AtrcGuide* g, const float* records, size_t n, float* grad_weights, float* grad_table,
                         float* loss) {
    if (!g || !records || n < kTile || !grad_weights || !grad_table)
        return gfail(ATRC_ERR_INVALID_ARG, "atrc_guide_gradients: invalid argument");
    return gguarded([&] {
        GuideImpl& G = g->impl;
        CK(cudaSetDevice(G.device));
        if (n > size_t(G.desc.record_capacity)) throw std::runtime_error("more records than the guide's capacity");
        cudaStream_t s = G.stream;
        CK(cudaMemcpyAsync(G.records.p, records, n * sizeof(GuideRecord), cudaMemcpyHostToDevice, s));
        float* sc = G.scratch.as<float>();
        CK(cudaMemsetAsync(sc, 0, 2 * sizeof(float), s));
        CK(cudaMemsetAsync(G.w_g.p, 0, kWeights * sizeof(float), s));
        CK(cudaMemsetAsync(G.t_g.p, 0, G.table_n * sizeof(float), s));
        const GuideRecord* rec = G.records.as<GuideRecord>();
        k_target_sum<<<G.sm_count * 2, 256, 0, s>>>(rec, int(n), sc);
        TrainArgs a;
        a.rec = rec;
        a.n = int(n);
        a.weight_sum = sc;
        a.grad_w = G.w_g.as<float>();
        a.grad_table = G.t_g.as<float>();
        a.loss = sc + 1;
        a.target_clamp = G.desc.target_clamp;
        const int tiles = int((n + kTile - 1) / kTile);
        k_guide_train<<<std::min(tiles, G.sm_count), kTile, kTrSmem, s>>>(G.view(), a, G.err.as<int>());
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(grad_weights, G.w_g.p, kWeights * sizeof(float), cudaMemcpyDeviceToHost, s));
        CK(cudaMemcpyAsync(grad_table, G.t_g.p, G.table_n * sizeof(float), cudaMemcpyDeviceToHost, s));
        float l = 0;
        CK(cudaMemcpyAsync(&l, sc + 1, sizeof(float), cudaMemcpyDeviceToHost, s));
        CK(cudaMemsetAsync(G.w_g.p, 0, kWeights * sizeof(float), s));
        CK(cudaMemsetAsync(G.t_g.p, 0, G.table_n * sizeof(float), s));
        check_err(G, "atrc_guide_gradients");
        if (loss) *loss = l;
        return int(ATRC_OK);
    });
}

// Copy the records of the last recording render to the host.
int atrc_guide_records(AtrcGuide* g, float* records, size_t cap, size_t* count) {
    if (!g || !count) return gfail(ATRC_ERR_INVALID_ARG, "atrc_guide_records: null argument");
    return gguarded([&] {
        GuideImpl& G = g->impl;
        CK(cudaSetDevice(G.device));
        int n = 0;
        CK(cudaMemcpyAsync(&n, G.rec_count.p, sizeof(int), cudaMemcpyDeviceToHost, G.stream));
        CK(cudaStreamSynchronize(G.stream));
        n = std::min(n, int(G.desc.record_capacity));
        *count = size_t(n);
        if (records && cap) {
            const size_t m = std::min(cap, size_t(n));
            CK(cudaMemcpyAsync(records, G.records.p, m * sizeof(GuideRecord), cudaMemcpyDeviceToHost, G.stream));
            CK(cudaStreamSynchronize(G.stream));
        }
        return int(ATRC_OK);
    });
}

}  // extern "C"
