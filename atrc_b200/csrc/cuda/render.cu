// Wavefront path tracer (`pt_cuda`) and the device half of the C ABI.
//
// Replaces PerPixelRenderer::render / render_grid
// (src/tracer/src/core/renderer/perpixel_renderer.cpp:13-207) driving
// render::trace_std (src/tracer/src/render/path_tracing.cpp:15-225) with the
// MIS direct lighting of src/tracer/src/render/direct_illum.cpp:11-278.
//
// Structure: a pool of P path slots in HBM (structure of arrays); every
// iteration runs six kernels over device-side queues, so the host never reads
// queue sizes inside the loop:
//   begin     - 1 thread: flip queues, plan how many new camera samples to take
//   generate  - camera rays for free slots (thin_lens.cpp:74-94)
//   extend    - closest hit for every queued path
//   shade     - resolve the previous vertex's MIS-BSDF term, Russian roulette,
//               medium sampling, emission, next-event estimation (one shadow
//               ray per light), BSDF sampling
//   shadow    - any hit for the shadow queue, unoccluded contributions added
//   finish    - FP64 film splat of completed paths, slots returned
// The BSDF sample of a vertex serves both as the MIS-BSDF ray of
// mis_sample_bsdf and as the continuation ray (the reference draws two
// independent samples from the same distribution; the expectation of both
// terms is unchanged), which saves one closest-hit ray per vertex.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "../../../include/atrc_cuda.h"
#include "../host/scene_build.h"
#include "dev_math.cuh"
#include "dev_scene.h"
#include "dev_shade.cuh"
#include "dev_trace.cuh"
#include "cuda_util.h"
#include "dev_guide_enc.cuh"
#include "guide.h"

#ifndef ATRC_SHADE_MIN_BLOCKS
#define ATRC_SHADE_MIN_BLOCKS 4  // k_shade blocks per SM the register budget must allow
#endif
#ifndef ATRC_TRACE_MIN_BLOCKS
#define ATRC_TRACE_MIN_BLOCKS 8  // the same for the traversal kernels
#endif
#ifndef ATRC_SHADOW_MIN_BLOCKS
#define ATRC_SHADOW_MIN_BLOCKS 10  // k_shadow: 48 registers (8 blocks, 64 registers, measured 2-6 % slower)
#endif

namespace atrc {
namespace {

using namespace dev;

// ------------------------------------------------------- warp aggregation
__device__ __forceinline__ int warp_append(int* counter, bool pred) {
    const unsigned active = __activemask();
    const unsigned mask = __ballot_sync(active, pred);
    if (!pred) return -1;
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(mask) - 1;
    int base = 0;
    if (lane == leader) base = atomicAdd(counter, __popc(mask));
    base = __shfl_sync(mask, base, leader);
    return base + __popc(mask & ((1u << lane) - 1u));
}

// ------------------------------------------------------------ ray queries
// Persistent warps step their traversals round by round and refill the
// lanes whose rays are done from `cursor`, as k_extend_fetch does: a batch of
// incoherent queries keeps most lanes busy instead of waiting for each
// warp's longest ray (4M incoherent rays on the instanced scene: 1.53 ->
// 1.74 G closest-hit queries/s, 1.89 -> 2.16 G any-hit, identical hits).
template <int ISECT, bool ANY>
__global__ void __launch_bounds__(kTraceBlock, ATRC_TRACE_MIN_BLOCKS) k_trace_rays(Scene S, const AtrcRay* __restrict__ rays, int n, AtrcHit* __restrict__ hits,
                             int* cursor, int* watchdog) {
    constexpr int kRefill = 16;
    const int lane = threadIdx.x & 31;
    TraceCount tc{0, 0, 0};
    int32_t stack[kStackSize];
    Tracer<ISECT, ANY, false> tr;
    int i = -1, wd = 0;
    bool drained = false;
    for (;;) {
        const unsigned idle = __ballot_sync(0xffffffffu, i < 0);
        if (!drained && __popc(idle) >= kRefill) {
            int base = 0;
            if (lane == 0) base = atomicAdd(cursor, __popc(idle));
            base = __shfl_sync(0xffffffffu, base, 0);
            if (base + __popc(idle) >= n) drained = true;
            if (i < 0) {
                const int k = base + __popc(idle & ((1u << lane) - 1u));
                if (k < n) {
                    i = k;
                    const AtrcRay q = rays[i];
                    tr.init(S, stack, Vec3(q.o[0], q.o[1], q.o[2]), Vec3(q.d[0], q.d[1], q.d[2]), q.t_min, q.t_max);
                }
            }
        }
        if (drained && __all_sync(0xffffffffu, i < 0)) break;
        if (i >= 0 && tr.step(S, &wd, &tc)) {
            Hit h;
            h.entity = -1;
            h.tri = -1;
            h.t = h.u = h.v = 0.0f;
            const bool hit = tr.result(&h);
            AtrcHit r;
            if (ANY) {
                r.t = hit ? 1.0f : -1.0f;
                r.entity = hit ? 0 : -1;
                r.prim = 0;
                r.u = 0;
            } else if (hit) {
                r.t = h.t;
                r.entity = h.entity;
                r.prim = h.tri >= 0 ? int32_t(S.tri_orig[h.tri]) : 0;
                r.u = h.u;
            } else {
                r.t = -1;
                r.entity = -1;
                r.prim = -1;
                r.u = 0;
            }
            hits[i] = r;
            i = -1;
        }
    }
    if (wd) atomicMax(watchdog, wd);
}

// ------------------------------------------------------------ wavefront
enum PathFlags : int {
    PF_MIS = 1,          // a MIS-BSDF term waits for this ray's hit
    PF_MIS_DELTA = 2,    // ... from a delta (specular) sample
    PF_TERMINATE = 4,    // finish after resolving the pending MIS term
    PF_REC_PENDING = 8,  // the path's last guide record waits for its arrival radiance
};

struct Counters {
    int in, out;              // queue buffers read / written this iteration
    int n_ext, n_next;        // paths to extend / continuations written
    int n_shadow, n_finish;
    int n_guide;              // guide queries this iteration
    int n_sss;                // subsurface walks queued this iteration
    int ext_cursor;           // next extend-queue entry for k_extend_fetch
    int sh_cursor;            // next shadow-queue entry for k_shadow_fetch
    int n_free, n_new, n_cont;
    int gen_ticket;           // k_generate: free slots claimed this iteration
    int ext_ticket;           // k_generate: extend-queue entries written (slot order)
    unsigned long long gen_base, issued, total, completed;
    unsigned long long rays_closest, rays_shadow, iterations;
    unsigned long long cnt_closest[3], cnt_shadow[3];  // nodes, tris, entities
    unsigned long long t_start;  // %globaltimer when the render's counters were reset
    int windows;                 // bounce-loop windows run by the device-side loop
    int watchdog, done;
};

// Watchdog code of the device-side bounce loop (atrc_cuda_render_batch):
// the loop ran more windows than any path length allows.
constexpr int kWatchdogLoop = 8;

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void flush_count(unsigned long long* dst, const TraceCount& tc) {
    unsigned long long v[3] = {tc.nodes, tc.tris, tc.ents};
    for (int k = 0; k < 3; ++k) {
        unsigned long long x = v[k];
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(__activemask(), x, o);
        if ((threadIdx.x & 31) == 0) atomicAdd(dst + k, x);
    }
}

struct Camera {
    float pos[3], fx[3], fy[3], fz[3];
    float film_w, film_h, focal, lens_radius;
};

struct Film {
    double *value, *weight, *value_sq, *albedo, *normal, *denoise;
};

// One camera view of a render.  A render is a batch of views (one for
// atrc_cuda_render) whose samples share one path pool: global sample index k
// belongs to the view with start <= k < start + count.
//
// The film is cut into tiles of G x G pixels (task_grid_size).  Each tile
// samples every pixel of its bound grown by the filter's reach
// (sample_bound_of, framebuffer.h:36-47) and splats only into itself
// (FilmGrid::apply, render_target.h:383-395), so a pixel near a tile edge is
// sampled once per tile that reaches it.  The sample grid lays the tiles'
// sample bounds side by side: column u belongs to tile column gx where
// tile_cols[gx].w <= u < tile_cols[gx + 1].w, and is pixel
// tile_cols[gx].z + (u - tile_cols[gx].w); rows likewise.  With the default
// box filter (radius 0.5 - eps) the sample grid is the film itself.
struct View {
    int W, H;
    int G, TX, TY;          // tile edge, tile columns / rows
    int SW, SH;             // sample grid size (sum of the tiles' sample bounds)
    int E0X, E0Y;           // sample-bound extent of the first tile column / row
    int4* tile_cols;        // per tile column: x0, x1, first sampled x, first u
    int4* tile_rows;        // per tile row:    y0, y1, first sampled y, first v
    int first_spp;
    unsigned long long seed;
    unsigned long long start, count;  // global sample indices of this view
    Camera cam;
    int filter_type;
    float filter_radius, filter_value, filter_alpha, filter_exp;
    Film film;
};
constexpr int kTileBits = 22;  // path state packs (view << kTileBits) | tile
constexpr int kMaxViews = 1024;

// Settings shared by every view of a render.
struct Params {
    int nviews;
    const View* views;                 // device array
    unsigned long long* view_done;     // per view: finished samples (batch renders; else null)
    unsigned long long* view_time;     // per view: %globaltimer when its last sample was splatted
    int sort_mode, nkeys;   // shade-queue sort (AtrcSortMode, resolved) and key count
    int slot_queue;         // 1: extend queue in slot order (AtrcTuning::queue_order)
    int min_depth, max_depth, specular_depth;
    float cont_prob, eps;
    int guide_on;           // sample surface vertices with the learned guide
    GuideFrame gf;          // guide buffers of this call (zero when guide_on == 0)
    int renderer;           // AtrcRendererType
    int ao_count;           // ao: occlusion rays per camera sample
    float ao_dist;          // ao: occlusion distance
    float ao_low[3], ao_high[3], ao_bg[3];
};

// Slot states: free, holding a path that continues next iteration, or
// holding a path between its queue entry and its continuation / finish.
constexpr int kSlotBusy = 0, kSlotFree = 1, kSlotCont = 2;

struct Pool {
    float4 *ray_o, *ray_d;        // o.xyz tmin / d.xyz tmax
    float4* hit;                  // t, u, v, entity(bits)
    int* hit_tri;
    float4* coef;                 // coef.xyz, mis_pdf
    float4* L;                    // radiance.xyz, film x
    float4* mis_f;                // pending MIS numerator.xyz, film y
    float4* gb_albedo;            // albedo.xyz, denoise
    float4* gb_normal;            // normal.xyz
    uint4* st;                    // pixel, rng lo, rng hi, unused
    int4* ctr;                    // depth, s_depth, scattering_count, flags | medium << 8
    int* q[2];                    // extend queues
    int* q_sorted;                // the extend queue sorted by material key
    int* keys;                    // material key per extend-queue entry
    int* key_count;               // per key: entries this iteration
    int* key_cursor;              // per key: next write position in q_sorted
    int* q_finish;
    int* q_sss;                   // paths whose BSDF sample entered a subsurface material
    int* slot_state;              // per slot: kSlotFree / kSlotCont / kSlotBusy
    float4 *sh_o, *sh_d, *sh_c;   // shadow rays: o.tmin, d.tmax, contribution + path
    // shadow-queue sort by origin cell (AtrcTuning.shadow_sort): a 16^3 grid
    // over the scene bound in Morton order; k_shadow reads the queue through
    // sh_sorted so that a warp's rays start near each other
    int shadow_sort;
    int* sh_key;                  // per shadow entry: its origin's cell
    int* sh_sorted;               // shadow entries in cell order
    int* sh_count;                // per cell: entries this iteration
    int* sh_cursor;               // per cell: next write position in sh_sorted
    float sk_lo[3], sk_scale[3];  // origin -> cell coordinates (16 / extent)
    int cap, shadow_cap;
};
constexpr int kShadowKeys = 4096;  // 16 x 16 x 16 origin cells

__global__ void k_init(Pool P, int cap, int nkeys, Counters* c, unsigned long long total) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < cap) P.slot_state[i] = kSlotFree;
    if (i < nkeys) P.key_count[i] = 0;
    if (i < kShadowKeys) P.sh_count[i] = 0;
    if (i == 0) {
        memset(c, 0, sizeof(Counters));
        c->n_free = cap;
        c->total = total;
        c->out = 0;
        c->t_start = global_ns();
    }
}

// End of one window of the device-side bounce loop: run another window
// unless the work is done or a watchdog fired; after max_windows the loop
// stops with kWatchdogLoop instead of running on (no path lives that long).
__global__ void k_loop_cond(Counters* c, cudaGraphConditionalHandle h, int max_windows) {
    const int w = ++c->windows;
    bool more = c->done == 0 && c->watchdog == 0;
    if (more && w >= max_windows) {
        c->watchdog = kWatchdogLoop;
        more = false;
    }
    cudaGraphSetConditional(h, more ? 1u : 0u);
}

__global__ void k_begin(Counters* c) {
    c->iterations++;
    c->rays_shadow += c->n_shadow;
    c->n_free += c->n_finish;
    c->completed += c->n_finish;
    const int n_cont = c->n_next;
    c->in = c->out;
    c->out = c->in ^ 1;
    const unsigned long long remaining = c->total - c->issued;
    const int n_new = int(remaining < (unsigned long long)c->n_free ? remaining : (unsigned long long)c->n_free);
    c->gen_base = c->issued;
    c->issued += n_new;
    c->gen_ticket = 0;
    c->ext_ticket = 0;
    c->n_free -= n_new;
    c->n_new = n_new;
    c->n_cont = n_cont;
    c->n_ext = n_cont + n_new;
    c->rays_closest += c->n_ext;
    c->n_next = 0;
    c->n_shadow = 0;
    c->n_finish = 0;
    c->n_guide = 0;
    c->n_sss = 0;
    c->ext_cursor = 0;
    c->sh_cursor = 0;
    if (c->n_ext == 0) c->done = 1;
}

__device__ __forceinline__ Rng load_rng(const uint4& s) { Rng r; r.state = (uint64_t(s.z) << 32) | s.y; return r; }
__device__ __forceinline__ void store_rng(uint4& s, const Rng& r) { s.y = uint32_t(r.state); s.z = uint32_t(r.state >> 32); }
__device__ __forceinline__ Vec3 xyz(const float4& v) { return Vec3(v.x, v.y, v.z); }

// Tile tables of each view's sample grid (block = view, one thread; TX + TY
// entries).  The bounds use the reference's float expressions so both agree
// on every tile.
__global__ void k_tiles(Params p) {
    if (threadIdx.x != 0 || int(blockIdx.x) >= p.nviews) return;
    const View& v = p.views[blockIdx.x];
    const float r = v.filter_radius;
    int acc = 0;
    for (int g = 0; g < v.TX; ++g) {
        const int a0 = g * v.G, a1 = min(v.W, a0 + v.G) - 1;
        const int s0 = int(floorf(__fsub_rn(__fadd_rn(float(a0), 0.5f), r)));
        const int s1 = int(floorf(__fadd_rn(__fadd_rn(float(a1), 0.49999f), r)));
        v.tile_cols[g] = make_int4(a0, a1, s0, acc);
        acc += s1 - s0 + 1;
    }
    v.tile_cols[v.TX] = make_int4(0, 0, 0, acc);
    acc = 0;
    for (int g = 0; g < v.TY; ++g) {
        const int a0 = g * v.G, a1 = min(v.H, a0 + v.G) - 1;
        const int s0 = int(floorf(__fsub_rn(__fadd_rn(float(a0), 0.5f), r)));
        const int s1 = int(floorf(__fadd_rn(__fadd_rn(float(a1), 0.49999f), r)));
        v.tile_rows[g] = make_int4(a0, a1, s0, acc);
        acc += s1 - s0 + 1;
    }
    v.tile_rows[v.TY] = make_int4(0, 0, 0, acc);
}

// View of global sample index k (views are ordered by start).
__device__ __forceinline__ int view_of(const Params& p, unsigned long long k) {
    int lo = 0, hi = p.nviews - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (p.views[mid].start <= k) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// sample-grid coordinate -> (tile index along the axis, pixel coordinate)
__device__ __forceinline__ int tile_of(const int4* t, int n, int e0, int u, int* pix) {
    int g = min(n - 1, u / e0);
    while (g > 0 && t[g].w > u) --g;
    while (g + 1 < n && t[g + 1].w <= u) ++g;
    const int4 e = t[g];
    *pix = e.z + (u - e.w);
    return g;
}

// Block-wide ticket: the lanes with `pred` get consecutive values from
// *counter in thread order (one atomic per block); every thread receives its
// own ticket (or -1) and, in *first, the block's base.  All threads of the
// block call it together.
__device__ __forceinline__ int block_ticket(int* counter, bool pred, int* smem, int* first) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    const unsigned m = __ballot_sync(0xffffffffu, pred);
    if (lane == 0) smem[w] = __popc(m);
    __syncthreads();
    if (w == 0) {
        const int v = lane < nw ? smem[lane] : 0;
        int incl = v;
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        const int total = __shfl_sync(0xffffffffu, incl, 31);
        int base = 0;
        if (lane == 0 && total > 0) base = atomicAdd(counter, total);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (lane < nw) smem[lane] = base + incl - v;
        if (lane == 0) smem[32] = base;
    }
    __syncthreads();
    const int t = pred ? smem[w] + __popc(m & ((1u << lane) - 1u)) : -1;
    *first = smem[32];
    __syncthreads();
    return t;
}

// New samples go into free slots taken in ascending slot order: a block looks
// at blockDim consecutive slots and takes sample tickets for its free ones
// with one atomic (ticket t < n_new becomes sample gen_base + t), so new path
// state is written by neighbouring lanes whatever order the paths finished
// in.  Extend-queue positions: n_cont + t after the continuations k_shade
// appended (shade order), or, with p.slot_queue, one more ticket per block
// for its new paths and for its slots whose path continues, so the whole
// queue runs in slot order.  The sample -> pixel / random stream map does
// not depend on the slot, so the image does not either.
__global__ void k_generate(Scene S, Params p, Pool P, Counters* c) {
    __shared__ int tick[33];
    const int n = c->n_new;
    if (p.slot_queue ? c->n_ext == 0 : n == 0) return;
    const int in = c->in, n_cont = c->n_cont;
    const unsigned long long gen = c->gen_base;
    for (int i0 = blockIdx.x * blockDim.x; i0 < P.cap; i0 += gridDim.x * blockDim.x) {  // block-uniform
        const int slot = i0 + int(threadIdx.x);
        const int state = slot < P.cap ? P.slot_state[slot] : kSlotBusy;
        const bool is_free = state == kSlotFree && n > 0;
        int first;
        int i = block_ticket(&c->gen_ticket, is_free, tick, &first);
        // tickets only grow: past n_new every sample of this iteration is placed
        if (first >= n && !p.slot_queue) return;  // block-uniform
        const bool fresh = is_free && i < n;
        int qpos = n_cont + i;
        if (p.slot_queue) qpos = block_ticket(&c->ext_ticket, fresh || state == kSlotCont, tick, &first);
        if (qpos < 0 || (!p.slot_queue && !fresh)) continue;
        P.slot_state[slot] = kSlotBusy;
        P.q[in][qpos] = slot;
        if (!fresh) continue;
        const unsigned long long k = gen + i;
        const int vi = view_of(p, k);
        const View& v = p.views[vi];
        const unsigned long long local = k - v.start;
        const unsigned long long npix = (unsigned long long)v.SW * v.SH;
        const unsigned long long pixel = local % npix;
        const unsigned long long s = (unsigned long long)v.first_spp + local / npix;
        Rng rng;
        rng.state = mix64(v.seed ^ mix64(pixel * 0x9E3779B97F4A7C15ULL + s * 0xD1B54A32D192ED03ULL + 1));
        int px, py;
        const int gx = tile_of(v.tile_cols, v.TX, v.E0X, int(pixel % v.SW), &px);
        const int gy = tile_of(v.tile_rows, v.TY, v.E0Y, int(pixel / v.SW), &py);
        // render_grid (perpixel_renderer.cpp:27-36) + ThinLensCamera::sample_we
        const float fx = px + rng.u(), fy = py + rng.u();
        const float film_x = fx / v.W, film_y = fy / v.H;
        const float au = rng.u(), av = rng.u();
        const Camera& cam = v.cam;
        const Vec3 focal((0.5f - film_x) * cam.film_w, (film_y - 0.5f) * cam.film_h, cam.focal);
        float dx, dy;
        concentric_disk(au, av, &dx, &dy);
        const Vec3 lens(cam.lens_radius * dx, cam.lens_radius * dy, 0);
        const Vec3 FX(cam.fx[0], cam.fx[1], cam.fx[2]), FY(cam.fy[0], cam.fy[1], cam.fy[2]), FZ(cam.fz[0], cam.fz[1], cam.fz[2]);
        const Vec3 o = Vec3(cam.pos[0], cam.pos[1], cam.pos[2]) + FX * lens.x + FY * lens.y;
        const Vec3 ld = focal - lens;
        const Vec3 d = normalize(FX * ld.x + FY * ld.y + FZ * ld.z);
        P.ray_o[slot] = make_float4(o.x, o.y, o.z, 0.0f);
        P.ray_d[slot] = make_float4(d.x, d.y, d.z, INFINITY);
        P.coef[slot] = make_float4(1, 1, 1, 0);
        P.L[slot] = make_float4(0, 0, 0, fx);
        P.mis_f[slot] = make_float4(0, 0, 0, fy);
        P.gb_albedo[slot] = make_float4(0, 0, 0, 1);
        P.gb_normal[slot] = make_float4(0, 0, 0, 0);
        uint4 st;
        st.x = uint32_t(pixel);
        // the view and tile this sample splats into
        st.w = (uint32_t(vi) << kTileBits) | uint32_t(gy * v.TX + gx);
        store_rng(st, rng);
        P.st[slot] = st;
        P.ctr[slot] = make_int4(1, 1, 0, 0);
    }
}

constexpr int kMaterialTypes = 8;  // AtrcMaterialType values 0..7: type-sort keys 1..8
static_assert(ATRC_MAT_PHONG + 1 == kMaterialTypes, "one sort key per material type");

// Material key of a hit record: 0 for a miss, nkeys - 1 for a path inside a
// medium (its next step is medium sampling), else 1 + the material type or
// index of the hit entity.  Counted per warp (one atomic per distinct key).
__device__ __forceinline__ void count_key(const Scene& S, Pool& P, int sort_mode, int nkeys, int i, int slot,
                                          bool hit, int entity) {
    int key;
    const int med = reinterpret_cast<const int*>(P.ctr + slot)[3] >> 8;
    if (med != 0) key = nkeys - 1;
    else if (!hit) key = 0;
    else {
        const int m = S.entities[entity].material;
        key = 1 + (sort_mode == ATRC_SORT_TYPE ? S.materials[m].type : m);
    }
    P.keys[i] = key;
    const unsigned same = __match_any_sync(__activemask(), key);
    if ((threadIdx.x & 31) == __ffs(same) - 1) atomicAdd(P.key_count + key, __popc(same));
}

// Exclusive scan of key counts into write cursors (one block of 1024);
// clears the counts for the next iteration.
__device__ __forceinline__ void scan_counts(int* count, int* cursor, int nkeys) {
    __shared__ int part[1024];
    const int t = threadIdx.x, per = (nkeys + 1023) / 1024;
    const int b0 = min(nkeys, t * per), b1 = min(nkeys, b0 + per);
    int sum = 0;
    for (int k = b0; k < b1; ++k) sum += count[k];
    part[t] = sum;
    __syncthreads();
    for (int o = 1; o < 1024; o <<= 1) {
        const int v = t >= o ? part[t - o] : 0;
        __syncthreads();
        part[t] += v;
        __syncthreads();
    }
    int acc = part[t] - sum;
    for (int k = b0; k < b1; ++k) {
        const int cnt = count[k];
        cursor[k] = acc;
        acc += cnt;
        count[k] = 0;
    }
}

__global__ void __launch_bounds__(1024) k_sort_scan(Pool P, int nkeys) { scan_counts(P.key_count, P.key_cursor, nkeys); }

__global__ void __launch_bounds__(1024) k_shsort_scan(Pool P) { scan_counts(P.sh_count, P.sh_cursor, kShadowKeys); }

// Scatter the extend queue into key order (order within a key is arbitrary).
// A block takes kScatterPer x blockDim entries per pass, counts them per key
// in shared memory and reserves each key's run with one global atomic, so the
// few key cursors see one atomic per key per block pass instead of one per
// warp (same-address atomics serialise in L2).  More keys than kScatterKeys
// (material sort of a large scene): one atomic per key per warp.
constexpr int kScatterKeys = 1024, kScatterPer = 8;

__global__ void k_sort_scatter(Pool P, Counters* c, int nkeys) {
    __shared__ int run[kScatterKeys];
    const int n = c->n_ext, in = c->in, lane = threadIdx.x & 31;
    if (nkeys > kScatterKeys) {
        for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
            const int key = P.keys[i];
            const unsigned same = __match_any_sync(__activemask(), key);
            const int leader = __ffs(same) - 1;
            int base = 0;
            if (lane == leader) base = atomicAdd(P.key_cursor + key, __popc(same));
            base = __shfl_sync(same, base, leader);
            P.q_sorted[base + __popc(same & ((1u << lane) - 1u))] = P.q[in][i];
        }
        return;
    }
    const int span = kScatterPer * blockDim.x;
    for (int i0 = blockIdx.x * span; i0 < n; i0 += gridDim.x * span) {  // block-uniform
        for (int k = threadIdx.x; k < nkeys; k += blockDim.x) run[k] = 0;
        __syncthreads();
        int key[kScatterPer], rank[kScatterPer], slot[kScatterPer];
#pragma unroll
        for (int e = 0; e < kScatterPer; ++e) {
            const int i = i0 + e * int(blockDim.x) + int(threadIdx.x);
            key[e] = i < n ? P.keys[i] : -1;
            slot[e] = i < n ? P.q[in][i] : 0;
            const unsigned same = __match_any_sync(0xffffffffu, key[e]);
            const int leader = __ffs(same) - 1;
            int r = 0;
            if (lane == leader && key[e] >= 0) r = atomicAdd(run + key[e], __popc(same));
            rank[e] = __shfl_sync(0xffffffffu, r, leader) + __popc(same & ((1u << lane) - 1u));
        }
        __syncthreads();
        for (int k = threadIdx.x; k < nkeys; k += blockDim.x)
            if (run[k] > 0) run[k] = atomicAdd(P.key_cursor + k, run[k]);
        __syncthreads();
#pragma unroll
        for (int e = 0; e < kScatterPer; ++e)
            if (key[e] >= 0) P.q_sorted[run[key[e]] + rank[e]] = slot[e];
        __syncthreads();
    }
}

// Scatter the shadow queue's entry indices into cell order, with the same
// block-aggregated key runs as k_sort_scatter (4096 cells: 16 KB of shared
// memory per block).
__global__ void __launch_bounds__(128) k_shsort_scatter(Pool P, Counters* c) {
    __shared__ int run[kShadowKeys];
    const int n = min(c->n_shadow, P.shadow_cap), lane = threadIdx.x & 31;
    const int span = kScatterPer * blockDim.x;
    for (int i0 = blockIdx.x * span; i0 < n; i0 += gridDim.x * span) {  // block-uniform
        for (int k = threadIdx.x; k < kShadowKeys; k += blockDim.x) run[k] = 0;
        __syncthreads();
        int key[kScatterPer], rank[kScatterPer];
#pragma unroll
        for (int e = 0; e < kScatterPer; ++e) {
            const int i = i0 + e * int(blockDim.x) + int(threadIdx.x);
            key[e] = i < n ? P.sh_key[i] : -1;
            const unsigned same = __match_any_sync(0xffffffffu, key[e]);
            const int leader = __ffs(same) - 1;
            int r = 0;
            if (lane == leader && key[e] >= 0) r = atomicAdd(run + key[e], __popc(same));
            rank[e] = __shfl_sync(0xffffffffu, r, leader) + __popc(same & ((1u << lane) - 1u));
        }
        __syncthreads();
        for (int k = threadIdx.x; k < kShadowKeys; k += blockDim.x)
            if (run[k] > 0) run[k] = atomicAdd(P.sh_cursor + k, run[k]);
        __syncthreads();
#pragma unroll
        for (int e = 0; e < kScatterPer; ++e) {
            const int i = i0 + e * int(blockDim.x) + int(threadIdx.x);
            if (key[e] >= 0) P.sh_sorted[run[key[e]] + rank[e]] = i;
        }
        __syncthreads();
    }
}

template <int ISECT, bool COUNT>
__global__ void __launch_bounds__(kTraceBlock, ATRC_TRACE_MIN_BLOCKS) k_extend(Scene S, Pool P, Counters* c,
                                                                              int sort_mode, int nkeys) {
    const int n = c->n_ext, in = c->in;
    TraceCount tc{0, 0, 0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int slot = P.q[in][i];
        const float4 o = P.ray_o[slot], d = P.ray_d[slot];
        Hit h;
        h.entity = -1;
        h.tri = -1;
        int wd = 0;
        const bool hit = trace_ray<ISECT, false, COUNT>(S, xyz(o), xyz(d), o.w, d.w, &h, &wd, &tc);
        if (wd) atomicMax(&c->watchdog, wd);
        P.hit[slot] = make_float4(h.t, h.u, h.v, __int_as_float(hit ? h.entity : -1));
        P.hit_tri[slot] = h.tri;
        if (sort_mode != ATRC_SORT_NONE) count_key(S, P, sort_mode, nkeys, i, slot, hit, h.entity);
    }
    if (COUNT) flush_count(c->cnt_closest, tc);
}

// k_extend with dynamic ray fetch (Aila and Laine 2009): persistent warps
// trace the queue round by round (Tracer::step), and whenever at least
// kRefillLanes lanes of a warp have finished their rays, those lanes take
// the next queue entries (one atomic per warp).  Lanes whose rays end early
// no longer idle until the warp's longest ray is done, which is where the
// one-ray-per-thread kernel loses most of its SIMD lanes on secondary rays.
// Results, sort keys and counts are those of k_extend.
constexpr int kRefillLanes = 16;

template <int ISECT, bool COUNT>
__global__ void __launch_bounds__(kTraceBlock, ATRC_TRACE_MIN_BLOCKS) k_extend_fetch(Scene S, Pool P, Counters* c,
                                                                                    int sort_mode, int nkeys) {
    const int n = c->n_ext, in = c->in;
    const int lane = threadIdx.x & 31;
    TraceCount tc{0, 0, 0};
    int32_t stack[kStackSize];
    Tracer<ISECT, false, COUNT> tr;
    int i = -1, slot = -1, wd = 0;
    bool drained = false;
    for (;;) {
        const unsigned idle = __ballot_sync(0xffffffffu, i < 0);
        if (!drained && __popc(idle) >= kRefillLanes) {
            int base = 0;
            if (lane == 0) base = atomicAdd(&c->ext_cursor, __popc(idle));
            base = __shfl_sync(0xffffffffu, base, 0);
            if (base + __popc(idle) >= n) drained = true;
            if (i < 0) {
                const int k = base + __popc(idle & ((1u << lane) - 1u));
                if (k < n) {
                    i = k;
                    slot = P.q[in][i];
                    const float4 o = P.ray_o[slot], d = P.ray_d[slot];
                    tr.init(S, stack, xyz(o), xyz(d), o.w, d.w);
                }
            }
        }
        if (drained && __all_sync(0xffffffffu, i < 0)) break;
        if (i >= 0 && tr.step(S, &wd, &tc)) {
            Hit h;
            h.entity = -1;
            h.tri = -1;
            h.t = h.u = h.v = 0.0f;
            const bool hit = tr.result(&h);
            P.hit[slot] = make_float4(h.t, h.u, h.v, __int_as_float(hit ? h.entity : -1));
            P.hit_tri[slot] = h.tri;
            if (sort_mode != ATRC_SORT_NONE) count_key(S, P, sort_mode, nkeys, i, slot, hit, h.entity);
            i = -1;
        }
    }
    if (wd) atomicMax(&c->watchdog, wd);
    if (COUNT) flush_count(c->cnt_closest, tc);
}

// Morton code of the 16^3 cell holding p (coordinates clamped to the grid).
__device__ __forceinline__ int shadow_cell(const Pool& P, Vec3 p) {
    const float v[3] = {p.x, p.y, p.z};
    int code = 0;
    for (int a = 0; a < 3; ++a) {
        const float x = (v[a] - P.sk_lo[a]) * P.sk_scale[a];
        const int c = min(15, max(0, int(x)));  // NaN and out-of-range origins go to the edge cells
        for (int b = 0; b < 4; ++b) code |= ((c >> b) & 1) << (3 * b + a);
    }
    return code;
}

__device__ __forceinline__ void push_shadow(Pool& P, Counters* c, Vec3 o, Vec3 d, float tmin, float tmax, Vec3 contrib,
                                            int slot) {
    const int k = warp_append(&c->n_shadow, true);
    if (k >= P.shadow_cap) { atomicMax(&c->watchdog, 4); return; }
    P.sh_o[k] = make_float4(o.x, o.y, o.z, tmin);
    P.sh_d[k] = make_float4(d.x, d.y, d.z, tmax);
    P.sh_c[k] = make_float4(contrib.x, contrib.y, contrib.z, __int_as_float(slot));
    if (P.shadow_sort) {
        const int key = shadow_cell(P, o);
        P.sh_key[k] = key;
        const unsigned same = __match_any_sync(__activemask(), key);
        if ((threadIdx.x & 31) == __ffs(same) - 1) atomicAdd(P.sh_count + key, __popc(same));
    }
}

// Materials the guide samples for: the non-delta BSDFs whose sampler
// reports the density it samples with (with disney_fixed for Disney), not
// those with subsurface scattering.
__device__ __forceinline__ bool guidable(const Material& m) {
    const int type = m.type;
    return (type == ATRC_MAT_IDEAL_DIFFUSE || type == ATRC_MAT_DISNEY || type == ATRC_MAT_METAL ||
            type == ATRC_MAT_PHONG) && m.bssrdf[1] < 0;
}

// Next-event estimation at surface vertex sv over every light
// (path_tracing.cpp:134-146, direct_illum.cpp:11-128): one light sample
// each, MIS-weighted against the BSDF-side pdf -- the guide's one-sample
// mixture where `guided` -- and pushed to the shadow queue.
__device__ __forceinline__ void nee_surface(const Scene& S, Pool& P, Counters* c, int slot, const Surface& sv,
                                            const BSDF& bv, const Entity& e, Vec3 coef, bool guided,
                                            const GuideMix& mix, Rng& rng, int* wd, float eps) {
    auto side_pdf = [&](Vec3 dir, float pb) {
        return guided ? mix.c * guide_pdf(mix, dir) + (1.0f - mix.c) * pb : pb;
    };
    for (int li = 0; li < S.light_count; ++li) {
        const int le_i = S.light_entity[li];
        const float u0 = rng.u(), u1 = rng.u(), u2 = rng.u();
        if (le_i < 0) {
            float lpdf;
            const Vec3 dir = env_sample(S, u0, u1, u2, &lpdf);
            const Vec3 rad = env_radiance(S, dir);
            if (black(rad)) continue;
            const Vec3 lpos = env_emit_pos(S, sv.pos, dir);
            const Vec3 to_light = normalize(lpos - sv.pos);
            const Vec3 bf = bsdf_eval(bv, to_light, sv.wr);
            if (black(bf)) continue;
            const Vec3 contrib = coef * rad * bf *
                                 (fabsf(cosv(to_light, sv.geo.z)) / (lpdf + side_pdf(to_light, bsdf_pdf(bv, to_light, sv.wr))));
            push_shadow(P, c, sv.pos, to_light, eps, length(sv.pos - lpos) - eps, contrib, slot);
        } else {
            const Entity& le = S.entities[le_i];
            LightSample ls;
            if (!area_light_sample(S, le, sv.pos, u0, u1, u2, &ls)) continue;
            if (black(ls.rad) || ls.pdf == 0.0f) continue;
            const float slen = length(ls.pos - sv.pos) - eps;
            if (slen <= eps) continue;
            const Vec3 to_light = normalize(ls.pos - sv.pos);
            const Vec3 bf = bsdf_eval(bv, to_light, sv.wr);
            if (black(bf)) continue;
            Vec3 tr(1.0f);
            if (S.has_media) tr = medium_tr(S, medium_of(sv, e, to_light), ls.pos, sv.pos, rng, wd);
            const Vec3 contrib = coef * tr * ls.rad * bf *
                                 (fabsf(cosv(to_light, sv.geo.z)) / (ls.pdf + side_pdf(to_light, bsdf_pdf(bv, to_light, sv.wr))));
            push_shadow(P, c, sv.pos, to_light, eps, slen, contrib, slot);
        }
    }
}

constexpr int kMaxProbeHits = 64;  // entity crossings one subsurface probe records

// SeparableBSSRDF::sample_pi (separable.cpp:107-220) of the normalized
// diffusion profile, from entry surface `s` of entity `ei`: a colour channel,
// a projection axis (the normal with 1/2, each tangent with 1/4) and a
// radius r ~ p(r / d); the probe segment through the sphere of radius
// r_max = P^-1(0.996) d crosses the entity at every point it meets, and one
// crossing is kept uniformly.  On success *x is the exit point, *bx its
// separable BSDF and *w = (1 - Fr(cos wo)) eval_r(|x - s|) / pdf.
// Inlined: as a real call its outputs and the caller's live state took a
// 2.4 KB local-memory frame per thread, and k_subsurface wrote 2.5 GB of it
// to DRAM per launch on the 1024^2 subsurface Cornell box (now a 400-byte
// frame, the traversal stack: the workload runs 1.28x faster).
__device__ __forceinline__ bool subsurface_sample(const Scene& S, const Material& m, const Surface& s, Rng& rng, int* wd, float eps,
                                  Surface* x, BSDF* bx, Vec3* w) {
    const Vec3 A = tex2d_sample(S, m.bssrdf[0], s.u, s.v);
    const Vec3 dmfp = tex2d_sample(S, m.bssrdf[1], s.u, s.v);
    const float eta = tex2d_sample(S, m.bssrdf[2], s.u, s.v).x;
    const float dch[3] = {dmfp.x / nd_scale(A.x), dmfp.y / nd_scale(A.y), dmfp.z / nd_scale(A.z)};
    const float u0 = rng.u(), u1 = rng.u(), u2 = rng.u();
    const int ch = min(int(u0 * 3.0f), 2);  // extract_uniform_int
    const float su = u0 * 3.0f - float(ch);
    Coord proj;
    float sv;
    if (u1 < 0.5f) {
        proj = s.geo;
        sv = 2.0f * u1;
    } else if (u1 < 0.75f) {
        proj = Coord{s.geo.y, s.geo.z, s.geo.x};
        sv = 4.0f * (u1 - 0.5f);
    } else {
        proj = Coord{s.geo.z, s.geo.x, s.geo.y};
        sv = 4.0f * (u1 - 0.75f);
    }
    const float r = nd_inv_cdf(su) * dch[ch];
    const float r_max = nd_inv_cdf(0.996f) * dch[ch];
    if (!(r > 0.0f) || r > r_max) return false;
    float sp, cp;
    sincosf(2.0f * kPi * sv, &sp, &cp);
    const float hl = sqrtf(fmaxf(0.0f, r_max * r_max - r * r));
    Vec3 o = s.pos + proj.local_to_global(Vec3(r * cp, r * sp, hl));
    const Vec3 dir = -proj.z;
    float tmax = fmaxf(eps, 2.0f * hl);
    int cnt = 0;
    Hit pick{};
    Vec3 pick_o;
    for (int k = 0; k < kMaxProbeHits && eps < tmax; ++k) {
        Hit h;
        if (!trace_entity<false>(S, s.entity, o, dir, eps, tmax, &h, wd)) break;
        ++cnt;
        if (rng.u() * float(cnt) < 1.0f) {  // reservoir: each crossing kept with probability 1 / cnt
            pick = h;
            pick_o = o;
        }
        o = o + dir * (h.t + eps);
        tmax -= h.t + eps;
    }
    (void)u2;
    if (cnt == 0) return false;
    *x = make_surface(S, pick, pick_o, dir);
    // pdf_pi (separable.cpp:222-248): all three axes and channels
    const Vec3 ld = s.geo.global_to_local(s.pos - x->pos);
    const Vec3 ln = s.geo.global_to_local(x->geo.z);
    const float rp[3] = {sqrtf(ld.y * ld.y + ld.z * ld.z), sqrtf(ld.z * ld.z + ld.x * ld.x),
                         sqrtf(ld.x * ld.x + ld.y * ld.y)};
    const float lnc[3] = {ln.x, ln.y, ln.z};
    const float axis_pdf[3] = {0.25f, 0.25f, 0.5f};
    float pr = 0.0f;
    for (int a = 0; a < 3; ++a)
        for (int c = 0; c < 3; ++c) pr += fabsf(lnc[a]) * nd_pdf_r(dch[c], rp[a]) * axis_pdf[a];
    pr *= 1.0f / 3.0f;
    const float pdf = pr / (2.0f * kPi) / float(cnt);
    if (!(pdf > 0.0f)) return false;
    const float fro = 1.0f - dielectric_fresnel(eta, 1.0f, cosv(s.wr, s.geo.z));
    *w = fro * nd_eval_r(A, Vec3(dch[0], dch[1], dch[2]), length(x->pos - s.pos)) / pdf;
    BSDF b{};
    b.type = kMatSeparable;
    b.geo = x->geo;
    b.shd = x->geo;
    b.IOR = eta;
    b.sep_ci = 1.0f - 2.0f * fresnel_moment1(1.0f / eta);
    b.eps = eps;
    *bx = b;
    return true;
}

// Guide queries of the shade queue (same order as k_shade): surface hits
// with a Lambert or Disney material, consistent frames and a depth the guide
// serves are appended to a compact query list; gidx[i] is the query of
// shade-queue entry i, or -1.
__global__ void k_guide_features(Scene S, Params p, Pool P, Counters* c) {
    const int n = c->n_ext, in = c->in;
    const int* queue = p.sort_mode != ATRC_SORT_NONE ? P.q_sorted : P.q[in];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int slot = queue[i];
        GuideQuery q;
        q.slot = -1;
        q.pad = 0;
        const float4 hv = P.hit[slot];
        const int ent = __float_as_int(hv.w);
        const int4 ct = P.ctr[slot];
        const int flags = ct.w & 0xff;
        if (ent >= 0 && !(flags & PF_TERMINATE) && (p.gf.max_depth <= 0 || ct.x <= p.gf.max_depth)) {
            const float4 ro = P.ray_o[slot], rd = P.ray_d[slot];
            Hit h;
            h.t = hv.x; h.u = hv.y; h.v = hv.z; h.entity = ent; h.tri = P.hit_tri[slot];
            const Surface s = make_surface(S, h, xyz(ro), xyz(rd));
            Vec3 sn;
            const BSDF b = shade(S, s, &sn);
            if (guidable(S.materials[S.entities[ent].material]) && !fringes(b, s.wr)) {
                q.pos[0] = s.pos.x; q.pos[1] = s.pos.y; q.pos[2] = s.pos.z;
                q.nrm[0] = sn.x; q.nrm[1] = sn.y; q.nrm[2] = sn.z;
                q.wo[0] = s.wr.x; q.wo[1] = s.wr.y; q.wo[2] = s.wr.z;
                q.rough = b.type == ATRC_MAT_DISNEY || b.type == ATRC_MAT_METAL ? b.roughness : 1.0f;
                q.slot = slot;
            }
        }
        const int k = warp_append(&c->n_guide, q.slot >= 0);
        if (q.slot >= 0) {
            p.gf.queries[k] = q;
            write_inputs<__half>(p.gf.grid, p.gf.table_h, q, k % kGuideTile,
                                 p.gf.xtiles + size_t(k / kGuideTile) * kGuideTileBytes, nullptr);
        }
        p.gf.gidx[i] = q.slot >= 0 ? k : -1;
    }
}

__global__ void __launch_bounds__(128, ATRC_SHADE_MIN_BLOCKS) k_shade(Scene S, Params p, Pool P, Counters* c) {
    const int n = c->n_ext, in = c->in, out = c->out;
    const float eps = p.eps;
    const int* queue = p.sort_mode != ATRC_SORT_NONE ? P.q_sorted : P.q[in];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int slot = queue[i];
        int4 ct = P.ctr[slot];
        int depth = ct.x, s_depth = ct.y, scat = ct.z, flags = ct.w & 0xff, ray_med = ct.w >> 8;
        uint4 st = P.st[slot];
        Rng rng = load_rng(st);
        const float4 ro = P.ray_o[slot], rd = P.ray_d[slot];
        const Vec3 o = xyz(ro), d = xyz(rd);
        const float4 hv = P.hit[slot];
        const int ent = __float_as_int(hv.w);
        float4 coef4 = P.coef[slot];
        Vec3 coef = xyz(coef4);
        float4 L4 = P.L[slot];
        Vec3 L = xyz(L4);
        float4 mf4 = P.mis_f[slot];
        int wd = 0;
        bool finish = false, cont = false, subsurface = false;
        if (flags & PF_REC_PENDING) {
            // radiance gathered up to this vertex: the previous record's
            // incident radiance is what the path brings back from here on
            GuideRecord* r = p.gf.records + p.gf.record_last[slot];
            r->l_arrive[0] = L.x; r->l_arrive[1] = L.y; r->l_arrive[2] = L.z;
            flags &= ~PF_REC_PENDING;
        }
        Surface s;
        bool have_surface = false;
        if (ent >= 0) {
            Hit h;
            h.t = hv.x; h.u = hv.y; h.v = hv.z; h.entity = ent; h.tri = P.hit_tri[slot];
            s = make_surface(S, h, o, d);
            have_surface = true;
        }
        if (p.renderer == ATRC_RENDERER_AO) {
            // trace_ao (path_tracing.cpp:383-415): the pixel is
            // lerp(low, high, unblocked fraction); it starts at `low` and each
            // unblocked occlusion ray adds (high - low) / count in k_shadow
            if (!have_surface) {
                L = Vec3(p.ao_bg[0], p.ao_bg[1], p.ao_bg[2]);
            } else {
                const Entity& e = S.entities[ent];
                P.gb_albedo[slot] = make_float4(p.ao_high[0], p.ao_high[1], p.ao_high[2],
                                                (e.flags & ENT_NO_DENOISE) ? 0.0f : 1.0f);
                P.gb_normal[slot] = make_float4(s.geo.z.x, s.geo.z.y, s.geo.z.z, 0);
                L = Vec3(p.ao_low[0], p.ao_low[1], p.ao_low[2]);
                const Vec3 step = (Vec3(p.ao_high[0], p.ao_high[1], p.ao_high[2]) - L) / float(p.ao_count);
                const Vec3 start = eps_offset(s, s.geo.z, eps);
                for (int k = 0; k < p.ao_count; ++k) {
                    const float u = rng.u(), v = rng.u();
                    float pdf;
                    const Vec3 dir = normalize(s.geo.local_to_global(zweighted_on_hemisphere(u, v, &pdf)));
                    // Scene::visible(start, end): segment trimmed by eps at both ends
                    const Vec3 seg = (start + dir * p.ao_dist) - start;
                    const float dis = length(seg);
                    push_shadow(P, c, start, normalize(seg), eps, dis - eps, step, slot);
                }
            }
            store_rng(st, rng);
            P.st[slot] = st;
            P.L[slot] = make_float4(L.x, L.y, L.z, L4.w);
            const int fi = warp_append(&c->n_finish, true);
            P.q_finish[fi] = slot;
            continue;
        }
        // (1) pending MIS-BSDF term of the previous vertex (direct_illum.cpp:130-192)
        if (flags & PF_MIS) {
            const Vec3 mis_f = xyz(mf4);
            const float mis_pdf = coef4.w;
            if (!have_surface) {
                if (S.env.type != ATRC_ENV_NONE) {
                    const Vec3 le = env_radiance(S, d);
                    if (!black(le)) L += mis_f * le / ((flags & PF_MIS_DELTA) ? mis_pdf : mis_pdf + env_pdf(S, d));
                }
            } else {
                const Entity& e = S.entities[ent];
                if (e.flags & ENT_LIGHT) {
                    const Vec3 le = area_light_radiance(e, s.geo.z, s.wr);
                    if (!black(le)) {
                        const Vec3 tr = medium_tr(S, ray_med, o, s.pos, rng, &wd);
                        const Vec3 f = tr * le * mis_f;
                        L += (flags & PF_MIS_DELTA) ? f / mis_pdf : f / (mis_pdf + area_light_pdf(S, e, o, s.pos, s.geo.z));
                    }
                }
            }
            flags &= ~(PF_MIS | PF_MIS_DELTA);
        }
        if ((flags & PF_TERMINATE) || depth > p.max_depth) finish = true;
        // (2) Russian roulette (path_tracing.cpp:30-35)
        if (!finish && depth > p.min_depth) {
            if (rng.u() > p.cont_prob) finish = true;
            else coef = coef / p.cont_prob;
        }
        if (!finish && !have_surface) {
            if (depth == 1 && S.env.type != ATRC_ENV_NONE) L += coef * env_radiance(S, d);
            finish = true;
        }
        if (!finish) {
            const Entity& e = S.entities[ent];
            Vec3 sn;
            const BSDF b = shade(S, s, &sn);
            if (depth == 1) {
                const Vec3 alb = bsdf_albedo(b);
                P.gb_albedo[slot] = make_float4(alb.x, alb.y, alb.z, (e.flags & ENT_NO_DENOISE) ? 0.0f : 1.0f);
                P.gb_normal[slot] = make_float4(sn.x, sn.y, sn.z, 0);
            }
            bool scattered = false;
            Vec3 spos, swr;
            Phase ph;
            int med = dot(s.wr, s.geo.z) >= 0 ? e.med_out : e.med_in;
            if (S.has_media) {
                if (scat < S.media[med].max_scattering_count) {
                    Vec3 tp;
                    scattered = medium_sample(S, med, o, s.pos, scat > 0, rng, &tp, &spos, &swr, &ph, &wd);
                    coef *= tp;
                } else {
                    coef *= medium_ab(S, med, o, s.pos, rng, &wd);
                }
            }
            if (scattered) {
                // medium vertex (path_tracing.cpp:73-104)
                ++scat;
                for (int li = 0; li < S.light_count; ++li) {
                    const int le_i = S.light_entity[li];
                    if (le_i < 0) continue;  // env NEE from a medium point is 0 (direct_illum.cpp:101-108)
                    LightSample ls;
                    const float u0 = rng.u(), u1 = rng.u(), u2 = rng.u();
                    if (!area_light_sample(S, S.entities[le_i], spos, u0, u1, u2, &ls)) continue;
                    if (black(ls.rad) || ls.pdf == 0.0f) continue;
                    const Vec3 to_light = normalize(ls.pos - spos);
                    const float fph = hg_pdf(ph, to_light, swr);
                    if (fph == 0.0f) continue;
                    const Vec3 tr = medium_tr(S, med, spos, ls.pos, rng, &wd);
                    const Vec3 contrib = coef * tr * ls.rad * fph / (ls.pdf + fph);
                    const float dis = length(ls.pos - spos);
                    push_shadow(P, c, ls.pos, normalize(spos - ls.pos), eps, dis - eps, contrib, slot);
                }
                const BSDFSample bs = hg_sample(ph, swr, rng.u(), rng.u());
                if (black(bs.f)) {
                    finish = true;
                } else {
                    const Vec3 dir = normalize(bs.dir);
                    mf4 = make_float4(coef.x * bs.f.x, coef.y * bs.f.y, coef.z * bs.f.z, mf4.w);
                    coef4.w = bs.pdf;
                    flags |= PF_MIS;
                    ray_med = med;
                    if (bs.pdf < eps) flags |= PF_TERMINATE;
                    else coef = coef * bs.f / bs.pdf;
                    P.ray_o[slot] = make_float4(spos.x, spos.y, spos.z, 0.0f);
                    P.ray_d[slot] = make_float4(dir.x, dir.y, dir.z, INFINITY);
                    ++depth;
                    cont = true;
                }
            } else {
                scat = 0;
                // learned guide of this vertex (one-sample MIS with the BSDF)
                GuideMix mix;
                bool guided = false;
                const int gq_i = p.guide_on ? p.gf.gidx[i] : -1;
                if (gq_i >= 0) {
                    const float* gm = p.gf.mixes + size_t(gq_i) * kGuideOut;
                    guided = guidable(S.materials[e.material]) && !fringes(b, s.wr);
                    if (guided) {
                        for (int k = 0; k < kGuideLobes; ++k) {
                            mix.mu[k][0] = gm[5 * k]; mix.mu[k][1] = gm[5 * k + 1]; mix.mu[k][2] = gm[5 * k + 2];
                            mix.kappa[k] = gm[5 * k + 3];
                            mix.w[k] = gm[5 * k + 4];
                        }
                        mix.c = gm[kGuideUsed - 1];
                    }
                }
                // pdf of the BSDF-side strategy (BSDF or guide) for a direction
                auto side_pdf = [&](Vec3 dir, float pb) {
                    return guided ? mix.c * guide_pdf(mix, dir) + (1.0f - mix.c) * pb : pb;
                };
                if (depth == 1 && (e.flags & ENT_LIGHT)) L += coef * area_light_radiance(e, s.geo.z, s.wr);
                // next-event estimation over every light (path_tracing.cpp:134-146)
                nee_surface(S, P, c, slot, s, b, e, coef, guided, mix, rng, &wd, eps);
                // BSDF sample: MIS-BSDF ray and continuation (path_tracing.cpp:148-169)
                BSDFSample bs;
                float pdf_bsdf = 0.0f;
                if (guided) {
                    // one-sample MIS: the guide with probability c, else the BSDF
                    if (rng.u() < mix.c) {
                        const float g0 = rng.u(), g1 = rng.u(), g2 = rng.u();
                        bs.dir = guide_sample(mix, g0, g1, g2);
                        bs.f = bsdf_eval(b, bs.dir, s.wr);
                        pdf_bsdf = bsdf_pdf(b, bs.dir, s.wr);
                    } else {
                        const float u0 = rng.u(), u1 = rng.u(), u2 = rng.u();
                        bs = bsdf_sample(b, s.wr, u0, u1, u2);
                        pdf_bsdf = bs.pdf;
                    }
                    bs.delta = false;
                    bs.pdf = side_pdf(bs.dir, pdf_bsdf);
                } else {
                    const float u0 = rng.u(), u1 = rng.u(), u2 = rng.u();
                    bs = bsdf_sample(b, s.wr, u0, u1, u2);
                }
                if (black(bs.f) || (guided && !(bs.pdf > 0.0f))) {
                    finish = true;
                } else {
                    // training record of this vertex, kept with probability
                    // record_keep so that a pass's records sample all its
                    // guided vertices (every depth, every pixel) rather than
                    // the first record_cap of them; targets are set when the
                    // path ends
                    bool keep = false;
                    if (guided && p.gf.records) {
                        atomicAdd(p.gf.record_count + 1, 1);
                        keep = p.gf.record_keep >= 1.0f || rng.u() < p.gf.record_keep;
                    }
                    if (keep) {
                        const int r = atomicAdd(p.gf.record_count, 1);
                        if (r < p.gf.record_cap) {
                            const GuideQuery& gq = p.gf.queries[gq_i];
                            GuideRecord R;
                            for (int k = 0; k < 3; ++k) { R.pos[k] = gq.pos[k]; R.nrm[k] = gq.nrm[k]; R.wo[k] = gq.wo[k]; }
                            R.rough = gq.rough;
                            R.wi[0] = bs.dir.x; R.wi[1] = bs.dir.y; R.wi[2] = bs.dir.z;
                            R.pdf_bsdf = pdf_bsdf;
                            R.coef[0] = coef.x; R.coef[1] = coef.y; R.coef[2] = coef.z;
                            R.target = 0.0f;
                            R.l_arrive[0] = R.l_arrive[1] = R.l_arrive[2] = 0.0f;
                            R.prev = p.gf.record_last[slot];
                            R.pad[0] = R.pad[1] = 0.0f;
                            p.gf.records[r] = R;
                            p.gf.record_last[slot] = r;
                            flags |= PF_REC_PENDING;
                        }
                    }
                    // subsurface scattering (path_tracing.cpp:173-221): a
                    // direction into the surface re-emerges at a probed exit
                    // point; the walk runs in k_subsurface.  The entry's
                    // MIS-BSDF term is the continuation's, which re-emerges
                    // instead: exact while the inside of the object holds
                    // no light.
                    if (S.has_subsurface && S.materials[e.material].bssrdf[1] >= 0 && bs.pdf >= eps &&
                        !s.geo.positive(bs.dir) && s.geo.positive(s.wr)) {
                        coef = coef * bs.f * (fabsf(cosv(s.geo.z, bs.dir)) / bs.pdf);
                        subsurface = true;
                    }
                }
                if (!finish && !subsurface) {
                    const Vec3 dir = normalize(bs.dir);
                    const float gcos = fabsf(dot(s.geo.z, dir));
                    mf4 = make_float4(coef.x * bs.f.x * gcos, coef.y * bs.f.y * gcos, coef.z * bs.f.z * gcos, mf4.w);
                    coef4.w = bs.pdf;
                    flags |= PF_MIS | (bs.delta ? PF_MIS_DELTA : 0);
                    ray_med = medium_of(s, e, dir);
                    if (bs.pdf < eps) flags |= PF_TERMINATE;
                    else coef = coef * bs.f * (fabsf(cosv(s.geo.z, bs.dir)) / bs.pdf);
                    const Vec3 no = eps_offset(s, bs.dir, eps);
                    P.ray_o[slot] = make_float4(no.x, no.y, no.z, 0.0f);
                    P.ray_d[slot] = make_float4(dir.x, dir.y, dir.z, INFINITY);
                    if (!(bs.delta && depth >= 2 && s_depth <= p.specular_depth)) ++depth;
                    else ++s_depth;
                    cont = true;
                }
            }
        }
        if (wd) atomicMax(&c->watchdog, wd);
        store_rng(st, rng);
        P.st[slot] = st;
        P.coef[slot] = make_float4(coef.x, coef.y, coef.z, coef4.w);
        P.L[slot] = make_float4(L.x, L.y, L.z, L4.w);
        P.mis_f[slot] = mf4;
        P.ctr[slot] = make_int4(depth, s_depth, scat, (flags & 0xff) | (ray_med << 8));
        const int qi = warp_append(&c->n_next, cont);
        if (cont) {
            if (p.slot_queue) P.slot_state[slot] = kSlotCont;
            else P.q[out][qi] = slot;
        }
        if (S.has_subsurface) {
            const int si = warp_append(&c->n_sss, subsurface);
            if (subsurface) P.q_sss[si] = slot;
        }
        const bool ends = !cont && !subsurface;
        const int fi = warp_append(&c->n_finish, ends);
        if (ends) P.q_finish[fi] = slot;
    }
}

// Subsurface walks queued by k_shade (path_tracing.cpp:173-221): the probe
// from the entry point, light samples at the exit point with its separable
// BSDF, and the exit's BSDF sample that continues the path (its MIS-BSDF
// term pending like every other vertex).  Paths end here when the probe
// finds no exit or the exit sample is black.
__global__ void __launch_bounds__(128) k_subsurface(Scene S, Params p, Pool P, Counters* c) {
    const int n = c->n_sss, out = c->out;
    const float eps = p.eps;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int slot = P.q_sss[i];
        const int4 ct = P.ctr[slot];
        int depth = ct.x, flags = ct.w & 0xff, ray_med = ct.w >> 8;
        uint4 st = P.st[slot];
        Rng rng = load_rng(st);
        const float4 ro = P.ray_o[slot], rd = P.ray_d[slot], hv = P.hit[slot];
        Hit h;
        h.t = hv.x; h.u = hv.y; h.v = hv.z; h.entity = __float_as_int(hv.w); h.tri = P.hit_tri[slot];
        const Surface s = make_surface(S, h, xyz(ro), xyz(rd));
        const Entity& e = S.entities[h.entity];
        float4 coef4 = P.coef[slot];
        Vec3 coef = xyz(coef4);
        float4 mf4 = P.mis_f[slot];
        int wd = 0;
        bool cont = false;
        Surface x;
        BSDF bx;
        Vec3 w;
        if (subsurface_sample(S, S.materials[e.material], s, rng, &wd, eps, &x, &bx, &w)) {
            coef = coef * w;
            GuideMix none;
            nee_surface(S, P, c, slot, x, bx, e, coef, false, none, rng, &wd, eps);
            const float u0 = rng.u(), u1 = rng.u(), u2 = rng.u();
            const BSDFSample bs = bsdf_sample(bx, x.wr, u0, u1, u2);
            if (!black(bs.f)) {
                const Vec3 dir = normalize(bs.dir);
                const float gcos = fabsf(dot(x.geo.z, dir));
                mf4 = make_float4(coef.x * bs.f.x * gcos, coef.y * bs.f.y * gcos, coef.z * bs.f.z * gcos, mf4.w);
                coef4.w = bs.pdf;
                flags |= PF_MIS;
                ray_med = medium_of(x, e, dir);
                if (bs.pdf < eps) flags |= PF_TERMINATE;
                else coef = coef * bs.f * (fabsf(cosv(x.geo.z, bs.dir)) / bs.pdf);
                const Vec3 no = eps_offset(x, bs.dir, eps);
                P.ray_o[slot] = make_float4(no.x, no.y, no.z, 0.0f);
                P.ray_d[slot] = make_float4(dir.x, dir.y, dir.z, INFINITY);
                ++depth;
                cont = true;
            }
        }
        if (wd) atomicMax(&c->watchdog, wd);
        store_rng(st, rng);
        P.st[slot] = st;
        P.coef[slot] = make_float4(coef.x, coef.y, coef.z, coef4.w);
        P.mis_f[slot] = mf4;
        P.ctr[slot] = make_int4(depth, ct.y, ct.z, (flags & 0xff) | (ray_med << 8));
        const int qi = warp_append(&c->n_next, cont);
        if (cont) {
            if (p.slot_queue) P.slot_state[slot] = kSlotCont;
            else P.q[out][qi] = slot;
        }
        const int fi = warp_append(&c->n_finish, !cont);
        if (!cont) P.q_finish[fi] = slot;
    }
}

template <int ISECT, bool COUNT>
__global__ void __launch_bounds__(kTraceBlock, ATRC_SHADOW_MIN_BLOCKS) k_shadow(Scene S, Pool P, Counters* c) {
    const int n = min(c->n_shadow, P.shadow_cap);
    TraceCount tc{0, 0, 0};
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        const int i = P.shadow_sort ? P.sh_sorted[j] : j;
        const float4 o = P.sh_o[i], d = P.sh_d[i];
        Hit h;
        int wd = 0;
        const bool occluded = trace_ray<ISECT, true, COUNT>(S, xyz(o), xyz(d), o.w, d.w, &h, &wd, &tc);
        if (wd) atomicMax(&c->watchdog, wd);
        if (!occluded) {
            const float4 cc = P.sh_c[i];
            const int slot = __float_as_int(cc.w);
            float* l = reinterpret_cast<float*>(P.L + slot);
            atomicAdd(l, cc.x);
            atomicAdd(l + 1, cc.y);
            atomicAdd(l + 2, cc.z);
        }
    }
    if (COUNT) flush_count(c->cnt_shadow, tc);
}

// k_shadow with dynamic ray fetch, as k_extend_fetch: persistent warps
// step their any-hit traversals round by round and refill the lanes whose
// rays are done (occluded at the first hit, or through the scene) from the
// shadow queue.  Contributions and counts are those of k_shadow.
template <int ISECT, bool COUNT>
__global__ void __launch_bounds__(kTraceBlock, ATRC_TRACE_MIN_BLOCKS) k_shadow_fetch(Scene S, Pool P, Counters* c) {
    const int n = min(c->n_shadow, P.shadow_cap);
    const int lane = threadIdx.x & 31;
    TraceCount tc{0, 0, 0};
    int32_t stack[kStackSize];
    Tracer<ISECT, true, COUNT> tr;
    int i = -1, wd = 0;
    bool drained = false;
    for (;;) {
        const unsigned idle = __ballot_sync(0xffffffffu, i < 0);
        if (!drained && __popc(idle) >= kRefillLanes) {
            int base = 0;
            if (lane == 0) base = atomicAdd(&c->sh_cursor, __popc(idle));
            base = __shfl_sync(0xffffffffu, base, 0);
            if (base + __popc(idle) >= n) drained = true;
            if (i < 0) {
                const int k = base + __popc(idle & ((1u << lane) - 1u));
                if (k < n) {
                    i = P.shadow_sort ? P.sh_sorted[k] : k;
                    const float4 o = P.sh_o[i], d = P.sh_d[i];
                    tr.init(S, stack, xyz(o), xyz(d), o.w, d.w);
                }
            }
        }
        if (drained && __all_sync(0xffffffffu, i < 0)) break;
        if (i >= 0 && tr.step(S, &wd, &tc)) {
            Hit h;
            if (!tr.result(&h)) {
                const float4 cc = P.sh_c[i];
                float* l = reinterpret_cast<float*>(P.L + __float_as_int(cc.w));
                atomicAdd(l, cc.x);
                atomicAdd(l + 1, cc.y);
                atomicAdd(l + 2, cc.z);
            }
            i = -1;
        }
    }
    if (wd) atomicMax(&c->watchdog, wd);
    if (COUNT) flush_count(c->cnt_shadow, tc);
}

__device__ __forceinline__ float filter_eval(const View& p, float x, float y) {
    if (p.filter_type == ATRC_FILTER_BOX) return p.filter_value;
    const float gx = fmaxf(0.0f, __expf(-p.filter_alpha * x * x) - p.filter_exp);
    const float gy = fmaxf(0.0f, __expf(-p.filter_alpha * y * y) - p.filter_exp);
    return gx * gy;
}

__global__ void k_finish(Params p, Pool P, Counters* c) {
    const int n = c->n_finish;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int slot = P.q_finish[i];
        const float4 L = P.L[slot];
        const float sx = L.w, sy = P.mis_f[slot].w;
        const uint32_t vt = P.st[slot].w;
        const int vi = int(vt >> kTileBits), tile = int(vt & ((1u << kTileBits) - 1u));
        const View& v = p.views[vi];
        const Film& F = v.film;
        if (p.view_done) {  // one atomic per view present in the warp
            const unsigned same = __match_any_sync(__activemask(), vi);
            if (int(threadIdx.x & 31) == __ffs(same) - 1) {
                const unsigned long long k = (unsigned long long)__popc(same);
                const unsigned long long before = atomicAdd(p.view_done + vi, k);
                // the one add that completes the view stamps its time
                if (p.view_time && before < v.count && before + k >= v.count) p.view_time[vi] = global_ns();
            }
        }
        if (p.gf.records) {
            // targets of the path's guide records: luminance of the radiance
            // gathered after each vertex over the throughput arriving at it,
            // i.e. f cos L_i / pdf of the sampled direction
            int r = p.gf.record_last[slot];
            for (int k = 0; r >= 0 && k < 256; ++k) {
                GuideRecord& R = p.gf.records[r];
                float t = 0.0f;
                for (int ch = 0; ch < 3; ++ch) {
                    const float lc = (ch == 0 ? L.x : ch == 1 ? L.y : L.z) - R.l_arrive[ch];
                    const float w = ch == 0 ? 0.2126f : ch == 1 ? 0.7152f : 0.0722f;
                    if (R.coef[ch] > 0.0f) t += w * fmaxf(lc, 0.0f) / R.coef[ch];
                }
                R.target = isfinite(t) ? t : 0.0f;
                r = R.prev;
            }
            p.gf.record_last[slot] = -1;
        }
        if (isfinite(L.x) && isfinite(L.y) && isfinite(L.z)) {
            const float4 ga = P.gb_albedo[slot], gn = P.gb_normal[slot];
            // apply_image_filter (framebuffer.h:49-80) over the sample's tile;
            // the distances step by one pixel from the tile-clamped start
            const int tx0 = (tile % v.TX) * v.G, ty0 = (tile / v.TX) * v.G;
            const int tx1 = min(v.W, tx0 + v.G) - 1, ty1 = min(v.H, ty0 + v.G) - 1;
            const float r = v.filter_radius;
            const int x0 = max(tx0, int(ceilf(sx - r - 0.5f))), y0 = max(ty0, int(ceilf(sy - r - 0.5f)));
            const int x1 = min(tx1, int(floorf(sx + r - 0.5f))), y1 = min(ty1, int(floorf(sy + r - 0.5f)));
            float yrel = fabsf(y0 + 0.5f - sy);
            for (int y = y0; y <= y1; ++y, yrel += 1) {
                if (yrel > r) continue;
                float xrel = fabsf(x0 + 0.5f - sx);
                for (int x = x0; x <= x1; ++x, xrel += 1) {
                    if (xrel > r) continue;
                    const double w = filter_eval(v, xrel, yrel);
                    const size_t px = size_t(y) * v.W + x;
                    atomicAdd(F.value + 3 * px, w * L.x);
                    atomicAdd(F.value + 3 * px + 1, w * L.y);
                    atomicAdd(F.value + 3 * px + 2, w * L.z);
                    atomicAdd(F.weight + px, w);
                    if (F.value_sq) {
                        atomicAdd(F.value_sq + 3 * px, w * double(L.x) * L.x);
                        atomicAdd(F.value_sq + 3 * px + 1, w * double(L.y) * L.y);
                        atomicAdd(F.value_sq + 3 * px + 2, w * double(L.z) * L.z);
                    }
                    if (F.albedo) {
                        atomicAdd(F.albedo + 3 * px, w * ga.x);
                        atomicAdd(F.albedo + 3 * px + 1, w * ga.y);
                        atomicAdd(F.albedo + 3 * px + 2, w * ga.z);
                    }
                    if (F.normal) {
                        atomicAdd(F.normal + 3 * px, w * gn.x);
                        atomicAdd(F.normal + 3 * px + 1, w * gn.y);
                        atomicAdd(F.normal + 3 * px + 2, w * gn.z);
                    }
                    if (F.denoise) atomicAdd(F.denoise + px, w * ga.w);
                }
            }
        }
        P.slot_state[slot] = kSlotFree;
    }
}

int grid_for(int sm_count, int blocks_per_sm) { return std::max(1, sm_count * blocks_per_sm); }

// Stream capture scope: ends the capture (and drops the partial graph) if
// anything throws before end() is called, so the stream never stays in
// capture mode.
struct CaptureGuard {
    cudaStream_t s;
    bool open = true;
    explicit CaptureGuard(cudaStream_t st) : s(st) { CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal)); }
    cudaGraph_t end() {
        cudaGraph_t g = nullptr;
        open = false;
        CK(cudaStreamEndCapture(s, &g));
        return g;
    }
    ~CaptureGuard() {
        if (!open) return;
        cudaGraph_t g = nullptr;
        cudaStreamEndCapture(s, &g);
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
    }
};

// Capture of a stream's work into an existing graph (the body of a
// conditional node); ends the capture on scope exit if end() was not reached.
struct BodyCapture {
    cudaStream_t s;
    bool open = false;
    BodyCapture(cudaStream_t st, cudaGraph_t body) : s(st) {
        CK(cudaStreamBeginCaptureToGraph(s, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
        open = true;
    }
    void end() {
        open = false;
        cudaGraph_t g = nullptr;
        CK(cudaStreamEndCapture(s, &g));
    }
    ~BodyCapture() {
        if (!open) return;
        cudaGraph_t g = nullptr;
        cudaStreamEndCapture(s, &g);
        cudaGetLastError();
    }
};

// Reuse an executable graph when the new graph has the same topology (only
// kernel parameters differ); otherwise instantiate afresh.
cudaGraphExec_t instantiate_or_update(cudaGraphExec_t exec, cudaGraph_t g) {
    if (exec) {
        cudaGraphExecUpdateResultInfo info;
        if (cudaGraphExecUpdate(exec, g, &info) == cudaSuccess) return exec;
        cudaGetLastError();
        cudaGraphExecDestroy(exec);
    }
    cudaGraphExec_t out = nullptr;
    CK(cudaGraphInstantiate(&out, g, 0));
    return out;
}

}  // namespace

// ==================================================================== scene
struct DeviceSceneImpl {
    int device = 0;
    int sm_count = 148;
    cudaStream_t stream = nullptr;
    Scene scene{};
    DevBuf nodes, tris, tri_bc, tri_shade, tri_orig, entities, tlas_order, materials, tex2d, tex3d, texels, media, alias_prob,
        alias_idx, env_probs, env_alias_prob, env_alias_idx;
    DevBuf watchdog;
    DevBuf tiles;  // tile tables of the film's sample grid
    // render workspace (kept between calls)
    DevBuf pool_buf, counters, film_buf;
    // per-call resources kept between render calls
    static constexpr int kWindow = 4;  // wavefront iterations between host checks
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, kev[kWindow * 4] = {};
    static constexpr int kCopyChunks = 16;  // host-film download in pieces
    cudaEvent_t copy_ev[kCopyChunks] = {};
    void* pinned_counters = nullptr;
    DevBuf views_buf;                   // view table (+ per-view completion counters)
    void* view_stage = nullptr;         // pinned copy of the completion counters
    size_t view_stage_bytes = 0;
    void ensure_view_stage(size_t bytes) {
        if (view_stage_bytes >= bytes) return;
        if (view_stage) cudaFreeHost(view_stage);
        view_stage = nullptr;
        view_stage_bytes = 0;
        CK(cudaMallocHost(&view_stage, bytes));
        view_stage_bytes = bytes;
    }
    cudaGraphExec_t window_exec = nullptr;  // the captured bounce-loop window
    cudaGraphExec_t loop_exec = nullptr;    // the device-side bounce loop (batches)
    void* stage = nullptr;             // pinned host staging for host films
    size_t stage_bytes = 0;
    // launch configuration (atrc_cuda_autotune chooses it; these are the
    // defaults): ATRC_SORT_AUTO resolves to tuned_sort, path_pool 0 to
    // tuned_pool; k_generate / k_finish use the grid and block shapes
    int tuned_sort = ATRC_SORT_NONE;
    int tuned_pool = 1 << 21;
    int tuned_gen_blocks = 16;    // k_generate / k_finish blocks per SM
    int tuned_gen_threads = 256;  // k_generate block
    int tuned_fin_threads = 128;  // k_finish block
    int tuned_fetch = 0;          // k_extend_fetch instead of k_extend
    int tuned_queue = 0;          // extend queue in slot order (1) or shade order (0)
    int tuned_shadow_fetch = 0;   // k_shadow_fetch instead of k_shadow
    int tuned_shadow_sort = 0;    // shadow queue in origin-cell order
    int tuned_trials = 0;
    double tuned_ms = 0, default_ms = 0;
    DevBuf tune_film;
    void resolve_sort(Params* p, int requested) const {
        p->sort_mode = requested == ATRC_SORT_AUTO ? tuned_sort : requested;
        p->slot_queue = tuned_queue;
        p->nkeys = std::max(scene.material_count, kMaterialTypes) + 2;
    }
    void ensure_render_resources() {
        if (!ev0) {
            CK(cudaEventCreate(&ev0));
            CK(cudaEventCreate(&ev1));
            for (auto& e : kev) CK(cudaEventCreate(&e));
            for (auto& e : copy_ev) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        }
        if (!pinned_counters) CK(cudaMallocHost(&pinned_counters, 512));
    }
    void ensure_stage(size_t bytes) {
        if (stage_bytes >= bytes) return;
        if (stage) cudaFreeHost(stage);
        stage = nullptr;
        stage_bytes = 0;
        CK(cudaMallocHost(&stage, bytes));
        stage_bytes = bytes;
    }
    ~DeviceSceneImpl() {
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        for (auto& e : kev) if (e) cudaEventDestroy(e);
        for (auto& e : copy_ev) if (e) cudaEventDestroy(e);
        if (window_exec) cudaGraphExecDestroy(window_exec);
        if (loop_exec) cudaGraphExecDestroy(loop_exec);
        if (view_stage) cudaFreeHost(view_stage);
        if (pinned_counters) cudaFreeHost(pinned_counters);
        if (stage) cudaFreeHost(stage);
        if (stream) cudaStreamDestroy(stream);
    }
};

}  // namespace atrc

struct AtrcScene {
    atrc::DeviceSceneImpl impl;
};

namespace atrc {
namespace {

int fail(int code, const std::string& msg) {
    set_last_error(msg);
    return code;
}

template <class F>
int guarded(F&& f) {
    try {
        return f();
    } catch (const CudaError& e) {
        return fail(ATRC_ERR_CUDA, e.what());
    } catch (const std::bad_alloc&) {
        return fail(ATRC_ERR_OUT_OF_MEMORY, "host allocation failed");
    } catch (const std::exception& e) {
        return fail(ATRC_ERR_UNSUPPORTED, e.what());
    }
}

void check_device_ready() {
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0)
        throw CudaError(std::string("no usable CUDA device: ") + (e != cudaSuccess ? cudaGetErrorString(e) : "count is 0"));
}

// Layout of the path pool inside one allocation.
struct PoolLayout {
    size_t off[28];
    size_t total;
};

// k_shadow's grid.  The queue's length is known only on the device, so the
// grid is fixed when the window is captured; k_shadow strides over the queue
// and a thread traces one ray as long as the queue holds at most
// kShadowGridWaves resident waves (148 SMs x 10 blocks x 128 threads each).
// A grid covering the whole capacity (the pool times the rays one path can
// emit) would launch tens of thousands of blocks that find no ray: an
// iteration of the instanced workload queues about 260,000 occlusion rays
// against a capacity of 4M.
constexpr int kShadowGridWaves = 8;
int shadow_grid(size_t shadow_cap, int sm_count) {
    const size_t full = (shadow_cap + 127) / 128;
    return int(std::min<size_t>(full, size_t(sm_count) * ATRC_SHADOW_MIN_BLOCKS * kShadowGridWaves));
}

PoolLayout pool_layout(size_t cap, size_t shadow_cap, int nkeys) {
    PoolLayout L{};
    size_t o = 0;
    auto take = [&](int i, size_t bytes) {
        o = (o + 255) & ~size_t(255);
        L.off[i] = o;
        o += bytes;
    };
    take(0, cap * 16); take(1, cap * 16); take(2, cap * 16); take(3, cap * 4);
    take(4, cap * 16); take(5, cap * 16); take(6, cap * 16); take(7, cap * 16); take(8, cap * 16);
    take(9, cap * 16); take(10, cap * 16);
    take(11, cap * 4); take(12, cap * 4); take(13, cap * 4); take(14, cap * 4);
    take(15, shadow_cap * 16); take(16, shadow_cap * 16); take(17, shadow_cap * 16);
    take(18, cap * 4); take(19, cap * 4); take(20, size_t(nkeys) * 4); take(21, size_t(nkeys) * 4);
    take(22, cap * 4);
    take(23, shadow_cap * 4); take(24, shadow_cap * 4); take(25, kShadowKeys * 4); take(26, kShadowKeys * 4);
    L.total = (o + 255) & ~size_t(255);
    return L;
}

Pool pool_from(void* base, const PoolLayout& L, size_t cap, size_t shadow_cap) {
    char* b = static_cast<char*>(base);
    Pool P;
    P.ray_o = reinterpret_cast<float4*>(b + L.off[0]);
    P.ray_d = reinterpret_cast<float4*>(b + L.off[1]);
    P.hit = reinterpret_cast<float4*>(b + L.off[2]);
    P.hit_tri = reinterpret_cast<int*>(b + L.off[3]);
    P.coef = reinterpret_cast<float4*>(b + L.off[4]);
    P.L = reinterpret_cast<float4*>(b + L.off[5]);
    P.mis_f = reinterpret_cast<float4*>(b + L.off[6]);
    P.gb_albedo = reinterpret_cast<float4*>(b + L.off[7]);
    P.gb_normal = reinterpret_cast<float4*>(b + L.off[8]);
    P.st = reinterpret_cast<uint4*>(b + L.off[9]);
    P.ctr = reinterpret_cast<int4*>(b + L.off[10]);
    P.q[0] = reinterpret_cast<int*>(b + L.off[11]);
    P.q[1] = reinterpret_cast<int*>(b + L.off[12]);
    P.q_finish = reinterpret_cast<int*>(b + L.off[13]);
    P.slot_state = reinterpret_cast<int*>(b + L.off[14]);
    P.sh_o = reinterpret_cast<float4*>(b + L.off[15]);
    P.sh_d = reinterpret_cast<float4*>(b + L.off[16]);
    P.sh_c = reinterpret_cast<float4*>(b + L.off[17]);
    P.q_sorted = reinterpret_cast<int*>(b + L.off[18]);
    P.keys = reinterpret_cast<int*>(b + L.off[19]);
    P.key_count = reinterpret_cast<int*>(b + L.off[20]);
    P.key_cursor = reinterpret_cast<int*>(b + L.off[21]);
    P.q_sss = reinterpret_cast<int*>(b + L.off[22]);
    P.sh_key = reinterpret_cast<int*>(b + L.off[23]);
    P.sh_sorted = reinterpret_cast<int*>(b + L.off[24]);
    P.sh_count = reinterpret_cast<int*>(b + L.off[25]);
    P.sh_cursor = reinterpret_cast<int*>(b + L.off[26]);
    P.shadow_sort = 0;
    for (int a = 0; a < 3; ++a) P.sk_lo[a] = P.sk_scale[a] = 0.0f;
    P.cap = int(cap);
    P.shadow_cap = int(shadow_cap);
    return P;
}

// The shadow-queue sort of a render: on when the scene's tuning asks for
// it, over the scene's bound.
void set_shadow_sort(Pool* P, const Scene& S, int on) {
    P->shadow_sort = on;
    for (int a = 0; a < 3; ++a) {
        const float ext = S.scene_hi[a] - S.scene_lo[a];
        P->sk_lo[a] = S.scene_lo[a];
        P->sk_scale[a] = ext > 0.0f ? 16.0f / ext : 0.0f;
    }
}

// Settings shared by the views of a render (taken from the first view).
// Shadow rays one path emits per iteration: one per light (pt), or the
// occlusion rays of a camera hit (ao).
static int shadow_rays_per_path(const Scene& S, const AtrcRenderDesc& d) {
    return d.renderer == ATRC_RENDERER_AO ? std::max(1, d.ao_sample_count) : std::max(1, S.light_count);
}

Params make_params(const AtrcRenderDesc& d) {
    Params p{};
    p.min_depth = d.min_depth;
    p.max_depth = d.max_depth;
    p.specular_depth = d.specular_depth;
    p.cont_prob = d.cont_prob;
    p.eps = d.eps;
    p.renderer = d.renderer;
    p.ao_count = d.ao_sample_count;
    p.ao_dist = d.ao_max_distance;
    for (int k = 0; k < 3; ++k) {
        p.ao_low[k] = d.ao_low[k];
        p.ao_high[k] = d.ao_high[k];
        p.ao_bg[k] = d.ao_background[k];
    }
    return p;
}

// One view: camera, film geometry, tiles and filter (count and start, tile
// tables and film are filled in by the caller).
View make_view(const AtrcRenderDesc& d) {
    View p{};
    p.W = d.width;
    p.H = d.height;
    p.first_spp = d.first_spp;
    p.seed = d.seed;
    // ThinLensCamera::init_from_params (thin_lens.cpp:34-55)
    const AtrcCameraDesc& c = d.camera;
    const Vec3 pos(c.pos[0], c.pos[1], c.pos[2]), dst(c.dst[0], c.dst[1], c.dst[2]), up(c.up[0], c.up[1], c.up[2]);
    const Vec3 fz = normalize(dst - pos);
    const Vec3 fx = normalize(cross(up, fz));
    const Vec3 fy = cross(fz, fx);
    for (int k = 0; k < 3; ++k) {
        p.cam.pos[k] = pos[k];
        p.cam.fx[k] = fx[k];
        p.cam.fy[k] = fy[k];
        p.cam.fz[k] = fz[k];
    }
    const float aspect = float(d.width) / float(d.height);
    p.cam.film_h = 2 * c.focal_distance * std::tan(c.fov / 2);
    p.cam.film_w = aspect * p.cam.film_h;
    p.cam.focal = c.focal_distance;
    p.cam.lens_radius = c.lens_radius;
    // film filters (box_filter.cpp:6-34, gaussian_filter.cpp:6-78)
    p.filter_type = d.filter_type;
    if (d.filter_type == ATRC_FILTER_BOX) {
        p.filter_radius = d.filter_radius - d.eps;
        p.filter_value = 1 / (4 * p.filter_radius * p.filter_radius);
    } else {
        p.filter_radius = d.filter_radius;
        p.filter_alpha = d.filter_alpha;
        p.filter_exp = std::exp(-d.filter_alpha * d.filter_radius * d.filter_radius);
        p.filter_value = 1;
    }
    // sample grid (the same float expressions as k_tiles)
    p.G = d.task_grid_size > 0 ? d.task_grid_size : 32;
    p.TX = (d.width + p.G - 1) / p.G;
    p.TY = (d.height + p.G - 1) / p.G;
    const float r = p.filter_radius;
    auto extent = [&](int n, int* first) {
        int acc = 0;
        for (int g = 0; g * p.G < n; ++g) {
            const int a0 = g * p.G, a1 = std::min(n, a0 + p.G) - 1;
            const int s0 = int(std::floor(float(a0) + 0.5f - r)), s1 = int(std::floor(float(a1) + 0.49999f + r));
            if (g == 0) *first = s1 - s0 + 1;
            acc += s1 - s0 + 1;
        }
        return acc;
    };
    p.SW = extent(d.width, &p.E0X);
    p.SH = extent(d.height, &p.E0Y);
    return p;
}

size_t tile_table_bytes(const View& p) { return size_t(p.TX + p.TY + 2) * sizeof(int4); }

void* noalloc_scratch(int device);  // static scratch of atrc_cuda_render_noalloc (below)

// Point a view at its tile table (filled on the device by k_tiles).
void set_tiles(View* v, void* table) {
    v->tile_cols = static_cast<int4*>(table);
    v->tile_rows = v->tile_cols + v->TX + 1;
}

}  // namespace
}  // namespace atrc

using namespace atrc;

extern "C" {

int atrc_cuda_device_init(int device, AtrcDeviceInfo* info) {
    return guarded([&] {
        check_device_ready();
        CK(cudaSetDevice(device));
        cudaDeviceProp prop;
        CK(cudaGetDeviceProperties(&prop, device));
        if (info) {
            std::memset(info, 0, sizeof(*info));
            std::strncpy(info->name, prop.name, sizeof(info->name) - 1);
            info->sm_count = prop.multiProcessorCount;
            info->cc_major = prop.major;
            info->cc_minor = prop.minor;
            info->global_mem_bytes = prop.totalGlobalMem;
        }
        if (prop.major < 10) throw CudaError("pt_cuda is built for sm_100a (Blackwell); device is sm_" +
                                             std::to_string(prop.major) + std::to_string(prop.minor));
        return int(ATRC_OK);
    });
}

int atrc_cuda_scene_create(const AtrcSceneDesc* desc, AtrcScene** out) {
    if (!desc || !out) return fail(ATRC_ERR_INVALID_ARG, "atrc_cuda_scene_create: null argument");
    *out = nullptr;
    return guarded([&] {
        check_device_ready();
        int device = 0;
        CK(cudaGetDevice(&device));
        auto hs = std::make_unique<HostScene>();
        build_host_scene(*desc, hs.get(), device);
        auto sc = std::make_unique<AtrcScene>();
        DeviceSceneImpl& d = sc->impl;
        CK(cudaGetDevice(&d.device));
        CK(cudaDeviceGetAttribute(&d.sm_count, cudaDevAttrMultiProcessorCount, d.device));
        CK(cudaStreamCreateWithFlags(&d.stream, cudaStreamNonBlocking));
        cudaStream_t s = d.stream;
        Scene S = hs->scene;
        S.nodes = upload(d.nodes, hs->nodes, s);
        S.tris = upload(d.tris, hs->tris, s);
        S.tri_bc = upload(d.tri_bc, hs->tri_bc, s);
        S.tri_shade = upload(d.tri_shade, hs->tri_shade, s);
        S.tri_orig = upload(d.tri_orig, hs->tri_orig, s);
        S.entities = upload(d.entities, hs->entities, s);
        S.tlas_order = upload(d.tlas_order, hs->tlas_order, s);
        S.materials = upload(d.materials, hs->materials, s);
        S.material_count = int32_t(hs->materials.size());
        S.tex2d = upload(d.tex2d, hs->tex2d, s);
        S.tex3d = upload(d.tex3d, hs->tex3d, s);
        S.texels = upload(d.texels, hs->texels, s);
        S.media = upload(d.media, hs->media, s);
        S.alias_prob = upload(d.alias_prob, hs->alias_prob, s);
        S.alias_idx = upload(d.alias_idx, hs->alias_idx, s);
        S.env.probs = upload(d.env_probs, hs->env_probs, s);
        S.env.alias_prob = upload(d.env_alias_prob, hs->env_alias_prob, s);
        S.env.alias_idx = upload(d.env_alias_idx, hs->env_alias_idx, s);
        S.eps = 3e-4f;
        d.scene = S;
        d.watchdog.alloc(2 * sizeof(int));  // [0] watchdog code, [1] ray-query cursor
        // load the module's static scratch onto this device now, so that
        // atrc_cuda_render_noalloc neither allocates nor looks it up itself
        noalloc_scratch(d.device);
        CK(cudaStreamSynchronize(s));
        *out = sc.release();
        return int(ATRC_OK);
    });
}

void atrc_cuda_scene_destroy(AtrcScene* scene) { delete scene; }

int atrc_cuda_trace_rays_device(AtrcScene* scene, const AtrcRay* d_rays, size_t n, AtrcHit* d_hits, int mode,
                                int exact) {
    if (!scene || (n && (!d_rays || !d_hits))) return fail(ATRC_ERR_INVALID_ARG, "atrc_cuda_trace_rays: null argument");
    if (mode != ATRC_QUERY_CLOSEST && mode != ATRC_QUERY_ANY) return fail(ATRC_ERR_INVALID_ARG, "bad query mode");
    if (exact < ATRC_ISECT_FAST || exact > ATRC_ISECT_WATERTIGHT)
        return fail(ATRC_ERR_INVALID_ARG, "atrc_cuda_trace_rays: bad intersection mode");
    return guarded([&] {
        DeviceSceneImpl& d = scene->impl;
        if (n == 0) return int(ATRC_OK);
        CK(cudaMemsetAsync(d.watchdog.p, 0, sizeof(int), d.stream));
        const int grid = grid_for(d.sm_count, 8);
        int* wd = d.watchdog.as<int>();
        int* cur = wd + 1;
        cudaStream_t st = d.stream;
        // the query cursor is an int: batches of at most 2^30 rays
        for (size_t off = 0; off < n; off += size_t(1) << 30) {
            const int m = int(std::min(n - off, size_t(1) << 30));
            const AtrcRay* rr = d_rays + off;
            AtrcHit* hh = d_hits + off;
            CK(cudaMemsetAsync(cur, 0, sizeof(int), st));
            if (mode == ATRC_QUERY_ANY) {
                if (exact == ATRC_ISECT_WATERTIGHT)
                    k_trace_rays<ISECT_WATERTIGHT, true><<<grid, 128, 0, st>>>(d.scene, rr, m, hh, cur, wd);
                else if (exact == ATRC_ISECT_EXACT)
                    k_trace_rays<ISECT_EXACT, true><<<grid, 128, 0, st>>>(d.scene, rr, m, hh, cur, wd);
                else
                    k_trace_rays<ISECT_FAST, true><<<grid, 128, 0, st>>>(d.scene, rr, m, hh, cur, wd);
            } else {
                if (exact == ATRC_ISECT_WATERTIGHT)
                    k_trace_rays<ISECT_WATERTIGHT, false><<<grid, 128, 0, st>>>(d.scene, rr, m, hh, cur, wd);
                else if (exact == ATRC_ISECT_EXACT)
                    k_trace_rays<ISECT_EXACT, false><<<grid, 128, 0, st>>>(d.scene, rr, m, hh, cur, wd);
                else
                    k_trace_rays<ISECT_FAST, false><<<grid, 128, 0, st>>>(d.scene, rr, m, hh, cur, wd);
            }
        }
        CK(cudaGetLastError());
        int w = 0;
        CK(cudaMemcpyAsync(&w, wd, sizeof(int), cudaMemcpyDeviceToHost, d.stream));
        CK(cudaStreamSynchronize(d.stream));
        if (w) return fail(ATRC_ERR_WATCHDOG, "traversal stack limit reached (code " + std::to_string(w) + ")");
        return int(ATRC_OK);
    });
}

int atrc_cuda_trace_rays(AtrcScene* scene, const AtrcRay* rays, size_t n, AtrcHit* hits, int mode, int exact) {
    if (!scene || (n && (!rays || !hits))) return fail(ATRC_ERR_INVALID_ARG, "atrc_cuda_trace_rays: null argument");
    return guarded([&] {
        DeviceSceneImpl& d = scene->impl;
        if (n == 0) return int(ATRC_OK);
        DevBuf r, h;
        r.alloc(n * sizeof(AtrcRay));
        h.alloc(n * sizeof(AtrcHit));
        CK(cudaMemcpyAsync(r.p, rays, n * sizeof(AtrcRay), cudaMemcpyHostToDevice, d.stream));
        int rc = atrc_cuda_trace_rays_device(scene, r.as<AtrcRay>(), n, h.as<AtrcHit>(), mode, exact);
        if (rc != ATRC_OK) return rc;
        CK(cudaMemcpyAsync(hits, h.p, n * sizeof(AtrcHit), cudaMemcpyDeviceToHost, d.stream));
        CK(cudaStreamSynchronize(d.stream));
        return int(ATRC_OK);
    });
}

// n subsurface probes from the closest hit of one ray (a check of
// subsurface_sample against the oracle's; thread i draws its own stream).
__global__ void k_subsurface_probe(Scene S, Vec3 o, Vec3 d, int n, uint64_t seed, float eps, float* w, float* x,
                                   int* status) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Vec3 wv, xp;
    Hit h;
    int wd = 0;
    if (!trace_ray<ISECT_FAST, false>(S, o, d, 0.0f, INFINITY, &h, &wd)) {
        if (i == 0) *status = 1;
    } else {
        const Surface s = make_surface(S, h, o, d);
        const Material& m = S.materials[S.entities[h.entity].material];
        if (m.bssrdf[1] < 0) {
            if (i == 0) *status = 2;
        } else {
            Rng rng;
            rng.state = mix64(seed ^ (uint64_t(i) * 0x9E3779B97F4A7C15ULL));
            Surface ex;
            BSDF bx;
            if (subsurface_sample(S, m, s, rng, &wd, eps, &ex, &bx, &wv)) xp = ex.pos;
            else wv = Vec3();
        }
    }
    if (wd) *status = 3;
    w[3 * i] = wv.x; w[3 * i + 1] = wv.y; w[3 * i + 2] = wv.z;
    x[3 * i] = xp.x; x[3 * i + 1] = xp.y; x[3 * i + 2] = xp.z;
}

static int check_render_args(AtrcScene* scene, const AtrcRenderDesc* desc, const AtrcFilm* film) {
    if (!scene || !desc || !film || !film->value || !film->weight)
        return fail(ATRC_ERR_INVALID_ARG, "atrc_cuda_render: null argument");
    if (desc->width <= 0 || desc->height <= 0 || desc->spp <= 0 || desc->max_depth < 0)
        return fail(ATRC_ERR_INVALID_ARG, "atrc_cuda_render: invalid film size, spp or depth");
    if (desc->spp_count < 0 || desc->first_spp < 0)
        return fail(ATRC_ERR_INVALID_ARG, "atrc_cuda_render: invalid sample range");
    if (desc->sort_mode < ATRC_SORT_AUTO || desc->sort_mode > ATRC_SORT_MATERIAL)
        return fail(ATRC_ERR_INVALID_ARG, "atrc_cuda_render: invalid sort_mode");
    if (desc->filter_type == ATRC_FILTER_BOX ? !(desc->filter_radius - desc->eps > 0) : !(desc->filter_radius > 0 && desc->filter_alpha > 0))
        return fail(ATRC_ERR_INVALID_ARG, "atrc_cuda_render: invalid film filter");
    if (desc->renderer != ATRC_RENDERER_PT && desc->renderer != ATRC_RENDERER_AO)
        return fail(ATRC_ERR_INVALID_ARG, "atrc_cuda_render: invalid renderer");
    if (desc->renderer == ATRC_RENDERER_AO && (desc->ao_sample_count <= 0 || desc->ao_sample_count > 4096))
        return fail(ATRC_ERR_INVALID_ARG, "atrc_cuda_render: ao_sample_count must be in [1, 4096]");
    if (desc->isect_mode != ATRC_ISECT_FAST && desc->isect_mode != ATRC_ISECT_WATERTIGHT)
        return fail(ATRC_ERR_INVALID_ARG,
                    "atrc_cuda_render: isect_mode must be ATRC_ISECT_FAST (0) or ATRC_ISECT_WATERTIGHT (2)");
    // the reference's pt runs trace_nomis for use_mis = 0 (pt.cpp:8-42), an
    // estimator whose image differs from trace_std's; it is not built here
    if (desc->renderer == ATRC_RENDERER_PT && !desc->use_mis)
        return fail(ATRC_ERR_UNSUPPORTED, "atrc_cuda_render: use_mis = 0 (trace_nomis) is not supported by pt_cuda");
    return ATRC_OK;
}

int atrc_cuda_subsurface_probe(AtrcScene* scene, const float o[3], const float d[3], int32_t n, uint64_t seed,
                               float* w, float* exit_pos) {
    if (!scene || !o || !d || !w || !exit_pos || n <= 0)
        return fail(ATRC_ERR_INVALID_ARG, "atrc_cuda_subsurface_probe: null argument");
    return guarded([&] {
        DeviceSceneImpl& dv = scene->impl;
        CK(cudaSetDevice(dv.device));
        DevBuf bw, bx, bs;
        bw.alloc(size_t(n) * 12);
        bx.alloc(size_t(n) * 12);
        bs.alloc(4);
        CK(cudaMemsetAsync(bs.p, 0, 4, dv.stream));
        const Vec3 ov(o[0], o[1], o[2]), dvv = normalize(Vec3(d[0], d[1], d[2]));
        k_subsurface_probe<<<(n + 127) / 128, 128, 0, dv.stream>>>(dv.scene, ov, dvv, n, seed, dv.scene.eps,
                                                                 bw.as<float>(), bx.as<float>(), bs.as<int>());
        CK(cudaGetLastError());
        int status = 0;
        CK(cudaMemcpyAsync(w, bw.p, size_t(n) * 12, cudaMemcpyDeviceToHost, dv.stream));
        CK(cudaMemcpyAsync(exit_pos, bx.p, size_t(n) * 12, cudaMemcpyDeviceToHost, dv.stream));
        CK(cudaMemcpyAsync(&status, bs.p, 4, cudaMemcpyDeviceToHost, dv.stream));
        CK(cudaStreamSynchronize(dv.stream));
        if (status == 1) return fail(ATRC_ERR_INVALID_ARG, "atrc_cuda_subsurface_probe: the ray hits nothing");
        if (status == 2) return fail(ATRC_ERR_INVALID_ARG, "atrc_cuda_subsurface_probe: no subsurface material");
        if (status == 3) return fail(ATRC_ERR_WATCHDOG, "atrc_cuda_subsurface_probe: traversal bound exceeded");
        return int(ATRC_OK);
    });
}


// The wavefront render behind atrc_cuda_render (arguments already checked;
// CUDA failures throw).  Launch shapes, path pool and sort mode left to
// the library (path_pool 0, sort_mode AUTO) come from the scene's tuning.
// `nviews` views share one path pool (a batch); descs[0] gives the settings
// they share.  A single view may use a host film (staged on the device);
// batches need device films.  view_seconds (optional, nviews entries)
// receives the time from the start of the call at which each view's last
// sample was splatted, observed at window granularity.
static int render_impl(AtrcScene* scene, const AtrcRenderDesc* descs, const AtrcFilm* films, int nviews,
                       AtrcCancelFn should_stop, AtrcProgressFn progress, void* user, AtrcRenderStats* stats,
                       GuideImpl* guide = nullptr, bool record = false, double* view_seconds = nullptr,
                       bool device_loop = false) {
    const auto t_start = std::chrono::steady_clock::now();
    const AtrcRenderDesc* desc = descs;
    const AtrcFilm* film = films;
    DeviceSceneImpl& d = scene->impl;
    CK(cudaSetDevice(d.device));
    cudaStream_t s = d.stream;
    d.scene.eps = desc->eps;
    d.scene.disney_fixed = desc->disney_fixed;
    Params p = make_params(*desc);
    d.resolve_sort(&p, desc->sort_mode);
    // views, their tile tables and sample ranges
    std::vector<View> views(nviews);
    size_t table_bytes = 0;
    unsigned long long total = 0;
    for (int v = 0; v < nviews; ++v) {
        views[v] = make_view(descs[v]);
        if (size_t(views[v].TX) * views[v].TY >= (size_t(1) << kTileBits))
            throw std::runtime_error("film too large: more than 2^22 filter tiles");
        table_bytes += (tile_table_bytes(views[v]) + 255) & ~size_t(255);
        const int spp_v = descs[v].spp_count > 0 ? descs[v].spp_count : descs[v].spp;
        views[v].start = total;
        views[v].count = (unsigned long long)views[v].SW * views[v].SH * spp_v;
        total += views[v].count;
    }
    if (d.tiles.bytes < table_bytes) d.tiles.alloc(table_bytes);
    {
        char* tb = d.tiles.as<char>();
        for (int v = 0; v < nviews; ++v) {
            set_tiles(&views[v], tb);
            tb += (tile_table_bytes(views[v]) + 255) & ~size_t(255);
        }
    }
    // path pool: enough paths to fill the GPU; shadow capacity = pool x
    // shadow rays one path can emit in one iteration
    const int nl = shadow_rays_per_path(d.scene, *desc);
    size_t cap = desc->path_pool > 0 ? size_t(desc->path_pool) : size_t(d.tuned_pool);
    cap = std::min<size_t>(cap, std::max<unsigned long long>(total, 1024ULL));
    cap = std::min<size_t>(cap, (size_t(1) << 28) / nl);
    const size_t shadow_cap = cap * nl;
    const PoolLayout L = pool_layout(cap, shadow_cap, p.nkeys);
    // the buffer only grows: a smaller pool is laid out inside it (k_init
    // resets every word that must start from a known value), so renders of
    // changing sizes do not pay a cudaFree + cudaMalloc each
    if (d.pool_buf.bytes < L.total) d.pool_buf.alloc(L.total);
    if (!d.counters.p) d.counters.alloc(sizeof(Counters));
    if (guide) {
        if (guide_device(guide) != d.device) throw std::runtime_error("the guide lives on another device than the scene");
        p.guide_on = 1;
        p.gf = guide_frame(guide, cap, record, s);
    }
    Pool P = pool_from(d.pool_buf.p, L, cap, shadow_cap);
    set_shadow_sort(&P, d.scene, d.tuned_shadow_sort);
    Counters* c = d.counters.as<Counters>();
    // films
    const size_t npix = size_t(desc->width) * desc->height;
    std::vector<std::pair<double*, size_t>> host_targets;
    DevBuf& local_film = d.film_buf;
    d.ensure_render_resources();
    for (int v = 1; v < nviews; ++v) {
        const AtrcFilm& f = films[v];
        views[v].film = Film{f.value, f.weight, f.value_sq, f.albedo, f.normal, f.denoise};
    }
    Film& F = views[0].film;
    if (film->on_device) {
        F.value = film->value; F.weight = film->weight; F.value_sq = film->value_sq;
        F.albedo = film->albedo; F.normal = film->normal; F.denoise = film->denoise;
    } else {
        size_t doubles = npix * 4 + (film->value_sq ? npix * 3 : 0) + (film->albedo ? npix * 3 : 0) +
                         (film->normal ? npix * 3 : 0) + (film->denoise ? npix : 0);
        if (local_film.bytes < doubles * sizeof(double)) local_film.alloc(doubles * sizeof(double));
        CK(cudaMemsetAsync(local_film.p, 0, doubles * sizeof(double), s));
        double* b = local_film.as<double>();
        F.value = b; b += npix * 3; host_targets.push_back({film->value, npix * 3});
        F.weight = b; b += npix; host_targets.push_back({film->weight, npix});
        if (film->value_sq) { F.value_sq = b; b += npix * 3; host_targets.push_back({film->value_sq, npix * 3}); }
        if (film->albedo) { F.albedo = b; b += npix * 3; host_targets.push_back({film->albedo, npix * 3}); }
        if (film->normal) { F.normal = b; b += npix * 3; host_targets.push_back({film->normal, npix * 3}); }
        if (film->denoise) { F.denoise = b; b += npix; host_targets.push_back({film->denoise, npix}); }
    }
    // view table on the device; the device-side loop (batches) also keeps
    // per-view finished-sample counters and completion timestamps
    const size_t vbytes = (nviews * sizeof(View) + 255) & ~size_t(255);
    const size_t dbytes = device_loop ? nviews * sizeof(unsigned long long) : 0;
    if (d.views_buf.bytes < vbytes + 2 * dbytes) d.views_buf.alloc(vbytes + 2 * dbytes);
    CK(cudaMemcpyAsync(d.views_buf.p, views.data(), nviews * sizeof(View), cudaMemcpyHostToDevice, s));
    p.nviews = nviews;
    p.views = d.views_buf.as<View>();
    p.view_done = nullptr;
    p.view_time = nullptr;
    if (dbytes) {
        p.view_done = reinterpret_cast<unsigned long long*>(d.views_buf.as<char>() + vbytes);
        p.view_time = p.view_done + nviews;
        CK(cudaMemsetAsync(p.view_done, 0, 2 * dbytes, s));
        d.ensure_view_stage(dbytes);
    }
    k_tiles<<<nviews, 32, 0, s>>>(p);
    const int gsm = grid_for(d.sm_count, d.tuned_gen_blocks);
    // one path / ray per thread for the heavy kernels (grids cover the
    // pool; threads past the device-side count return at once)
    const int g_path = int((cap + 127) / 128), g_shadow = shadow_grid(shadow_cap, d.sm_count);
    k_init<<<int((std::max<size_t>({cap, size_t(p.nkeys), size_t(kShadowKeys)}) + 255) / 256), 256, 0, s>>>(
        P, int(cap), p.nkeys, c, total);
    CK(cudaGetLastError());
    uint64_t launches = 2, ext_launches = 0;  // k_tiles, k_init
    cudaEvent_t ev0 = d.ev0, ev1 = d.ev1;
    cudaEvent_t* kev = d.kev;
    const int window = DeviceSceneImpl::kWindow;
    double t_ext = 0, t_shade = 0, t_shadow = 0;
    Counters hc{};
    static_assert(sizeof(Counters) <= 512, "pinned counter buffer too small");
    Counters* pinned = static_cast<Counters*>(d.pinned_counters);
    int status = ATRC_OK;
    // the traversal counts (count_traversal) are taken with Moller-Trumbore
    // only; a watertight render ignores them
    const bool wt = desc->isect_mode == ATRC_ISECT_WATERTIGHT;
    const bool count = desc->count_traversal != 0 && !wt;
    const int per_iter = 6 + (p.sort_mode != ATRC_SORT_NONE ? 2 : 0) + (guide ? 2 : 0) + (d.scene.has_subsurface ? 1 : 0) +
                         (P.shadow_sort ? 2 : 0);
    // The kernels of one window of `window` wavefront iterations.  The
    // kernels take their sizes from the device-side counters, so every window
    // is the same sequence of launches.  `timed` records the events that
    // split the window's device time into traversal, shading and shadow rays
    // (event nodes are not allowed inside the device-side loop).
    auto enqueue_window = [&](bool timed) {
        for (int k = 0; k < window; ++k) {
            k_begin<<<1, 1, 0, s>>>(c);
            k_generate<<<gsm, d.tuned_gen_threads, 0, s>>>(d.scene, p, P, c);
            if (timed) CK(cudaEventRecordWithFlags(kev[k * 4 + 0], s, cudaEventRecordExternal));
            if (d.tuned_fetch) {
                const int g_fetch = d.sm_count * ATRC_TRACE_MIN_BLOCKS;
                if (wt) k_extend_fetch<ISECT_WATERTIGHT, false><<<g_fetch, kTraceBlock, 0, s>>>(d.scene, P, c, p.sort_mode, p.nkeys);
                else if (count) k_extend_fetch<ISECT_FAST, true><<<g_fetch, kTraceBlock, 0, s>>>(d.scene, P, c, p.sort_mode, p.nkeys);
                else k_extend_fetch<ISECT_FAST, false><<<g_fetch, kTraceBlock, 0, s>>>(d.scene, P, c, p.sort_mode, p.nkeys);
            } else if (wt) {
                k_extend<ISECT_WATERTIGHT, false><<<g_path, 128, 0, s>>>(d.scene, P, c, p.sort_mode, p.nkeys);
            } else if (count) {
                k_extend<ISECT_FAST, true><<<g_path, 128, 0, s>>>(d.scene, P, c, p.sort_mode, p.nkeys);
            } else {
                k_extend<ISECT_FAST, false><<<g_path, 128, 0, s>>>(d.scene, P, c, p.sort_mode, p.nkeys);
            }
            if (p.sort_mode != ATRC_SORT_NONE) {
                k_sort_scan<<<1, 1024, 0, s>>>(P, p.nkeys);
                k_sort_scatter<<<d.sm_count * 8, 128, 0, s>>>(P, c, p.nkeys);
            }
            if (timed) CK(cudaEventRecordWithFlags(kev[k * 4 + 1], s, cudaEventRecordExternal));
            if (guide) {
                k_guide_features<<<g_path, 128, 0, s>>>(d.scene, p, P, c);
                guide_infer(guide, &c->n_guide, s);
            }
            k_shade<<<g_path, 128, 0, s>>>(d.scene, p, P, c);
            if (d.scene.has_subsurface) k_subsurface<<<g_path, 128, 0, s>>>(d.scene, p, P, c);
            if (timed) CK(cudaEventRecordWithFlags(kev[k * 4 + 2], s, cudaEventRecordExternal));
            if (P.shadow_sort) {
                k_shsort_scan<<<1, 1024, 0, s>>>(P);
                k_shsort_scatter<<<d.sm_count * 8, 128, 0, s>>>(P, c);
            }
            if (d.tuned_shadow_fetch) {
                const int g_fetch = d.sm_count * ATRC_TRACE_MIN_BLOCKS;
                if (wt) k_shadow_fetch<ISECT_WATERTIGHT, false><<<g_fetch, kTraceBlock, 0, s>>>(d.scene, P, c);
                else if (count) k_shadow_fetch<ISECT_FAST, true><<<g_fetch, kTraceBlock, 0, s>>>(d.scene, P, c);
                else k_shadow_fetch<ISECT_FAST, false><<<g_fetch, kTraceBlock, 0, s>>>(d.scene, P, c);
            } else if (wt) {
                k_shadow<ISECT_WATERTIGHT, false><<<g_shadow, 128, 0, s>>>(d.scene, P, c);
            } else if (count) {
                k_shadow<ISECT_FAST, true><<<g_shadow, 128, 0, s>>>(d.scene, P, c);
            } else {
                k_shadow<ISECT_FAST, false><<<g_shadow, 128, 0, s>>>(d.scene, P, c);
            }
            if (timed) CK(cudaEventRecordWithFlags(kev[k * 4 + 3], s, cudaEventRecordExternal));
            k_finish<<<gsm, d.tuned_fin_threads, 0, s>>>(p, P, c);
        }
        CK(cudaGetLastError());
    };
    CK(cudaEventRecord(ev0, s));
    if (device_loop) {
        // The whole bounce loop is one graph launch: a WHILE conditional node
        // whose body is one window followed by k_loop_cond, which decides on
        // the device whether another window runs.  The host waits once, at
        // the end; per-view completion times are the device's timestamps.
        // No path lives longer than max_depth + specular_depth iterations
        // (plus a few for the MIS ray of its last vertex), and a slot starts
        // a new path as soon as one ends, so the loop is bounded by
        // (samples / pool + 1) path lengths; four times that stops it with a
        // watchdog status should a bug keep it from finishing.
        const unsigned long long per_path =
            (unsigned long long)std::max(desc->max_depth, 1) + (unsigned long long)std::max(desc->specular_depth, 0) + 8;
        const unsigned long long bound_iters = 4ULL * (total / cap + 2) * per_path + 256;
        const int max_windows = int(std::min<unsigned long long>(bound_iters / window + 1, (1ULL << 30)));
        cudaGraph_t outer = nullptr;
        CK(cudaGraphCreate(&outer, 0));
        struct GraphOwner {
            cudaGraph_t g;
            ~GraphOwner() { cudaGraphDestroy(g); }
        } owner{outer};
        cudaGraphConditionalHandle handle;
        CK(cudaGraphConditionalHandleCreate(&handle, outer, 1, cudaGraphCondAssignDefault));
        cudaGraphNodeParams np{};
        np.type = cudaGraphNodeTypeConditional;
        np.conditional.handle = handle;
        np.conditional.type = cudaGraphCondTypeWhile;
        np.conditional.size = 1;
        cudaGraphNode_t node = nullptr;
        CK(cudaGraphAddNode(&node, outer, nullptr, 0, &np));
        {
            BodyCapture body(s, np.conditional.phGraph_out[0]);
            enqueue_window(false);
            k_loop_cond<<<1, 1, 0, s>>>(c, handle, max_windows);
            CK(cudaGetLastError());
            body.end();
        }
        d.loop_exec = instantiate_or_update(d.loop_exec, outer);
        CK(cudaGraphLaunch(d.loop_exec, s));
        CK(cudaMemcpyAsync(pinned, c, sizeof(Counters), cudaMemcpyDeviceToHost, s));
        CK(cudaMemcpyAsync(d.view_stage, p.view_time, dbytes, cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        hc = *pinned;
        launches += uint64_t(hc.windows) * (uint64_t(window) * per_iter + 1);
        ext_launches = uint64_t(hc.windows) * window;
        if (view_seconds) {
            const unsigned long long* vt = static_cast<const unsigned long long*>(d.view_stage);
            for (int v = 0; v < nviews; ++v)
                view_seconds[v] = vt[v] >= hc.t_start ? double(vt[v] - hc.t_start) * 1e-9 : 0.0;
        }
        if (hc.watchdog) status = ATRC_ERR_WATCHDOG;
    } else {
        // One window (its kernels, the timing events and the counter
        // read-back) is captured once per call as a CUDA graph and relaunched
        // until the device-side counters say the work is done; the host
        // polls progress and the cancel callback between windows.  The
        // executable graph is kept with the scene and updated in place when
        // the next call's parameters differ.
        {
            CaptureGuard capg(s);
            enqueue_window(true);
            CK(cudaMemcpyAsync(pinned, c, sizeof(Counters), cudaMemcpyDeviceToHost, s));
            cudaGraph_t g = capg.end();
            d.window_exec = instantiate_or_update(d.window_exec, g);
            cudaGraphDestroy(g);
        }
        for (;;) {
            CK(cudaGraphLaunch(d.window_exec, s));
            launches += uint64_t(per_iter) * window;
            ext_launches += window;
            CK(cudaStreamSynchronize(s));
            hc = *pinned;
            for (int k = 0; k < window; ++k) {
                float a = 0, b2 = 0, e3 = 0;
                CK(cudaEventElapsedTime(&a, kev[k * 4 + 0], kev[k * 4 + 1]));
                CK(cudaEventElapsedTime(&b2, kev[k * 4 + 1], kev[k * 4 + 2]));
                CK(cudaEventElapsedTime(&e3, kev[k * 4 + 2], kev[k * 4 + 3]));
                t_ext += a * 1e-3;
                t_shade += b2 * 1e-3;
                t_shadow += e3 * 1e-3;
            }
            if (hc.watchdog) { status = ATRC_ERR_WATCHDOG; break; }
            if (hc.done) break;
            if (progress) progress(100.0 * double(hc.completed) / double(std::max(1ULL, total)), user);
            if (should_stop && should_stop(user)) { status = ATRC_ERR_CANCELLED; break; }
        }
    }
    CK(cudaEventRecord(ev1, s));
    CK(cudaEventSynchronize(ev1));
    float kms = 0;
    CK(cudaEventElapsedTime(&kms, ev0, ev1));
    // bring host films up to date
    uint64_t d2h = sizeof(Counters);
    if (!host_targets.empty()) {
        size_t doubles = 0;
        for (auto& t : host_targets) doubles += t.second;
        d.ensure_stage(doubles * sizeof(double));
        const double* tmp = static_cast<const double*>(d.stage);
        // the download runs in chunks, each followed by an event; host threads
        // add chunk k into the caller's arrays while chunk k + 1 is in flight
        constexpr int kc = DeviceSceneImpl::kCopyChunks;
        const size_t chunk = ((doubles + kc - 1) / kc + 511) / 512 * 512;
        int nchunks = 0;
        for (size_t c0 = 0; c0 < doubles; c0 += chunk, ++nchunks) {
            const size_t n_el = std::min(chunk, doubles - c0);
            CK(cudaMemcpyAsync(static_cast<double*>(d.stage) + c0, local_film.as<double>() + c0, n_el * sizeof(double),
                               cudaMemcpyDeviceToHost, s));
            CK(cudaEventRecord(d.copy_ev[nchunks], s));
        }
        d2h += doubles * sizeof(double);
        std::vector<size_t> start(host_targets.size() + 1, 0);  // target k covers [start[k], start[k + 1])
        for (size_t k = 0; k < host_targets.size(); ++k) start[k + 1] = start[k] + host_targets[k].second;
        const unsigned nt = std::min<unsigned>(16, std::max(1u, std::thread::hardware_concurrency()));
        std::atomic<int> copy_err{0};
        auto add = [&](unsigned t) {
            for (int k = 0; k < nchunks; ++k) {
                if (cudaEventSynchronize(d.copy_ev[k]) != cudaSuccess) { copy_err = 1; return; }
                const size_t c0 = size_t(k) * chunk, c1 = std::min(doubles, c0 + chunk);
                const size_t a = c0 + (c1 - c0) * t / nt, b = c0 + (c1 - c0) * (t + 1) / nt;
                for (size_t j = 0; j < host_targets.size(); ++j) {
                    const size_t lo = std::max(a, start[j]), hi = std::min(b, start[j + 1]);
                    double* dst = host_targets[j].first;
                    for (size_t q = lo; q < hi; ++q) dst[q - start[j]] += tmp[q];
                }
            }
        };
        std::vector<std::thread> th;
        for (unsigned t = 1; t < nt; ++t) th.emplace_back(add, t);
        add(0);
        for (auto& x : th) x.join();
        if (copy_err) throw CudaError("atrc_cuda_render: film download failed");
    }
    if (stats) {
        std::memset(stats, 0, sizeof(*stats));
        stats->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count();
        stats->kernel_seconds = kms * 1e-3;
        stats->samples = hc.completed;
        stats->rays_closest = hc.rays_closest;
        stats->rays_shadow = hc.rays_shadow;
        stats->iterations = hc.iterations;
        stats->kernel_launches = launches;
        stats->watchdog_flags = uint64_t(hc.watchdog);
        stats->extend_seconds = t_ext;
        stats->shade_seconds = t_shade;
        stats->shadow_seconds = t_shadow;
        stats->h2d_bytes = 0;
        stats->d2h_bytes = d2h;
        stats->extend_launches = ext_launches;
        stats->shadow_launches = ext_launches;
        stats->nodes_closest = hc.cnt_closest[0];
        stats->tris_closest = hc.cnt_closest[1];
        stats->ents_closest = hc.cnt_closest[2];
        stats->nodes_shadow = hc.cnt_shadow[0];
        stats->tris_shadow = hc.cnt_shadow[1];
        stats->ents_shadow = hc.cnt_shadow[2];
    }
    if (progress && status == ATRC_OK) progress(100.0, user);
    if (status == ATRC_ERR_WATCHDOG)
        return fail(status, "a device loop reached its iteration cap (code " + std::to_string(hc.watchdog) + ")");
    if (status == ATRC_ERR_CANCELLED) return fail(status, "render cancelled");
    return int(ATRC_OK);
}

int atrc_cuda_render(AtrcScene* scene, const AtrcRenderDesc* desc, AtrcFilm* film, AtrcCancelFn should_stop,
                     AtrcProgressFn progress, void* user, AtrcRenderStats* stats) {
    const int rc = check_render_args(scene, desc, film);
    if (rc != ATRC_OK) return rc;
    return guarded([&] { return render_impl(scene, desc, film, 1, should_stop, progress, user, stats); });
}

int atrc_cuda_scene_bounds(AtrcScene* scene, float lo[3], float hi[3]) {
    if (!scene || !lo || !hi) return fail(ATRC_ERR_INVALID_ARG, "atrc_cuda_scene_bounds: null argument");
    for (int a = 0; a < 3; ++a) {
        lo[a] = scene->impl.scene.scene_lo[a];
        hi[a] = scene->impl.scene.scene_hi[a];
    }
    return ATRC_OK;
}

int atrc_cuda_render_guided(AtrcScene* scene, AtrcGuide* guide, const AtrcRenderDesc* desc, int32_t record,
                            AtrcFilm* film, AtrcRenderStats* stats) {
    if (!guide) return fail(ATRC_ERR_INVALID_ARG, "atrc_cuda_render_guided: null guide");
    const int rc = check_render_args(scene, desc, film);
    if (rc != ATRC_OK) return rc;
    if (desc->renderer != ATRC_RENDERER_PT)
        return fail(ATRC_ERR_INVALID_ARG, "atrc_cuda_render_guided: guiding needs the pt renderer");
    return guarded([&] {
        return render_impl(scene, desc, film, 1, nullptr, nullptr, nullptr, stats, guide_impl(guide), record != 0);
    });
}

int atrc_cuda_render_batch(AtrcScene* scene, AtrcGuide* guide, const AtrcRenderDesc* views, int32_t n,
                           const AtrcFilm* films, double* view_seconds, AtrcRenderStats* stats) {
    if (!scene || !views || !films || n < 1) return fail(ATRC_ERR_INVALID_ARG, "atrc_cuda_render_batch: null argument");
    if (n > kMaxViews) return fail(ATRC_ERR_INVALID_ARG, "atrc_cuda_render_batch: more than 1024 views");
    if (guide && views[0].renderer != ATRC_RENDERER_PT)
        return fail(ATRC_ERR_INVALID_ARG, "atrc_cuda_render_batch: guiding needs the pt renderer");
    const AtrcRenderDesc& a = views[0];
    for (int v = 0; v < n; ++v) {
        const int rc = check_render_args(scene, views + v, films + v);
        if (rc != ATRC_OK) return rc;
        if (!films[v].on_device)
            return fail(ATRC_ERR_INVALID_ARG, "atrc_cuda_render_batch: every film must hold device pointers");
        const AtrcRenderDesc& b = views[v];
        if (b.min_depth != a.min_depth || b.max_depth != a.max_depth || b.cont_prob != a.cont_prob ||
            b.specular_depth != a.specular_depth || b.eps != a.eps || b.sort_mode != a.sort_mode ||
            b.disney_fixed != a.disney_fixed || b.path_pool != a.path_pool || b.count_traversal != a.count_traversal ||
            b.isect_mode != a.isect_mode ||
            b.renderer != a.renderer || b.ao_sample_count != a.ao_sample_count ||
            b.ao_max_distance != a.ao_max_distance ||
            std::memcmp(b.ao_low, a.ao_low, sizeof(a.ao_low)) || std::memcmp(b.ao_high, a.ao_high, sizeof(a.ao_high)) ||
            std::memcmp(b.ao_background, a.ao_background, sizeof(a.ao_background)))
            return fail(ATRC_ERR_INVALID_ARG,
                        "atrc_cuda_render_batch: views must share renderer, depth, roulette, eps, sort, Disney and "
                        "pool settings");
    }
    return guarded([&] {
        return render_impl(scene, views, films, n, nullptr, nullptr, nullptr, stats, guide ? guide_impl(guide) : nullptr,
                           false, view_seconds, true);
    });
}

static void tuning_out(const DeviceSceneImpl& d, AtrcTuning* out) {
    out->path_pool = d.tuned_pool;
    out->sort_mode = d.tuned_sort;
    out->gen_blocks_per_sm = d.tuned_gen_blocks;
    out->gen_threads = d.tuned_gen_threads;
    out->finish_threads = d.tuned_fin_threads;
    out->trials = d.tuned_trials;
    out->ms_per_msample = d.tuned_ms;
    out->default_ms_per_msample = d.default_ms;
    out->extend_fetch = d.tuned_fetch;
    out->queue_order = d.tuned_queue;
    out->shadow_fetch = d.tuned_shadow_fetch;
    out->shadow_sort = d.tuned_shadow_sort;
}

int atrc_cuda_get_tuning(AtrcScene* scene, AtrcTuning* out) {
    if (!scene || !out) return fail(ATRC_ERR_INVALID_ARG, "atrc_cuda_get_tuning: null argument");
    tuning_out(scene->impl, out);
    return ATRC_OK;
}

static bool tuning_valid(const AtrcTuning& t) {
    auto pow2_in = [](int v, int lo, int hi) { return v >= lo && v <= hi && (v & (v - 1)) == 0; };
    return t.path_pool >= 1024 && t.path_pool <= (1 << 26) && t.sort_mode >= ATRC_SORT_NONE &&
           t.sort_mode <= ATRC_SORT_MATERIAL && t.gen_blocks_per_sm >= 1 && t.gen_blocks_per_sm <= 64 &&
           pow2_in(t.gen_threads, 32, 1024) && pow2_in(t.finish_threads, 32, 1024) &&
           (t.extend_fetch == 0 || t.extend_fetch == 1) && (t.queue_order == 0 || t.queue_order == 1) &&
           (t.shadow_fetch == 0 || t.shadow_fetch == 1) && (t.shadow_sort == 0 || t.shadow_sort == 1);
}

int atrc_cuda_set_tuning(AtrcScene* scene, const AtrcTuning* in) {
    if (!scene || !in) return fail(ATRC_ERR_INVALID_ARG, "atrc_cuda_set_tuning: null argument");
    if (!tuning_valid(*in)) return fail(ATRC_ERR_INVALID_ARG, "atrc_cuda_set_tuning: value out of range");
    DeviceSceneImpl& d = scene->impl;
    d.tuned_pool = in->path_pool;
    d.tuned_sort = in->sort_mode;
    d.tuned_gen_blocks = in->gen_blocks_per_sm;
    d.tuned_gen_threads = in->gen_threads;
    d.tuned_fin_threads = in->finish_threads;
    d.tuned_fetch = in->extend_fetch;
    d.tuned_queue = in->queue_order;
    d.tuned_shadow_fetch = in->shadow_fetch;
    d.tuned_shadow_sort = in->shadow_sort;
    return ATRC_OK;
}

int atrc_cuda_autotune(AtrcScene* scene, const AtrcRenderDesc* desc, int32_t trial_spp, AtrcTuning* out) {
    const AtrcFilm probe{reinterpret_cast<double*>(1), reinterpret_cast<double*>(1), nullptr, nullptr, nullptr,
                         nullptr, 1, 0};
    const int rc = check_render_args(scene, desc, &probe);
    if (rc != ATRC_OK) return rc;
    return guarded([&] {
        DeviceSceneImpl& d = scene->impl;
        CK(cudaSetDevice(d.device));
        const size_t npix = size_t(desc->width) * desc->height;
        if (d.tune_film.bytes < npix * 4 * sizeof(double)) d.tune_film.alloc(npix * 4 * sizeof(double));
        AtrcFilm film{};
        film.value = d.tune_film.as<double>();
        film.weight = film.value + npix * 3;
        film.on_device = 1;
        AtrcRenderDesc t = *desc;
        // at least three default path pools of samples: the extend-queue
        // order only matters once slots are reused
        const int32_t three_pools = int32_t((3 * (size_t(1) << 21) + npix - 1) / npix);
        t.spp_count = std::min(std::max(trial_spp, three_pools), desc->spp);
        t.first_spp = 0;
        t.count_traversal = 0;
        // pools whose workspace stays under a quarter of the free memory
        size_t free_b = 0, total_b = 0;
        CK(cudaMemGetInfo(&free_b, &total_b));
        const int nl = shadow_rays_per_path(d.scene, *desc);
        const int nkeys = std::max(d.scene.material_count, kMaterialTypes) + 2;
        // (the workspace held now is freed before a larger one is allocated)
        auto pool_fits = [&](int pool) {
            return pool_layout(size_t(pool), size_t(pool) * nl, nkeys).total < (free_b + d.pool_buf.bytes) / 4;
        };
        AtrcTuning cur{};
        tuning_out(d, &cur);
        int trials = 0;
        auto measure = [&](const AtrcTuning& c) {
            atrc_cuda_set_tuning(scene, &c);
            t.sort_mode = ATRC_SORT_AUTO;
            t.path_pool = 0;
            double best = 1e30;
            for (int rep = 0; rep < 2; ++rep) {
                CK(cudaMemsetAsync(d.tune_film.p, 0, npix * 4 * sizeof(double), d.stream));
                AtrcRenderStats st{};
                const int r = render_impl(scene, &t, &film, 1, nullptr, nullptr, nullptr, &st);
                if (r != ATRC_OK) throw CudaError(std::string("autotune trial failed: ") + atrc_last_error());
                best = std::min(best, st.kernel_seconds * 1e3 / (double(st.samples) / 1e6));
                ++trials;
            }
            return best;
        };
        // defaults first (one warm-up trial compiles nothing but pages in)
        AtrcTuning base{1 << 21, ATRC_SORT_NONE, 16, 256, 128, 0, 0, 0, 0, 0};
        if (!pool_fits(base.path_pool)) base.path_pool = 1 << 19;
        measure(base);
        const double base_ms = measure(base);
        AtrcTuning best = base;
        double best_ms = base_ms;
        auto consider = [&](AtrcTuning c) {
            if (!tuning_valid(c) || !pool_fits(c.path_pool)) return;
            const double ms = measure(c);
            if (ms < best_ms * 0.99) { best_ms = ms; best = c; }
        };
        { AtrcTuning c = best; c.extend_fetch = 1; consider(c); }
        const AtrcTuning after_fetch = best;
        for (int q : {0, 1})
            for (int m : {ATRC_SORT_NONE, ATRC_SORT_TYPE, ATRC_SORT_MATERIAL}) {
                AtrcTuning c = after_fetch;
                c.sort_mode = m;
                c.queue_order = q;
                if (q != after_fetch.queue_order || m != after_fetch.sort_mode) consider(c);
            }
        const AtrcTuning after_sort = best;
        for (int pool : {1 << 19, 1 << 20, 1 << 22}) { AtrcTuning c = after_sort; c.path_pool = pool; consider(c); }
        const AtrcTuning after_pool = best;
        const int shapes[][3] = {{8, 256, 128}, {32, 256, 128}, {16, 128, 256}, {16, 512, 128}};
        for (const auto& sh : shapes) {
            AtrcTuning c = after_pool;
            c.gen_blocks_per_sm = sh[0]; c.gen_threads = sh[1]; c.finish_threads = sh[2];
            consider(c);
        }
        { AtrcTuning c = best; c.shadow_sort = 1; consider(c); }
        atrc_cuda_set_tuning(scene, &best);
        d.tuned_trials = trials;
        d.tuned_ms = best_ms;
        d.default_ms = base_ms;
        if (out) tuning_out(d, out);
        return int(ATRC_OK);
    });
}

// ------------------------------------------------------------------------
// Rendering without any allocation.
//
// Some callers cannot allocate device memory at render time: a host that owns
// every byte of the GPU through its own sub-allocator, a process whose memory
// budget is fixed when it starts, or a real-time loop that may not hit the
// driver's allocator (cudaMalloc can synchronise the device and its latency is
// unbounded).  atrc_cuda_render_noalloc serves them: the wavefront's scratch
// memory (path pool, queues, shadow rays, counters) lives in the file-scope
// array below, which every GPU that loads this file's module keeps until the
// process exits.  Under CUDA's lazy module loading (the default since 12.2)
// the module, and with it the array, is loaded onto a device the first time
// the module is used there, which would be an allocation of its own; so
// atrc_cuda_scene_create resolves the array's address on its device, and the
// array is reserved before any render call or stream capture.  The caller
// passes the scene (created beforehand) and a film of device pointers; the
// call itself makes no cudaMalloc / cudaFree / cudaMallocHost and no
// allocating library call.
//
// The array is shared by every call on a device and keeps the previous call's
// contents; the counters and the slot states are rewritten at the start of each
// call, and every other word is written before it is read.  Calls whose work
// overlaps on the GPU (two threads, two streams, or two scenes on the same
// device at once) race on the array: serialise them.
// ------------------------------------------------------------------------
}  // extern "C"

namespace atrc {
namespace {

static __device__ __align__(256) unsigned char g_noalloc_scratch[ATRC_NOALLOC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mutex;
void* g_noalloc_ptr[kMaxDevices] = {};

// Device address of the static scratch array on the current device.  The
// first call on a device looks the symbol up (cudaGetSymbolAddress, which
// also loads the module there under lazy loading); atrc_cuda_scene_create
// makes that first call, outside any stream capture.
void* noalloc_scratch(int device) {
    if (device < 0 || device >= kMaxDevices) throw CudaError("device index out of range for the static scratch");
    std::lock_guard<std::mutex> lk(g_noalloc_mutex);
    if (!g_noalloc_ptr[device]) {
        void* ptr = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
        if (e != cudaSuccess || !ptr)
            throw CudaError(std::string("cudaGetSymbolAddress of the static scratch: ") + cudaGetErrorString(e));
        g_noalloc_ptr[device] = ptr;
    }
    return g_noalloc_ptr[device];
}

}  // namespace
}  // namespace atrc

extern "C" {

int atrc_cuda_render_noalloc(AtrcScene* scene, const AtrcRenderDesc* desc, const AtrcFilm* film,
                             AtrcRenderStats* stats) {
    if (!scene || !desc || !film || !film->value || !film->weight)
        return fail(ATRC_ERR_INVALID_ARG, "atrc_cuda_render_noalloc: null argument");
    if (!film->on_device)
        return fail(ATRC_ERR_INVALID_ARG,
                    "atrc_cuda_render_noalloc: the film must hold device pointers (on_device = 1); a host film "
                    "would need a device staging buffer");
    if (desc->width <= 0 || desc->height <= 0 || desc->spp <= 0 || desc->max_depth < 0 || desc->spp_count < 0 ||
        desc->first_spp < 0)
        return fail(ATRC_ERR_INVALID_ARG, "atrc_cuda_render_noalloc: invalid film size, spp, depth or sample range");
    if (desc->sort_mode < ATRC_SORT_AUTO || desc->sort_mode > ATRC_SORT_MATERIAL)
        return fail(ATRC_ERR_INVALID_ARG, "atrc_cuda_render_noalloc: invalid sort_mode");
    if (desc->filter_type == ATRC_FILTER_BOX ? !(desc->filter_radius - desc->eps > 0)
                                             : !(desc->filter_radius > 0 && desc->filter_alpha > 0))
        return fail(ATRC_ERR_INVALID_ARG, "atrc_cuda_render_noalloc: invalid film filter");
    if (desc->renderer != ATRC_RENDERER_PT && desc->renderer != ATRC_RENDERER_AO)
        return fail(ATRC_ERR_INVALID_ARG, "atrc_cuda_render_noalloc: invalid renderer");
    if (desc->renderer == ATRC_RENDERER_AO && (desc->ao_sample_count <= 0 || desc->ao_sample_count > 4096))
        return fail(ATRC_ERR_INVALID_ARG, "atrc_cuda_render_noalloc: ao_sample_count must be in [1, 4096]");
    if (desc->isect_mode != ATRC_ISECT_FAST && desc->isect_mode != ATRC_ISECT_WATERTIGHT)
        return fail(ATRC_ERR_INVALID_ARG, "atrc_cuda_render_noalloc: isect_mode must be 0 or 2");
    if (desc->renderer == ATRC_RENDERER_PT && !desc->use_mis)
        return fail(ATRC_ERR_UNSUPPORTED,
                    "atrc_cuda_render_noalloc: use_mis = 0 (trace_nomis) is not supported by pt_cuda");
    return guarded([&] {
        DeviceSceneImpl& d = scene->impl;
        CK(cudaSetDevice(d.device));
        void* scratch = noalloc_scratch(d.device);
        cudaStream_t s = d.stream;
        d.scene.eps = desc->eps;
        d.scene.disney_fixed = desc->disney_fixed;
        Params p = make_params(*desc);
        d.resolve_sort(&p, desc->sort_mode);
        View view = make_view(*desc);
        const int spp = desc->spp_count > 0 ? desc->spp_count : desc->spp;
        view.start = 0;
        view.count = (unsigned long long)view.SW * view.SH * spp;
        const unsigned long long total = view.count;
        // the path state packs (view << kTileBits) | tile: a larger tile grid
        // would spill into the view bits
        if (size_t(view.TX) * view.TY >= (size_t(1) << kTileBits))
            return fail(ATRC_ERR_INVALID_ARG, "atrc_cuda_render_noalloc: film too large: more than 2^22 filter tiles");
        const int nl = shadow_rays_per_path(d.scene, *desc);
        const bool wt = desc->isect_mode == ATRC_ISECT_WATERTIGHT;
        // the array holds the counters, the view, the tile tables, then the path pool
        const size_t counters_bytes = 512;
        const size_t view_bytes = (sizeof(View) + 255) & ~size_t(255);
        const size_t tiles_bytes = view_bytes + ((tile_table_bytes(view) + 255) & ~size_t(255));
        if (counters_bytes + tiles_bytes >= ATRC_NOALLOC_SCRATCH_BYTES / 2)
            return fail(ATRC_ERR_INVALID_ARG, "atrc_cuda_render_noalloc: film too large for the static scratch");
        const size_t budget = ATRC_NOALLOC_SCRATCH_BYTES - counters_bytes - tiles_bytes;
        size_t cap = 0;
        for (size_t c = 256; pool_layout(c, c * nl, p.nkeys).total <= budget; c += 256) cap = c;
        if (cap < 1024)
            return fail(ATRC_ERR_UNSUPPORTED, "atrc_cuda_render_noalloc: " + std::to_string(nl) +
                                                  " shadow / occlusion rays per path (one per light for pt, "
                                                  "ao_sample_count for ao) leave room for fewer than 1024 paths in the " +
                                                  std::to_string(ATRC_NOALLOC_SCRATCH_BYTES) + "-byte scratch");
        if (desc->path_pool > 0) {
            if (size_t(desc->path_pool) > cap)
                return fail(ATRC_ERR_INVALID_ARG, "atrc_cuda_render_noalloc: path_pool " +
                                                      std::to_string(desc->path_pool) + " exceeds the maximum " +
                                                      std::to_string(cap) + " that fits the static scratch");
            cap = size_t(desc->path_pool);
        }
        cap = std::min<size_t>(cap, std::max<unsigned long long>(total, 1024ULL));
        const size_t shadow_cap = cap * nl;
        const PoolLayout L = pool_layout(cap, shadow_cap, p.nkeys);
        char* base = static_cast<char*>(scratch);
        Counters* c = reinterpret_cast<Counters*>(base);
        set_tiles(&view, base + counters_bytes + view_bytes);
        view.film = Film{film->value, film->weight, film->value_sq, film->albedo, film->normal, film->denoise};
        View* dview = reinterpret_cast<View*>(base + counters_bytes);
        CK(cudaMemcpyAsync(dview, &view, sizeof(View), cudaMemcpyHostToDevice, s));
        p.nviews = 1;
        p.views = dview;
        p.view_done = nullptr;
        k_tiles<<<1, 32, 0, s>>>(p);
        Pool P = pool_from(base + counters_bytes + tiles_bytes, L, cap, shadow_cap);
        set_shadow_sort(&P, d.scene, d.tuned_shadow_sort);
        const int gsm = grid_for(d.sm_count, d.tuned_gen_blocks);
        const int g_path = int((cap + 127) / 128), g_shadow = shadow_grid(shadow_cap, d.sm_count);
        // k_init rewrites the counters and the slot states (all state that must
        // start from a known value)
        k_init<<<int((std::max<size_t>({cap, size_t(p.nkeys), size_t(kShadowKeys)}) + 255) / 256), 256, 0, s>>>(
            P, int(cap), p.nkeys, c, total);
        CK(cudaGetLastError());
        uint64_t launches = 2, ext_launches = 0;  // k_tiles, k_init
        Counters hc{};
        const auto t0 = std::chrono::steady_clock::now();
        for (;;) {
            for (int k = 0; k < DeviceSceneImpl::kWindow; ++k) {
                k_begin<<<1, 1, 0, s>>>(c);
                k_generate<<<gsm, d.tuned_gen_threads, 0, s>>>(d.scene, p, P, c);
                const int g_fetch = d.sm_count * ATRC_TRACE_MIN_BLOCKS;
                if (d.tuned_fetch && wt)
                    k_extend_fetch<ISECT_WATERTIGHT, false><<<g_fetch, kTraceBlock, 0, s>>>(d.scene, P, c, p.sort_mode, p.nkeys);
                else if (d.tuned_fetch)
                    k_extend_fetch<ISECT_FAST, false><<<g_fetch, kTraceBlock, 0, s>>>(d.scene, P, c, p.sort_mode, p.nkeys);
                else if (wt)
                    k_extend<ISECT_WATERTIGHT, false><<<g_path, 128, 0, s>>>(d.scene, P, c, p.sort_mode, p.nkeys);
                else
                    k_extend<ISECT_FAST, false><<<g_path, 128, 0, s>>>(d.scene, P, c, p.sort_mode, p.nkeys);
                if (p.sort_mode != ATRC_SORT_NONE) {
                    k_sort_scan<<<1, 1024, 0, s>>>(P, p.nkeys);
                    k_sort_scatter<<<d.sm_count * 8, 128, 0, s>>>(P, c, p.nkeys);
                    launches += 2;
                }
                k_shade<<<g_path, 128, 0, s>>>(d.scene, p, P, c);
                if (d.scene.has_subsurface) {
                    k_subsurface<<<g_path, 128, 0, s>>>(d.scene, p, P, c);
                    launches += 1;
                }
                if (P.shadow_sort) {
                    k_shsort_scan<<<1, 1024, 0, s>>>(P);
                    k_shsort_scatter<<<d.sm_count * 8, 128, 0, s>>>(P, c);
                    launches += 2;
                }
                if (d.tuned_shadow_fetch && wt)
                    k_shadow_fetch<ISECT_WATERTIGHT, false><<<g_fetch, kTraceBlock, 0, s>>>(d.scene, P, c);
                else if (d.tuned_shadow_fetch)
                    k_shadow_fetch<ISECT_FAST, false><<<g_fetch, kTraceBlock, 0, s>>>(d.scene, P, c);
                else if (wt)
                    k_shadow<ISECT_WATERTIGHT, false><<<g_shadow, 128, 0, s>>>(d.scene, P, c);
                else
                    k_shadow<ISECT_FAST, false><<<g_shadow, 128, 0, s>>>(d.scene, P, c);
                k_finish<<<gsm, d.tuned_fin_threads, 0, s>>>(p, P, c);
                launches += 6;
                ext_launches += 1;
            }
            CK(cudaGetLastError());
            // plain synchronous copy into a stack variable: no pinned buffer
            CK(cudaStreamSynchronize(s));
            CK(cudaMemcpy(&hc, c, sizeof(Counters), cudaMemcpyDeviceToHost));
            if (hc.watchdog || hc.done) break;
        }
        if (stats) {
            std::memset(stats, 0, sizeof(*stats));
            stats->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
            stats->samples = hc.completed;
            stats->rays_closest = hc.rays_closest;
            stats->rays_shadow = hc.rays_shadow;
            stats->iterations = hc.iterations;
            stats->kernel_launches = launches;
            stats->extend_launches = ext_launches;
            stats->shadow_launches = ext_launches;
            stats->watchdog_flags = uint64_t(hc.watchdog);
        }
        if (hc.watchdog)
            return fail(ATRC_ERR_WATCHDOG, "a device loop reached its iteration cap (code " + std::to_string(hc.watchdog) + ")");
        return int(ATRC_OK);
    });
}

}  // extern "C"
