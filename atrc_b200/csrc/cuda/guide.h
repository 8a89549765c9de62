// Internal interface between the wavefront (render.cu) and the learned guide
// (guide.cu).  Not part of the C ABI.
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "dev_guide.cuh"

namespace atrc {

// One training record: a guided surface vertex and what the rest of its path
// brought back (96 bytes).
struct GuideRecord {
    float pos[3], nrm[3], wo[3], rough;  // the guide's query
    float wi[3], pdf_bsdf;               // sampled direction, BSDF pdf of it
    float coef[3], target;               // path throughput arriving at the vertex; training weight
    float l_arrive[3];                   // path radiance when the next vertex was reached
    int32_t prev;                        // previous record of the same path (-1: none)
    float pad[2];
};
static_assert(sizeof(GuideRecord) == 96, "record layout");

// What the wavefront kernels need from a guide during one render call.
struct GuideFrame {
    // inference inputs / outputs, indexed by shade-queue position
    dev::GuideQuery* queries; // compact list of this iteration's queries
    float* mixes;             // decoded GuideMix, kGuideOut floats per query
    int* gidx;                // per shade-queue entry: its query, or -1
    int max_depth;            // guide vertices up to this depth (0: all)
    uint8_t* xtiles;          // encoded inputs of the queries, 128-row tiles
    const __half* table_h;    // FP16 hash table
    // recording (null when the call does not record)
    GuideRecord* records;
    int* record_count;        // records stored ([0]) and guided vertices seen ([1])
    int record_cap;
    float record_keep;        // probability that a guided vertex is recorded
    int* record_last;         // per path slot: last record of the path
    dev::HashGrid grid;
};

struct GuideImpl;
}  // namespace atrc

struct AtrcGuide;

namespace atrc {
GuideImpl* guide_impl(AtrcGuide* g);

// Size the per-slot buffers for a pool of `cap` paths; returns the frame.
GuideFrame guide_frame(GuideImpl* g, size_t cap, bool record, cudaStream_t s);
// Enqueue the network on the queries whose count is *n_dev.
void guide_infer(GuideImpl* g, const int* n_dev, cudaStream_t s);
// Device of the guide (for checks).
int guide_device(const GuideImpl* g);

}  // namespace atrc
