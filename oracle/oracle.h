/*
 * oracle.h — C ABI of the CPU oracle.
 *
 * TEST INFRASTRUCTURE ONLY.  The oracle is a CPU restatement of the
 * reference's `pt` hot path (AirGuanZ/Atrc, files cited in pt_oracle.cpp).
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may
 * load it, and only as the checker / the timed CPU baseline.  The product
 * (libatrc_cuda.so) never links, loads or calls it.
 *
 * Parity status: pinned to the reference's own code.  The reference ships no
 * tests, golden images or known-answer vectors for this path, and its
 * agz-utils submodule is absent, so oracle/ref/ builds the reference's tracer
 * and factory sources, unchanged, against a compatibility shim for the
 * agz-utils parts they use (vector/matrix/colour types, texture containers,
 * sampling helpers, threads, file loaders) into oracle/_ref/libatrc_ref.so.
 * tests/test_ref_oracle.py checks this restatement against that library
 * (closest hits bit-identical in t where no rotation or nested wrapper is
 * involved; images within the 3-sigma band), and the analytic known-answer
 * tests in tests/ (furnace, slab transmittance, MT edge cases, pdf
 * normalisation) check both.  What remains unpinned is what the shim itself
 * restates: agz-utils' matrix inverse / rotation rounding and its sampling
 * helpers' exact sequences (they are distribution-level equal, not
 * bit-equal).
 */
#ifndef ATRC_ORACLE_H
#define ATRC_ORACLE_H

#include "../include/atrc_cuda.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct OracleScene OracleScene;

const char* oracle_last_error(void);

/* Build the reference's object graph from a flattened scene: per-mesh
 * midpoint/median BVH (triangle_bvh.cpp:122-304), entity BVH or native
 * aggregate (entity_bvh.cpp:46-116, native_aggregate.cpp), lights in the
 * order of scene_default.cpp:66-82.  `eps` is the scene epsilon. */
int oracle_scene_create(const AtrcSceneDesc* desc, float eps, OracleScene** out);
void oracle_scene_destroy(OracleScene* s);

/* Closest / any hit for each ray (Scene::closest_intersection /
 * has_intersection).  `isect` is ATRC_ISECT_EXACT (the reference's
 * Moller-Trumbore) or ATRC_ISECT_WATERTIGHT (the watertight triangle test and
 * cancellation-free sphere roots, not in the reference).  `threads` <= 0 uses
 * all hardware threads. */
int oracle_trace_rays(OracleScene* s, const AtrcRay* rays, size_t n,
                      AtrcHit* hits, int mode, int isect, int threads);

/* The `isect` test of one primitive of one entity against a world ray (ray
 * moved to the entity's local space as transform_wrapper does).  Writes t (or
 * -1 when the primitive is not hit).  Used to adjudicate hit mismatches. */
int oracle_prim_hit(OracleScene* s, const AtrcRay* ray, int entity, int prim,
                    int isect, float* t_out);

/* Render with the reference's `pt` algorithm (perpixel_renderer.cpp:13-53 +
 * path_tracing.cpp:15-225) and ADD into `film` (host pointers).  Samples
 * [desc->first_spp, first_spp + spp_count) of every pixel are taken; tile
 * random streams are seeded from (desc->seed, sample range, tile). */
int oracle_render(OracleScene* s, const AtrcRenderDesc* desc, AtrcFilm* film,
                  int threads);

/* Same, on a uniform spatial sample: only every `tile_stride`-th 32x32 tile
 * (in row-major tile order) is rendered.  Used to time a bounded sample of a
 * large workload. */
int oracle_render_sample(OracleScene* s, const AtrcRenderDesc* desc, AtrcFilm* film,
                         int threads, int tile_stride);

/* Number of hardware threads the oracle would use for threads <= 0. */
int oracle_hardware_threads(void);

/* Environment-light pdf / radiance probes (ibl.cpp, env_sampler.h), used by
 * the pdf-normalisation known-answer test. */
int oracle_env_pdf(OracleScene* s, const float* dirs, size_t n, float* pdf);
int oracle_env_sample(OracleScene* s, const float* u3, size_t n, float* dirs,
                      float* pdf);

/* BSDF probes on a synthetic shading point (geometric frame = shading frame =
 * world axes).  material: index into the scene's materials.  For each i:
 * eval f(wi, wo) -> f[3], pdf(wi, wo) -> pdf. */
int oracle_bsdf_eval(OracleScene* s, int material, const float* wi,
                     const float* wo, size_t n, float* f, float* pdf);
/* sample(wo, u3) -> wi[3], f[3], pdf, delta; disney_fixed selects the
 * fixed Disney sampling mode of pt_cuda (0 = the reference's sampler) */
int oracle_bsdf_sample(OracleScene* s, int material, const float* wo,
                       const float* u3, size_t n, float* wi, float* f,
                       float* pdf, int* is_delta, int disney_fixed);
/* Subsurface probe (SeparableBSSRDF::sample_pi) from the closest hit of the
 * ray (o, d), which must meet an entity whose material has subsurface
 * scattering: n samples of the weight coef / pdf -> w[3] (0 when the
 * sample is invalid) and the exit point -> exit_pos[3]. */
int oracle_subsurface(OracleScene* s, const float* o, const float* d, size_t n, uint64_t seed,
                      float* w, float* exit_pos);

#ifdef __cplusplus
}
#endif

#endif
