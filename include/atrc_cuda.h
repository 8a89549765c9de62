/*
 * atrc_cuda.h — C ABI of the B200 path tracer (`pt_cuda`).
 *
 * Two layers live behind this header, both exported from libatrc_cuda.so:
 *
 *  1. Scene ingestion (host only, no GPU needed).  The Atrc JSON scene format
 *     is parsed by a factory that mirrors the reference's creators and is
 *     flattened into the POD `AtrcSceneDesc` below.  This replaces the
 *     reference's `CreatingContext::create<Scene>` path
 *     (src/factory/include/agz/factory/context.h:280-300,
 *      src/factory/src/creator/scene_creators.cpp:24-65) plus the parsing of
 *     `rendering` settings (src/factory/src/utility/render_session.cpp:14-66).
 *
 *  2. Device execution.  `atrc_cuda_scene_create` uploads a scene and builds the
 *     device acceleration structure; `atrc_cuda_trace_rays` replaces
 *     `Scene::closest_intersection / has_intersection`
 *     (src/tracer/include/agz/tracer/core/scene.h, aggregate.h;
 *      src/tracer/src/core/scene/scene_default.cpp:136-147) for batches of rays;
 *     `atrc_cuda_render` replaces `Renderer::render` of the `pt` renderer
 *     (src/tracer/include/agz/tracer/core/renderer.h:33-35,
 *      src/tracer/src/core/renderer/pt.cpp:8-48,
 *      src/tracer/src/core/renderer/perpixel_renderer.cpp:13-207).
 *
 * Conventions
 *  - Every function returns int: 0 on success, a negative AtrcStatus on error.
 *    The message of the last error on the calling thread is available from
 *    atrc_last_error().
 *  - Handles are opaque, owned by the caller, and destroyed explicitly.
 *  - Calls block the calling thread.  One CUDA stream per device scene is used
 *    internally.  A scene handle is not re-entrant; distinct handles may be
 *    used from distinct threads.
 *  - Vectors are float[3] (x, y, z); colours are float[3] (r, g, b).
 *  - Affine transforms are row-major 3x4 matrices m[12]: row r = (m[4r+0],
 *    m[4r+1], m[4r+2], m[4r+3]); p' = M[:, :3] p + M[:, 3].
 */
#ifndef ATRC_CUDA_H
#define ATRC_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ATRC_ABI_VERSION 2

/* ---------------------------------------------------------------- status */

typedef enum AtrcStatus {
    ATRC_OK               = 0,
    ATRC_ERR_INVALID_ARG  = -1,  /* bad pointer, size or enum value          */
    ATRC_ERR_CONFIG       = -2,  /* malformed JSON / unknown creator / file  */
    ATRC_ERR_OUT_OF_MEMORY= -3,  /* host or device allocation failed         */
    ATRC_ERR_CUDA         = -4,  /* CUDA runtime error or no usable device   */
    ATRC_ERR_CANCELLED    = -5,  /* the cancel callback asked to stop        */
    ATRC_ERR_WATCHDOG     = -6,  /* a device loop hit its iteration cap      */
    ATRC_ERR_UNSUPPORTED  = -7   /* scene feature outside pt_cuda's support  */
} AtrcStatus;

/* ---------------------------------------------------------- scene format */

typedef struct AtrcTransform {
    float m[12];    /* local -> world, row-major 3x4                         */
    float inv[12];  /* world -> local, row-major 3x4 (computed on the host)  */
} AtrcTransform;

/* Triangle mesh in the reference's `.bm` memory layout: per triangle three
 * vertices of {position[3], normal[3], tex_coord[2]} floats (96 bytes), in the
 * file's original order (src/factory/src/utility/bin_mesh.cpp:7-27). */
typedef struct AtrcMeshDesc {
    uint64_t     triangle_count;
    const float* vertices;      /* triangle_count * 24 floats */
} AtrcMeshDesc;

typedef enum AtrcGeometryType {
    ATRC_GEOM_TRIANGLE_BVH = 0,  /* mesh, vertices baked by `transform`      */
    ATRC_GEOM_TRIANGLE     = 1,  /* single triangle, ray moved to local space*/
    ATRC_GEOM_QUAD         = 2,  /* ABC + ACD, vertices baked by `transform` */
    ATRC_GEOM_SPHERE       = 3,  /* radius around local origin               */
    ATRC_GEOM_DISK         = 4   /* radius, local z = normal                 */
} AtrcGeometryType;

/* A leaf geometry as created by its creator
 * (src/factory/src/creator/geometry_creators.cpp).  Leaf geometries may be
 * shared by several entities through the `reference` creator. */
typedef struct AtrcGeometryDesc {
    int32_t       type;          /* AtrcGeometryType                         */
    int32_t       mesh;          /* index into meshes (TRIANGLE_BVH)         */
    AtrcTransform transform;     /* the geometry's own `transform` list      */
    float         p[4][3];       /* A, B, C (, D) for TRIANGLE / QUAD        */
    float         uv[4][2];      /* tA, tB, tC (, tD)                        */
    float         radius;        /* SPHERE / DISK                            */
    int32_t       pad_;
} AtrcGeometryDesc;

/* A `geometric` entity (src/tracer/src/core/entity/geometric.cpp:10-58).
 * The entity's geometry chain is flattened into: an optional instance
 * transform (`transform_wrapper`, transform_wrapper.cpp:51-68), an optional
 * `double_sided` adapter, and a leaf geometry. */
typedef struct AtrcEntityDesc {
    int32_t       geometry;      /* leaf geometry index                      */
    int32_t       has_instance;  /* 1 if wrapped by transform_wrapper        */
    AtrcTransform instance;      /* transform_wrapper local -> world         */
    int32_t       double_sided;  /* 1 if wrapped by double_sided             */
    int32_t       material;      /* material index                           */
    int32_t       medium_in;     /* medium index (0 = the void medium)       */
    int32_t       medium_out;
    float         emit_radiance[3];
    int32_t       no_denoise;
    float         power;         /* user light power, <= 0 means automatic   */
    int32_t       pad_;
} AtrcEntityDesc;

typedef enum AtrcTextureType {
    ATRC_TEX_CONSTANT = 0,
    ATRC_TEX_IMAGE    = 1,       /* float RGB texels (`hdr`, `image`)        */
    ATRC_TEX_CHECKER  = 2,       /* `checker_board`: texel = color1,         */
                                 /* texel2 = color2, grid_count cells        */
    ATRC_TEX_SOLID    = 3        /* `solid_image` (solid_image.cpp:6-45):    */
                                 /* the texture3d `tex3d` read at (u, v, 0), */
                                 /* or at the world position where the       */
                                 /* material passes the intersection (ideal  */
                                 /* diffuse albedo, glass maps)              */
} AtrcTextureType;

typedef enum AtrcWrapMode {
    ATRC_WRAP_CLAMP = 0, ATRC_WRAP_REPEAT = 1, ATRC_WRAP_MIRROR = 2
} AtrcWrapMode;

/* Texture2D (src/tracer/include/agz/tracer/core/texture2d.h:55-174). */
typedef struct AtrcTexture2DDesc {
    int32_t      type;           /* AtrcTextureType                          */
    float        texel[3];       /* CONSTANT                                 */
    int32_t      width, height;  /* IMAGE                                    */
    const float* data;           /* IMAGE: height rows of width RGB floats,  */
                                 /* row 0 is v = 0                           */
    int32_t      nearest;        /* 1 = nearest, 0 = bilinear                */
    float        uv_transform[6];/* 2x3 row-major affine applied to uv       */
    int32_t      wrap_u, wrap_v; /* AtrcWrapMode                             */
    float        inv_gamma;
    int32_t      grid_count;     /* CHECKER                                  */
    float        texel2[3];      /* CHECKER                                  */
    int32_t      tex3d;          /* SOLID: texture3d index                   */
} AtrcTexture2DDesc;

/* Texture3D (src/tracer/include/agz/tracer/core/texture3d.h:30-223). */
typedef struct AtrcTexture3DDesc {
    int32_t      type;           /* AtrcTextureType                          */
    float        texel[3];
    int32_t      width, height, depth;
    int32_t      channels;       /* 1 (real/gray8) or 3 (spec/rgb8)          */
    const float* data;           /* depth x height x width x channels, z-major */
    int32_t      nearest;
    float        uvw_transform[12]; /* 3x4 row-major affine on uvw          */
    int32_t      uvw_perm[3];
    int32_t      wrap[3];
    float        inv_gamma;
    float        max_real;       /* max over texels of the real channel      */
} AtrcTexture3DDesc;

typedef enum AtrcMaterialType {
    ATRC_MAT_IDEAL_DIFFUSE     = 0,
    ATRC_MAT_IDEAL_BLACK       = 1,
    ATRC_MAT_DISNEY            = 2,
    ATRC_MAT_INVISIBLE_SURFACE = 3,
    ATRC_MAT_MIRROR            = 4,  /* tex[0] color_map, tex[1] eta, tex[2] k        */
    ATRC_MAT_GLASS             = 5,  /* tex[0] reflection color, tex[1] refraction     */
                                     /* color, tex[2] ior                             */
    ATRC_MAT_METAL             = 6,  /* tex[0] color, tex[1] eta, tex[2] k,           */
                                     /* tex[3] roughness, tex[4] anisotropic          */
    ATRC_MAT_PHONG             = 7   /* tex[0] d, tex[1] s, tex[2] ns                 */
} AtrcMaterialType;

/* Disney texture slots, in the order of create_disney
 * (src/factory/src/creator/material_creators.cpp:56-113). */
typedef enum AtrcDisneySlot {
    ATRC_DISNEY_BASE_COLOR = 0, ATRC_DISNEY_METALLIC, ATRC_DISNEY_ROUGHNESS,
    ATRC_DISNEY_TRANSMISSION, ATRC_DISNEY_TRANSMISSION_ROUGHNESS,
    ATRC_DISNEY_IOR, ATRC_DISNEY_SPECULAR_SCALE, ATRC_DISNEY_SPECULAR_TINT,
    ATRC_DISNEY_ANISOTROPIC, ATRC_DISNEY_SHEEN, ATRC_DISNEY_SHEEN_TINT,
    ATRC_DISNEY_CLEARCOAT, ATRC_DISNEY_CLEARCOAT_GLOSS,
    ATRC_DISNEY_SLOT_COUNT
} AtrcDisneySlot;

typedef struct AtrcMaterialDesc {
    int32_t type;                    /* AtrcMaterialType                      */
    int32_t tex[ATRC_DISNEY_SLOT_COUNT]; /* texture2d indices; IDEAL_DIFFUSE */
                                     /* uses tex[0] as albedo                */
    int32_t normal_map;              /* texture2d index or -1                */
    int32_t bssrdf[3];               /* DISNEY subsurface scattering         */
                                     /* (init_bssrdf_surface, material_      */
                                     /* creators.cpp:20-45): texture2d       */
                                     /* indices of A, dmfp and eta; -1 each  */
                                     /* when the material has none           */
} AtrcMaterialDesc;

typedef enum AtrcMediumType {
    ATRC_MED_VOID = 0, ATRC_MED_HOMOGENEOUS = 1, ATRC_MED_HETEROGENEOUS = 2
} AtrcMediumType;

typedef struct AtrcMediumDesc {
    int32_t       type;              /* AtrcMediumType                       */
    float         sigma_a[3];        /* HOMOGENEOUS                          */
    float         sigma_s[3];
    float         g;
    int32_t       max_scattering_count;
    AtrcTransform transform;         /* HETEROGENEOUS: texture space -> world*/
    int32_t       density, albedo, g_tex;  /* texture3d indices             */
    int32_t       white_for_indirect;      /* heterogeneous.cpp:107-110     */
} AtrcMediumDesc;

typedef enum AtrcEnvType {
    ATRC_ENV_NONE = 0, ATRC_ENV_IBL = 1, ATRC_ENV_NATIVE_SKY = 2
} AtrcEnvType;

typedef struct AtrcEnvDesc {
    int32_t type;                    /* AtrcEnvType                          */
    int32_t tex;                     /* IBL texture2d index                  */
    int32_t no_importance_sampling;
    float   power;
    float   top[3], bottom[3];       /* NATIVE_SKY                           */
} AtrcEnvDesc;

typedef enum AtrcAggregateType {
    ATRC_AGG_NATIVE = 0, ATRC_AGG_BVH = 1
} AtrcAggregateType;

/* Builder of the per-mesh bottom-level trees of the device scene.  Hit
 * results do not depend on it; traversal cost and build time do. */
typedef enum AtrcBvhBuilder {
    ATRC_BVH_SAH  = 0,  /* binned SAH on the host (threads at the top levels)   */
    ATRC_BVH_PLOC = 1,  /* parallel locally-ordered clustering on the device    */
    ATRC_BVH_AUTO = 2   /* PLOC for meshes of at least 2^18 triangles, else SAH */
} AtrcBvhBuilder;

typedef struct AtrcSceneDesc {
    uint32_t abi_version;            /* ATRC_ABI_VERSION                     */
    int32_t  aggregate;              /* AtrcAggregateType (CPU semantics)    */
    int32_t  aggregate_max_leaf_size;
    int32_t  bvh_builder;            /* AtrcBvhBuilder (pt_cuda scene key    */
                                     /* "bvh_builder": sah / ploc / auto)    */
    const AtrcMeshDesc*      meshes;     uint32_t mesh_count;
    const AtrcGeometryDesc*  geometries; uint32_t geometry_count;
    const AtrcEntityDesc*    entities;   uint32_t entity_count;
    const AtrcMaterialDesc*  materials;  uint32_t material_count;
    const AtrcTexture2DDesc* textures2d; uint32_t texture2d_count;
    const AtrcTexture3DDesc* textures3d; uint32_t texture3d_count;
    const AtrcMediumDesc*    media;      uint32_t medium_count; /* [0]=void */
    AtrcEnvDesc env;
} AtrcSceneDesc;

/* ------------------------------------------------------ render settings */

typedef enum AtrcFilterType { ATRC_FILTER_BOX = 0, ATRC_FILTER_GAUSSIAN = 1 } AtrcFilterType;

typedef struct AtrcCameraDesc {      /* thin_lens (thin_lens.cpp:34-94)      */
    float pos[3], dst[3], up[3];
    float fov;                       /* radians, vertical                    */
    float lens_radius;
    float focal_distance;
} AtrcCameraDesc;

typedef struct AtrcRenderDesc {
    int32_t  width, height;
    int32_t  spp;
    int32_t  min_depth, max_depth;   /* pt keys (renderer_creators.cpp:127-146) */
    float    cont_prob;
    int32_t  specular_depth;
    int32_t  use_mis;                /* 1: trace_std (MIS).  0 selects the
                                        reference's trace_nomis, which is not
                                        built: renders of a pt entry with
                                        use_mis = 0 return
                                        ATRC_ERR_UNSUPPORTED                 */
    int32_t  filter_type;            /* AtrcFilterType                       */
    float    filter_radius;          /* user radius (box: 0.5 by default)    */
    float    filter_alpha;           /* gaussian                             */
    float    eps;                    /* scene epsilon (default 3e-4)         */
    uint64_t seed;                   /* random stream selector               */
    int32_t  first_spp;              /* render sample indices                */
    int32_t  spp_count;              /* [first_spp, first_spp + spp_count)   */
                                     /* of every pixel; 0 means all of spp   */
    AtrcCameraDesc camera;
    int32_t  path_pool;              /* wavefront path capacity, 0 = auto    */
    int32_t  count_traversal;        /* 1: count BVH work into the stats     */
                                     /* (slower; for roofline accounting)    */
    int32_t  task_grid_size;         /* pt key (default 32): the film filter */
                                     /* splats per tile of this edge, and    */
                                     /* pixels near a tile edge are sampled  */
                                     /* once per tile (render_target.h:      */
                                     /* 355-395); 0 means 32                 */
    int32_t  sort_mode;              /* order of the shade queue: ATRC_SORT_* */
    int32_t  disney_fixed;           /* 0: Disney sampling as the reference  */
                                     /* (its diffuse-lobe choice falls       */
                                     /* through, disney.cpp:578-589, so the  */
                                     /* samples do not follow the reported   */
                                     /* pdf); 1: the diffuse lobe is sampled */
                                     /* (sampling matches the pdf; needed by */
                                     /* guided rendering and error studies)  */
    int32_t  renderer;               /* AtrcRendererType                     */
    /* `ao` renderer keys (renderer_creators.cpp:19-38, trace_ao in         */
    /* path_tracing.cpp:383-415): a pixel is lerp(low, high, fraction of    */
    /* ao_sample_count cosine-distributed rays from the first hit that are  */
    /* not blocked within ao_max_distance); background on a miss            */
    int32_t  ao_sample_count;        /* default 5                            */
    float    ao_max_distance;        /* max_occlusion_distance, default 1    */
    float    ao_low[3];              /* low_color, default 0                 */
    float    ao_high[3];             /* high_color, default 1                */
    float    ao_background[3];       /* background_color, default 0          */
    int32_t  isect_mode;             /* ray-triangle test of the render:     */
                                     /* ATRC_ISECT_FAST (Moller-Trumbore,    */
                                     /* the reference's test) or             */
                                     /* ATRC_ISECT_WATERTIGHT                */
} AtrcRenderDesc;

/* Renderer of a render call. */
typedef enum AtrcRendererType {
    ATRC_RENDERER_PT = 0,   /* `pt` / `pt_cuda`: volumetric path tracing with NEE and MIS */
    ATRC_RENDERER_AO = 1    /* `ao`: ambient occlusion                                   */
} AtrcRendererType;

/* Sorting of hit records before shading (a counting sort by key). */
typedef enum AtrcSortMode {
    ATRC_SORT_AUTO     = -1,  /* the scene's tuned choice, else ATRC_SORT_NONE */
    ATRC_SORT_NONE     = 0,   /* shade in extend-queue order                   */
    ATRC_SORT_TYPE     = 1,   /* by material type (miss / each type / medium)  */
    ATRC_SORT_MATERIAL = 2    /* by material index (miss / each / medium)      */
} AtrcSortMode;

/* FP64 film accumulators, caller allocated, `width*height` pixels each.
 * Any pointer except `value` and `weight` may be NULL.  The renderer ADDS
 * into them (so several calls accumulate); the image is value / weight. */
typedef struct AtrcFilm {
    double* value;     /* 3 per pixel: sum of w * L                          */
    double* weight;    /* 1 per pixel: sum of w                              */
    double* value_sq;  /* 3 per pixel: sum of w * L^2 (for variance tests)   */
    double* albedo;    /* 3 per pixel: sum of w * first-hit albedo           */
    double* normal;    /* 3 per pixel: sum of w * first-hit shading normal   */
    double* denoise;   /* 1 per pixel: sum of w * denoise flag               */
    int32_t on_device; /* 1 if the pointers above are device pointers        */
    int32_t pad_;
} AtrcFilm;

typedef struct AtrcRenderStats {
    double   seconds;          /* wall time of the render call               */
    double   kernel_seconds;   /* device time of the wavefront loop          */
    uint64_t samples;          /* camera samples completed                   */
    uint64_t rays_closest;     /* closest-hit rays traced                    */
    uint64_t rays_shadow;      /* any-hit (shadow) rays traced               */
    uint64_t iterations;       /* wavefront iterations                       */
    uint64_t kernel_launches;  /* kernels launched by this call              */
    uint64_t watchdog_flags;   /* device loops that hit their caps           */
    double   extend_seconds;   /* device time inside closest-hit kernels     */
    double   shadow_seconds;   /* device time inside any-hit kernels         */
    double   shade_seconds;    /* device time inside shading kernels         */
    uint64_t h2d_bytes, d2h_bytes;
    uint64_t extend_launches;  /* closest-hit kernel launches               */
    uint64_t shadow_launches;  /* any-hit kernel launches                   */
    uint64_t nodes_closest, tris_closest, ents_closest;  /* count_traversal  */
    uint64_t nodes_shadow, tris_shadow, ents_shadow;
} AtrcRenderStats;

/* Progress callback, fired on the calling thread between wavefront
 * iterations with a percentage in [0, 100]. */
typedef void (*AtrcProgressFn)(double percent, void* user);

/* Cancel poll, called on the calling thread between wavefront iterations;
 * a non-zero return stops the render.  The reference's cancel flag is a
 * `std::atomic<bool> stop_rendering_` member of Renderer
 * (src/tracer/include/agz/tracer/core/renderer.h:20), which C cannot read
 * portably; a binding returns `stop_rendering_.load()` from this callback. */
typedef int (*AtrcCancelFn)(void* user);

/* ------------------------------------------------------------ ray queries */

typedef struct AtrcRay {       /* 32 bytes */
    float o[3];
    float t_min;
    float d[3];                /* not necessarily normalised                 */
    float t_max;
} AtrcRay;

typedef struct AtrcHit {       /* 16 bytes */
    float    t;                /* hit distance; -1 when nothing was hit      */
    int32_t  entity;           /* entity index or -1                         */
    int32_t  prim;             /* ORIGINAL triangle index within the mesh,   */
                               /* 0/1 = quad half ABC/ACD, 0 otherwise       */
    float    u;                /* barycentric alpha (or 0)                   */
} AtrcHit;

typedef enum AtrcQueryMode { ATRC_QUERY_CLOSEST = 0, ATRC_QUERY_ANY = 1 } AtrcQueryMode;

/* Ray-primitive tests.  The reference uses Moller-Trumbore
 * (src/tracer/include/agz/tracer/utility/triangle_aux.h:9-69), which can let
 * a ray through an edge or vertex shared by two triangles miss both. */
typedef enum AtrcIsectMode {
    ATRC_ISECT_FAST       = 0,  /* Moller-Trumbore, compiler-scheduled (FMAs)   */
    ATRC_ISECT_EXACT      = 1,  /* Moller-Trumbore in the reference's operation */
                                /* order without FMAs: bit-identical hits       */
    ATRC_ISECT_WATERTIGHT = 2   /* Woop, Benthin and Wald's watertight test     */
                                /* (JCGT 2(1), 2013) on the exact vertices, and */
                                /* sphere roots without cancellation            */
} AtrcIsectMode;

/* ------------------------------------------------------------- functions */

typedef struct AtrcConfig AtrcConfig;   /* parsed JSON config (host)        */
typedef struct AtrcScene  AtrcScene;    /* device scene                     */

typedef struct AtrcDeviceInfo {
    char    name[128];
    int32_t sm_count;
    int32_t cc_major, cc_minor;
    int32_t pad_;
    uint64_t global_mem_bytes;
} AtrcDeviceInfo;

/* Version of the ABI the library was built with. */
int atrc_abi_version(void);

/* sizeof of the ABI structs as compiled into the library, in this order:
 * AtrcSceneDesc, AtrcMeshDesc, AtrcGeometryDesc, AtrcEntityDesc,
 * AtrcTexture2DDesc, AtrcTexture3DDesc, AtrcMaterialDesc, AtrcMediumDesc,
 * AtrcEnvDesc, AtrcRenderDesc, AtrcFilm, AtrcRenderStats, AtrcRay, AtrcHit,
 * AtrcDeviceInfo.  Writes min(n, 15) values; returns 15.  Lets bindings in
 * other languages verify their struct layouts. */
int atrc_abi_struct_sizes(uint64_t* sizes, int n);

/* Thread-local message of the last failing call ("" if none). */
const char* atrc_last_error(void);

/* Parse an Atrc JSON configuration ({"scene": ..., "rendering": ...}) from a
 * file.  `${scene-directory}` maps to the file's directory and
 * `${working-directory}` to the current directory (src/cli/src/main.cpp:29-41).
 * Replaces json_to_config + CreatingContext::create<Scene>. */
int atrc_config_load_file(const char* path, AtrcConfig** out);

/* Same, from a JSON string; `scene_dir` stands for ${scene-directory}. */
int atrc_config_load_string(const char* json, const char* scene_dir,
                            AtrcConfig** out);

void atrc_config_destroy(AtrcConfig* cfg);

/* Flattened scene owned by `cfg` (valid until atrc_config_destroy). */
int atrc_config_scene(const AtrcConfig* cfg, const AtrcSceneDesc** out);

/* Number of `rendering` entries (1 for an object, N for an array). */
int atrc_config_rendering_count(const AtrcConfig* cfg, int* out);

/* Rendering settings of entry `index`.  `renderer_type` receives the
 * renderer's `type` string (e.g. "pt" or "pt_cuda"), at most cap bytes. */
int atrc_config_rendering(const AtrcConfig* cfg, int index,
                          AtrcRenderDesc* out,
                          char* renderer_type, size_t cap);

/* Post-processing list of entry `index` as a JSON text (for the CLI). */
int atrc_config_post_processors(const AtrcConfig* cfg, int index,
                                char* json_out, size_t cap, size_t* needed);

/* Query device 0..N-1 and make it current for this thread. */
int atrc_cuda_device_init(int device, AtrcDeviceInfo* info);

/* Upload a scene and build its acceleration structure on the current device.
 * The description is copied; the caller may free it afterwards. */
int atrc_cuda_scene_create(const AtrcSceneDesc* desc, AtrcScene** out);

void atrc_cuda_scene_destroy(AtrcScene* scene);

/* Trace `n` rays from host memory into host `hits`.  mode: AtrcQueryMode.
 * ANY mode writes t = 1 / entity = 0 for an occluded ray and t = -1 otherwise.
 * `exact` is an AtrcIsectMode: 1 selects the reference-exact Moller-Trumbore
 * test (same operation order, no fused multiply-add), 0 the fast test, 2 the
 * watertight test. */
int atrc_cuda_trace_rays(AtrcScene* scene, const AtrcRay* rays, size_t n,
                         AtrcHit* hits, int mode, int exact);

/* Same with device pointers (no copies). */
int atrc_cuda_trace_rays_device(AtrcScene* scene, const AtrcRay* d_rays,
                                size_t n, AtrcHit* d_hits, int mode, int exact);

/* Render `desc` (a pt_cuda / pt configuration) and ADD the samples into
 * `film`.  `should_stop` (may be NULL) is called with `user` between
 * wavefront iterations; a non-zero return ends the call with
 * ATRC_ERR_CANCELLED after the samples already taken are in the film (this
 * is the contract of Renderer::render_async / stop_async,
 * src/tracer/src/core/core/renderer.cpp:5-38).
 * `progress` (may be NULL) is called with the same `user` on this thread. */
int atrc_cuda_render(AtrcScene* scene, const AtrcRenderDesc* desc,
                     AtrcFilm* film, AtrcCancelFn should_stop,
                     AtrcProgressFn progress, void* user,
                     AtrcRenderStats* stats);

/* Launch configuration of the wavefront for one scene: the values that
 * renders with `path_pool` 0 and `sort_mode` ATRC_SORT_AUTO use. */
typedef struct AtrcTuning {
    int32_t path_pool;          /* paths in flight (queue capacity)              */
    int32_t sort_mode;          /* AtrcSortMode, never ATRC_SORT_AUTO            */
    int32_t gen_blocks_per_sm;  /* grid of the generate / finish kernels per SM  */
    int32_t gen_threads;        /* block size of the camera-ray generator        */
    int32_t finish_threads;     /* block size of the film splat                  */
    int32_t trials;             /* trial renders measured by the last autotune   */
    double  ms_per_msample;     /* device ms per million samples, chosen config  */
    double  default_ms_per_msample; /* the same for the built-in defaults        */
    int32_t extend_fetch;       /* closest-hit traversal: 1 = persistent warps   */
                                /* that refill finished lanes with new rays, 0 = */
                                /* one ray per thread                            */
    int32_t queue_order;        /* extend queue: 0 = continuing paths in the     */
                                /* order they were shaded, then new samples; 1 = */
                                /* every queued path in ascending slot order     */
    int32_t shadow_fetch;       /* any-hit traversal: 1 = persistent warps that  */
                                /* refill finished lanes, 0 = one ray per thread */
                                /* (set by the caller; the autotuner leaves 0)   */
    int32_t shadow_sort;        /* shadow queue: 1 = counting sort by the cell   */
                                /* of the ray origin (16^3 over the scene bound, */
                                /* Morton order) before any-hit traversal, so a  */
                                /* warp's rays start near each other; 0 = order  */
                                /* of shading                                    */
} AtrcTuning;

/* Project autotuner (the reference has no counterpart: it renders with a
 * fixed thread pool and 32x32 tiles, renderer_creators.cpp:127-128).  Renders
 * short trials of `desc` into scratch memory, each max(trial_spp, the spp
 * of three default path pools = 3 * 2^21 samples) samples per pixel, capped
 * at desc->spp (the extend-queue order only matters once path slots are
 * reused).  It searches the closest-hit kernel (extend_fetch), sort
 * granularity with the extend-queue order
 * (queue_order), then path-pool size, then the generate / finish launch
 * shapes, then the shadow-queue sort (coordinate descent, best of two
 * timings each), and stores the fastest configuration in the scene.  The
 * caller's films are untouched. */
int atrc_cuda_autotune(AtrcScene* scene, const AtrcRenderDesc* desc,
                       int32_t trial_spp, AtrcTuning* out);
/* Read or replace a scene's launch configuration (e.g. a cached tuning). */
int atrc_cuda_get_tuning(AtrcScene* scene, AtrcTuning* out);
int atrc_cuda_set_tuning(AtrcScene* scene, const AtrcTuning* in);

/* Streaming-read bandwidth (GB/s) of `device`: a zero-filled buffer of
 * `bytes` (a multiple of 16, at least 1 MiB) read `passes` (>= 2) times with
 * 16-byte loads that bypass L1, after one untimed pass, timed with CUDA
 * events.  A buffer of a few tens of MB stays in L2 and measures L2 read
 * bandwidth; one of several GB measures HBM.  The roofline denominator of
 * the traversal kernels, whose working set is served from L1 and L2.  No
 * counterpart in the reference (it has no GPU code). */
int atrc_cuda_stream_read_gbs(int device, uint64_t bytes, int passes, double* gbs);

/* Size of the static device array behind atrc_cuda_render_noalloc. */
#define ATRC_NOALLOC_SCRATCH_BYTES (24u * 1024u * 1024u)

/* atrc_cuda_render without any memory allocation, for callers that cannot
 * allocate device memory at render time (a host that sub-allocates the whole
 * GPU itself, a process with a memory budget fixed at start-up, a real-time
 * loop that must not enter the driver's allocator).  No counterpart in the
 * reference, whose CPU renderer allocates per tile and per sample.
 *  - The wavefront scratch (path pool, queues, shadow rays, counters) lives in
 *    a static device array of ATRC_NOALLOC_SCRATCH_BYTES that every GPU which
 *    loads this library keeps reserved until the process exits.  A path
 *    takes 192 bytes plus 56 per shadow ray it may emit in one iteration (one
 *    per light for pt, ao_sample_count for ao), so the pool holds about 100k
 *    paths with one light.  Calls that leave room for fewer than 1024 paths
 *    (more than 434 lights, or ao_sample_count above 434) are rejected with
 *    ATRC_ERR_UNSUPPORTED; a desc->path_pool above the maximum, and a film
 *    of 2^22 or more filter tiles, with ATRC_ERR_INVALID_ARG.  Nothing is
 *    launched before these checks.
 *  - `film` must hold device pointers (on_device = 1); samples are added.
 *  - Under CUDA's lazy module loading the array is reserved on a device when
 *    the library's module is first loaded there; atrc_cuda_scene_create
 *    loads it and looks up the array's device address on the scene's device,
 *    so this call neither allocates nor looks anything up.  Create the scene
 *    before capturing any stream.
 *  - The launch shapes and traversal kernels are the scene's tuning
 *    (atrc_cuda_autotune / atrc_cuda_set_tuning), as for atrc_cuda_render.
 *  - All calls share the array and it keeps the last call's contents (each
 *    call resets the counters it needs).  Calls that overlap on the GPU race
 *    on it: serialise them.
 *  - No progress callback or cancel flag; stats carries counts but no
 *    per-kernel timings.
 * Same status codes as atrc_cuda_render. */
int atrc_cuda_render_noalloc(AtrcScene* scene, const AtrcRenderDesc* desc,
                             const AtrcFilm* film, AtrcRenderStats* stats);

/* Write a resolved film (rgb, row 0 = bottom, as produced by
 * atrc_film_resolve) the way the `save_to_img` post processor does
 * (src/tracer/src/core/post_processor/save_to_img.cpp:10-69): flipped
 * vertically; "png": uint8(clamp(c^gamma, 0, 1) * 255); "hdr": Radiance RGBE;
 * "pfm": float.  `ext` may be NULL to use the filename's extension. */
int atrc_save_image(const char* filename, const char* ext, const float* rgb,
                    int width, int height, float gamma);

/* Average the accumulators into an image: rgb[3*i] = value / weight (0 where
 * weight == 0); host pointers. */
int atrc_film_resolve(const AtrcFilm* film, int width, int height, float* rgb);

/* Write 8-bit RGB (rows top to bottom, as atrc_cuda_encode_ldr produces)
 * as a PNG file. */
int atrc_save_png_bytes(const char* filename, const uint8_t* rgb8, int width, int height);

/* ---- the output path on the device (the post_processor directory) ------ */
typedef enum AtrcPostType {
    ATRC_POST_GAMMA = 0,            /* c^value (gamma.cpp:19-31)              */
    ATRC_POST_ACES = 1,             /* ACES curve of c * value (aces.cpp)     */
    ATRC_POST_NORMAL_TO_COLOR = 2   /* (c + 1) / 2 (save_gbuffer.cpp:21-33)   */
} AtrcPostType;

/* value / weight (and albedo / weight, normal / weight when both pointers
 * are given) of a device film into device images (3 floats per pixel, row 0
 * = bottom of the picture, perpixel_renderer.cpp:180-191). */
int atrc_cuda_film_resolve(const AtrcFilm* film, int width, int height,
                           float* rgb, float* albedo, float* normal);
/* One post-processing step on a device image, in place. */
int atrc_cuda_post_apply(float* rgb, int width, int height, int32_t type, float value);
/* The 8-bit encoding of save_to_img / save_gbuffer_to_png on the device:
 * flipped vertically, uint8(clamp(c^gamma, 0, 1) * 255). */
int atrc_cuda_encode_ldr(const float* rgb, int width, int height, float gamma, uint8_t* out);
/* Run a rendering's post-processor list (the JSON array returned by
 * atrc_config_post_processors) on a film (host or device): `gamma`, `aces`,
 * `save_to_img` (png, hdr, pfm) and `save_gbuffer_to_png` on the device and
 * in the listed order; `resize` and `oidn_denoiser` (third-party libraries)
 * are skipped.  ${scene-directory} maps to scene_dir.  `log` (may be NULL)
 * receives one line per file saved or step skipped. */
int atrc_cuda_post_process(const AtrcFilm* film, int width, int height, const char* post_json,
                           const char* scene_dir, char* log, size_t log_cap);

/* ------------------------------------------------------------------------
 * Learned path guiding (no counterpart in the reference, whose `pt` samples
 * the BSDF only, path_tracing.cpp:150-169).  A guide is a small network --
 * a 16-level hash grid over the scene bound (2 features per level), one-blob
 * encodings of the shading normal and outgoing direction, and roughness
 * (112 inputs), three hidden layers of 64 (ReLU, BF16 weights, FP32
 * accumulation on the tensor cores) and 48 outputs -- that gives each
 * surface vertex a mixture of 8 von Mises-Fisher lobes and a probability of
 * sampling it instead of the BSDF (one-sample MIS, so the render stays
 * unbiased; pair it with disney_fixed = 1 so that BSDF samples follow the
 * pdf they report).  It is trained online with Adam on records of the
 * vertices a recording render sampled and the radiance their paths brought
 * back (loss -w log(c q + (1 - c) p_bsdf), w = f cos L_i / pdf).
 * ------------------------------------------------------------------------ */
typedef struct AtrcGuide AtrcGuide;

typedef struct AtrcGuideDesc {
    int32_t  log2_table;       /* hash entries per level = 2^log2_table (19) */
    int32_t  base_resolution;  /* cells per axis of the coarsest level (4)   */
    int32_t  max_resolution;   /* ... of the finest level (64)               */
    int32_t  batch;            /* records per training step (2^18)           */
    int32_t  record_capacity;  /* records kept by a recording render (2^20)  */
    float    learning_rate;    /* Adam step size (1e-2)                      */
    int32_t  max_depth;        /* guide vertices up to this path depth (5;   */
                               /* 0: every depth)                            */
    float    max_select;       /* cap on the probability of sampling the     */
                               /* guide instead of the BSDF (0.15; at most   */
                               /* 0.99): the BSDF keeps 1 - max_select of    */
                               /* every sample, which bounds the variance an */
                               /* overconfident guide can add                */
    uint64_t seed;             /* parameter initialisation                   */
    float    target_clamp;     /* > 0: training targets capped at this       */
                               /* multiple of their batch mean (0: off)      */
    int32_t  pad_;
} AtrcGuideDesc;

typedef struct AtrcGuideInfo {
    uint64_t weights;          /* MLP weights (packed [out][in] per layer)   */
    uint64_t table_floats;     /* hash-table floats (levels x 2^log2 x 2)    */
    int32_t  levels, inputs, hidden, outputs, lobes, steps, log2_table, pad_;
    float    grid_lo[3], grid_inv_extent[3];  /* position -> [0,1]^3          */
    int32_t  grid_res[16];     /* cells per axis of each hash level          */
    float    max_select;       /* c = max_select * sigmoid(o[40] - 2)        */
    float    pad2_;
} AtrcGuideInfo;

int  atrc_guide_default_desc(AtrcGuideDesc* desc);
/* A guide for positions in [lo, hi] (e.g. atrc_cuda_scene_bounds). */
int  atrc_guide_create(int device, const float lo[3], const float hi[3],
                       const AtrcGuideDesc* desc, AtrcGuide** out);
void atrc_guide_destroy(AtrcGuide* guide);
int  atrc_guide_info(AtrcGuide* guide, AtrcGuideInfo* info);
/* Change the cap on the selection probability (0 < max_select <= 0.99) for
 * the renders and training steps that follow, e.g. a low cap while the guide
 * learns and a higher one once it has: every render uses one cap for both
 * its sampling and its pdfs, so the estimator stays unbiased. */
int  atrc_guide_set_max_select(AtrcGuide* guide, float max_select);
/* Read (set = 0) or replace (set = 1) the FP32 master parameters; either
 * pointer may be NULL.  Sizes as in AtrcGuideInfo. */
int  atrc_guide_params(AtrcGuide* guide, float* weights, float* table, int set);
/* Raw network outputs (n x 48) for host queries (n x 10: position, shading
 * normal, outgoing direction, roughness), on the tensor cores. */
int  atrc_guide_eval(AtrcGuide* guide, const float* queries, size_t n, float* raw);
/* Mixture pdf of directions dirs (n x 3) at queries (n x 10) and the
 * selection probability c, as the renderer computes them on the GPU. */
int  atrc_guide_pdf(AtrcGuide* guide, const float* queries, const float* dirs,
                    size_t n, float* pdf, float* select);
/* `steps` Adam steps over the records of the last recording render whose
 * target is positive (zero-target records add nothing to the loss or its
 * gradient and are dropped first), in batches of desc.batch; last_loss may be
 * NULL.  It also sets the recording probability of the next recording render
 * to about 0.95 record_capacity / (guided vertices of the last one), so that
 * a pass's records sample all of its guided vertices, not its first ones. */
int  atrc_guide_train(AtrcGuide* guide, int steps, float* last_loss);
/* The same on host records (n x 24 floats: position, normal, outgoing
 * direction, roughness, sampled direction, its BSDF pdf, throughput (3),
 * weight, and 6 unused). */
int  atrc_guide_train_records(AtrcGuide* guide, const float* records, size_t n,
                              int steps, float* last_loss);
/* Copy out the records of the last recording render (24 floats each). */
int  atrc_guide_records(AtrcGuide* guide, float* records, size_t cap, size_t* count);

/* Gradients of the training loss over `n` host records (n x 24 floats, as
 * atrc_guide_records returns them; 128 <= n <= record_capacity) at the
 * current parameters, computed by the tensor-core training kernel without
 * the Adam step: `grad_weights` (AtrcGuideInfo.weights floats), `grad_table`
 * (table_floats) and the loss sum.  Parameters and optimiser state are left
 * unchanged.  For checking the backward pass against a reference. */
int  atrc_guide_gradients(AtrcGuide* guide, const float* records, size_t n,
                          float* grad_weights, float* grad_table, float* loss);

/* Batched multi-view render (no counterpart in the reference, which renders
 * one camera per `rendering` entry): n views (camera, size, spp, seed,
 * filter may differ; depth, roulette, eps, sort, Disney, pool and
 * intersection settings must be equal) share one wavefront path pool, so
 * small views fill the GPU together and one view's tail overlaps the next
 * view's start.  The whole bounce loop is one graph launch: a device-side
 * WHILE conditional node runs windows of wavefront iterations until the
 * counters say every sample is splatted (bounded: a loop that ran longer than
 * any path allows ends with ATRC_ERR_WATCHDOG); the host waits once.  Films
 * must hold device pointers.  `guide` may be NULL (plain) or a trained guide
 * (sampling only).  view_seconds (may be NULL) receives per view the time,
 * on the device's global timer, from the start of the render to the splat of
 * the view's last sample.  `stats` has counts but no per-kernel timings.
 * At most 1024 views. */
int  atrc_cuda_render_batch(AtrcScene* scene, AtrcGuide* guide,
                            const AtrcRenderDesc* views, int32_t n,
                            const AtrcFilm* films, double* view_seconds,
                            AtrcRenderStats* stats);
/* Subsurface probe check: n samples of the subsurface walk (normalized
 * diffusion, separable.cpp:107-248) from the closest hit of the ray (o, d),
 * which must meet a Disney material with subsurface scattering: the weight
 * coef / pdf (zero for an invalid sample) -> w[3 n] and the exit point ->
 * exit_pos[3 n].  Uses the scene's eps of the last render (3e-4 before). */
int  atrc_cuda_subsurface_probe(AtrcScene* scene, const float o[3], const float d[3], int32_t n,
                                uint64_t seed, float* w, float* exit_pos);
/* Scene bound (for atrc_guide_create). */
int  atrc_cuda_scene_bounds(AtrcScene* scene, float lo[3], float hi[3]);
/* atrc_cuda_render with the guide sampling surface vertices; record = 1
 * also keeps training records (replacing the previous ones). */
int  atrc_cuda_render_guided(AtrcScene* scene, AtrcGuide* guide,
                             const AtrcRenderDesc* desc, int32_t record,
                             AtrcFilm* film, AtrcRenderStats* stats);

/* ------------------------------------------------ scene ingestion (BVH) */
/* The mesh trees of a device scene come from the builder its description
 * names (AtrcSceneDesc.bvh_builder).  These two entries run a builder alone
 * on a list of boxes, for comparing builders and checking the device build.
 * No reference counterpart: the reference builds triangle_bvh.cpp:122-304
 * on the CPU. */
typedef struct AtrcBvhBuildInfo {
    double   seconds;     /* tree, leaves, 4-wide collapse and validation    */
    double   sah_cost;    /* surface-area cost of the 4-wide tree (unit     */
                          /* traversal and intersection costs)              */
    uint64_t nodes;       /* 4-wide nodes                                    */
    int32_t  rounds;      /* PLOC rounds on the device (0 otherwise)         */
    int32_t  max_depth;   /* depth of the 4-wide tree                        */
} AtrcBvhBuildInfo;

/* boxes: n x 6 floats (lo x y z, hi x y z).  builder ATRC_BVH_SAH runs on
 * the host; ATRC_BVH_PLOC runs on `device`, or, with device < 0, as its
 * serial host specification (the same tree, slowly). */
int  atrc_bvh_build(int32_t builder, int32_t device, const float* boxes, uint64_t n,
                    AtrcBvhBuildInfo* info);
/* The PLOC cluster tree on the host (device < 0) or on `device`: order[n]
 * (sorted position -> box index), left[n-1], right[n-1] and
 * node_boxes[(n-1) x 6] of internal node n + k (nodes below n are the
 * leaves in sorted order), the root and the number of rounds.  The host and
 * the device give the same tree. */
int  atrc_bvh_cluster_tree(int32_t device, const float* boxes, uint64_t n, uint32_t* order,
                           int32_t* left, int32_t* right, float* node_boxes, int32_t* root,
                           int32_t* rounds);

#ifdef __cplusplus
}
#endif

#endif /* ATRC_CUDA_H */
