// C entry points over the reference's own renderer (test infrastructure):
// Atrc's factory parses the scene JSON and builds the scene exactly as its
// CLI does (src/cli/src/main.cpp:46-70); renders run the reference's
// render::trace_std (src/tracer/src/render/path_tracing.cpp:15-225) per
// sample, through the reference's camera and film-filter grids
// (FilmFilterApplier, render_target.h), in the reference's tile layout
// (parallel_for_2d_grid, perpixel_renderer.cpp:56-191).
//
// One thing differs from PerPixelRenderer, on purpose: its samplers are
// seeded with the fixed 42 + thread index (perpixel_renderer.cpp:77), so
// repeated renders are not independent.  Here each tile's NativeSampler is
// seeded from (seed, tile, first sample index), so renders with different
// seeds are independent estimates, and every pixel also accumulates
// sum w * L^2 for the per-pixel variance the parity tests need.
#include <agz/factory/factory.h>
#include <agz/factory/utility/config_cvt.h>
#include <agz/tracer/create/film_filter.h>
#include <agz/tracer/core/camera.h>
#include <agz/tracer/core/entity.h>
#include <agz/tracer/core/film_filter.h>
#include <agz/tracer/core/render_target.h>
#include <agz/tracer/core/sampler.h>
#include <agz/tracer/core/scene.h>
#include <agz/tracer/render/path_tracing.h>
#include <agz/tracer/utility/parallel_grid.h>
#include <spdlog/spdlog.h>
#include <spdlog/sinks/stdout_color_sinks.h>

#include <filesystem>
#include <fstream>
#include <mutex>
#include <sstream>

#include "atrc_cuda.h"

using namespace agz;
using namespace agz::tracer;

namespace {

thread_local std::string g_error;

int fail(const std::string& msg) {
    g_error = msg;
    return -1;
}

std::string describe(const std::exception& e) {
    std::string s = e.what();
    try {
        std::rethrow_if_nested(e);
    } catch (const std::exception& inner) {
        s += ": " + describe(inner);
    } catch (...) {
    }
    return s;
}

// Records the entities the factory creates, in creation order (the scene
// creator creates them in the order of the "entities" array,
// scene_creators.cpp:31-47), so hits can be reported by entity index.
class RecordingEntityCreator : public factory::Creator<Entity> {
public:
    RecordingEntityCreator(const factory::Creator<Entity>* original, std::vector<const Entity*>* out)
        : original_(original), out_(out) {}
    std::string name() const override { return original_->name(); }
    RC<Entity> create(const ConfigGroup& params, factory::CreatingContext& context) const override {
        RC<Entity> e = original_->create(params, context);
        if (std::find(out_->begin(), out_->end(), e.get()) == out_->end()) out_->push_back(e.get());
        return e;
    }

private:
    const factory::Creator<Entity>* original_;
    std::vector<const Entity*>* out_;
};

// FP64 texel for the film accumulators: the reference accumulates in FP32
// (Image2D<Spectrum>), whose rounding over hundreds of samples of a constant
// pixel (an emitter seen directly) is larger than the 1e-6 relative slack
// of the parity band; the per-sample values are still the reference's.
struct DSpec {
    double r = 0, g = 0, b = 0;
    DSpec() = default;
    DSpec(double r_, double g_, double b_) : r(r_), g(g_), b(b_) {}
    DSpec& operator+=(const DSpec& o) { r += o.r; g += o.g; b += o.b; return *this; }
    friend DSpec operator*(real w, const DSpec& s) { return {w * s.r, w * s.g, w * s.b}; }
};

}  // namespace

struct RefScene {
    factory::BasicPathMapper mapper;
    Config root;
    factory::CreatingContext pristine;
    factory::CreatingContext context;
    RC<Scene> scene;
    std::vector<const Entity*> entities;
    std::vector<const ConfigGroup*> renderings;
};

extern "C" {

const char* ref_last_error(void) { return g_error.c_str(); }

// Parse `json` (a whole {"scene", "rendering"} configuration) with the
// reference's factory; relative paths resolve against scene_dir.
int ref_scene_create(const char* json, const char* scene_dir, RefScene** out) {
    if (!json || !scene_dir || !out) return fail("null argument");
    *out = nullptr;
    try {
        // the reference logs through spdlog's default logger (AGZ_INFO,
        // logger.h:14), which writes to stdout: send it to stderr, so that a
        // caller's stdout holds only what the caller prints
        static std::once_flag log_once;
        std::call_once(log_once, [] { spdlog::set_default_logger(spdlog::stderr_color_mt("atrc_ref")); });
        auto rs = std::make_unique<RefScene>();
        rs->mapper.add_replacer(AGZ_FACTORY_SCENE_DESC_PATH_NAME, scene_dir);
        rs->mapper.add_replacer(AGZ_FACTORY_WORKING_DIR_PATH_NAME, std::filesystem::current_path().string());
        rs->root = factory::json_to_config(factory::string_to_json(json));
        const ConfigGroup& scene_config = rs->root.child_group("scene");
        rs->context.path_mapper = &rs->mapper;
        rs->context.reference_root = &scene_config;
        rs->context.factory<Entity>().add_creator(
            newBox<RecordingEntityCreator>(rs->pristine.factory<Entity>().get_creator("geometric"), &rs->entities));
        rs->scene = rs->context.create<Scene>(scene_config);
        const ConfigNode& rendering = rs->root.child("rendering");
        if (rendering.is_array()) {
            const auto& arr = rendering.as_array();
            for (size_t i = 0; i < arr.size(); ++i) rs->renderings.push_back(&arr.at_group(i));
        } else {
            rs->renderings.push_back(&rendering.as_group());
        }
        *out = rs.release();
        return 0;
    } catch (const std::exception& e) {
        return fail(describe(e));
    }
}

void ref_scene_destroy(RefScene* s) { delete s; }

int ref_entity_count(RefScene* s) { return s ? int(s->entities.size()) : -1; }

// Closest (mode 0) or any (mode 1) hit of each ray: Scene::closest_intersection
// / has_intersection (scene_default.cpp:136-147).  Closest hits report t,
// the entity index and u = the hit's uv.x; prim is -1 (the reference's
// intersection records carry no primitive index).
int ref_trace_rays(RefScene* s, const AtrcRay* rays, size_t n, AtrcHit* hits, int mode, int threads) {
    if (!s || (n && (!rays || !hits))) return fail("null argument");
    try {
        std::atomic<size_t> next{0};
        const int nt = thread::actual_worker_count(threads);
        auto work = [&] {
            for (;;) {
                const size_t c0 = next.fetch_add(4096);
                if (c0 >= n) break;
                for (size_t i = c0; i < std::min(n, c0 + 4096); ++i) {
                    const AtrcRay& q = rays[i];
                    const Ray r(FVec3(q.o[0], q.o[1], q.o[2]), FVec3(q.d[0], q.d[1], q.d[2]), q.t_min, q.t_max);
                    AtrcHit& h = hits[i];
                    h.prim = -1;
                    h.u = 0;
                    if (mode == 1) {
                        const bool occ = s->scene->has_intersection(r);
                        h.t = occ ? 1.0f : -1.0f;
                        h.entity = occ ? 0 : -1;
                        continue;
                    }
                    EntityIntersection inct;
                    if (s->scene->closest_intersection(r, &inct)) {
                        h.t = inct.t;
                        const auto it = std::find(s->entities.begin(), s->entities.end(), inct.entity);
                        h.entity = it == s->entities.end() ? -2 : int(it - s->entities.begin());
                        h.u = inct.uv.x;
                    } else {
                        h.t = -1;
                        h.entity = -1;
                    }
                }
            }
        };
        std::vector<std::thread> ts;
        for (int k = 1; k < nt; ++k) ts.emplace_back(work);
        work();
        for (auto& t : ts) t.join();
        return 0;
    } catch (const std::exception& e) {
        return fail(describe(e));
    }
}

// Render samples [first_spp, first_spp + spp_count) of every pixel of
// rendering entry `index` with the reference's pt (its renderer keys and
// defaults, renderer_creators.cpp:115-151) or ao (renderer_creators.cpp:8-44,
// render::trace_ao) and ADD into the caller's FP64 films (width x height
// pixels, rows as the reference's film): value (3 per pixel, sum w L),
// weight (sum w), value_sq (3 per pixel, sum w L^2), and the G-buffer the
// reference's PerPixelRenderer keeps (perpixel_renderer.cpp:38-44): albedo
// and normal (3 per pixel) and denoise (1 per pixel), each sum w x; the last
// four may be null.  `width` / `height` override the entry's film size when
// positive.  tile_stride > 1 renders only every tile_stride-th task tile
// (row-major tile index), a bounded sample of the image for timing.
int ref_render(RefScene* s, int index, int width, int height, int first_spp, int spp_count, uint64_t seed,
               int threads, int tile_stride, double* value, double* weight, double* value_sq, double* albedo,
               double* normal, double* denoise) {
    if (!s || !value || !weight || spp_count < 1 || first_spp < 0 || tile_stride < 1)
        return fail("invalid argument");
    if (index < 0 || size_t(index) >= s->renderings.size()) return fail("rendering index out of range");
    try {
        const ConfigGroup& r = *s->renderings[size_t(index)];
        const int W = width > 0 ? width : r.child_int("width");
        const int H = height > 0 ? height : r.child_int("height");
        // RenderSession: eps, film filter, camera (render_session.cpp:14-66)
        real eps = real(3e-4);
        if (auto node = r.find_child_value("eps")) eps = node->as_real();
        set_eps(eps);
        RC<FilmFilter> film_filter;
        if (auto group = r.find_child_group("film_filter")) film_filter = s->context.create<FilmFilter>(*group);
        else film_filter = create_box_filter(real(0.5));
        RC<Camera> camera = s->context.create<Camera>(r.child_group("camera"), real(W) / real(H));
        // the pt creator's keys (renderer_creators.cpp:127-146)
        const ConfigGroup& rp = r.child_group("renderer");
        const std::string type = rp.child_str("type");
        const bool is_ao = type == "ao";
        if (type != "pt" && type != "pt_cuda" && !is_ao) return fail("renderer must be pt, pt_cuda or ao, not " + type);
        // the ao creator's keys (renderer_creators.cpp:21-40)
        render::AOParams ao;
        if (is_ao) {
            ao.ao_sample_count = rp.child_int_or("ao_sample_count", 5);
            ao.low_color = rp.child_spectrum_or("low_color", Spectrum(0));
            ao.high_color = rp.child_spectrum_or("high_color", Spectrum(1));
            ao.max_occlusion_distance = rp.child_real_or("max_occlusion_distance", 1);
            ao.background_color = rp.child_spectrum_or("background_color", Spectrum(0));
        }
        render::TraceParams params;
        params.min_depth = rp.child_int_or("min_depth", 5);
        params.max_depth = rp.child_int_or("max_depth", 10);
        params.cont_prob = rp.child_real_or("cont_prob", real(0.9));
        params.specular_depth = rp.child_int_or("specular_depth", 20);
        const bool use_mis = rp.child_int_or("use_mis", 1) != 0;
        const int grid_size = rp.child_int_or("task_grid_size", 32);

        s->scene->set_camera(camera);
        s->scene->start_rendering();
        FilmFilterApplier filter(W, H, film_filter);
        Image2D<DSpec> img_value(H, W), img_value_sq(H, W), img_albedo(H, W), img_normal(H, W);
        Image2D<double> img_weight(H, W), img_denoise(H, W);
        std::mutex merge_mutex;
        const int tiles_x = (W + grid_size - 1) / grid_size;
        const int nt = thread::actual_worker_count(threads);
        thread::thread_group_t group(nt);
        parallel_for_2d_grid(nt, W, H, grid_size, grid_size, group, [&](int, const Rect2i& rect) {
            const int tile = (rect.low.y / grid_size) * tiles_x + rect.low.x / grid_size;
            if (tile % tile_stride != 0) return true;
            const uint64_t h = misc::hash(seed, uint64_t(tile), uint64_t(first_spp));
            NativeSampler sampler(int(h & 0x7fffffff), false);
            Arena arena;
            auto grid = filter.create_subgrid<DSpec, double, DSpec, DSpec, DSpec, double>(
                {rect.low, rect.high - Vec2i(1)});
            const auto bound = grid.sample_pixels();
            for (int py = bound.low.y; py <= bound.high.y; ++py)
                for (int px = bound.low.x; px <= bound.high.x; ++px)
                    for (int i = 0; i < spp_count; ++i) {
                        // PerPixelRenderer::render_grid (perpixel_renderer.cpp:13-53)
                        const Sample2 film_sam = sampler.sample2();
                        const real pixel_x = px + film_sam.u, pixel_y = py + film_sam.v;
                        auto cam_ray = camera->sample_we({pixel_x / W, pixel_y / H}, sampler.sample2());
                        const Ray ray(cam_ray.pos_on_cam, cam_ray.pos_to_out);
                        const render::Pixel pixel =
                            is_ao     ? render::trace_ao(ao, *s->scene, ray, sampler)
                            : use_mis ? render::trace_std(params, *s->scene, ray, sampler, arena)
                                      : render::trace_nomis(params, *s->scene, ray, sampler, arena);
                        if (pixel.value.is_finite()) {
                            const Spectrum v = cam_ray.throughput * pixel.value;
                            const DSpec dv(v.r, v.g, v.b);
                            grid.apply(pixel_x, pixel_y, dv, 1.0, DSpec(dv.r * dv.r, dv.g * dv.g, dv.b * dv.b),
                                       DSpec(pixel.albedo.r, pixel.albedo.g, pixel.albedo.b),
                                       DSpec(pixel.normal.x, pixel.normal.y, pixel.normal.z), double(pixel.denoise));
                        }
                        arena.release();
                    }
            std::lock_guard<std::mutex> lk(merge_mutex);
            grid.merge_into(img_value, img_weight, img_value_sq, img_albedo, img_normal, img_denoise);
            return true;
        });
        for (int y = 0; y < H; ++y)
            for (int x = 0; x < W; ++x) {
                const size_t i = size_t(y) * W + x;
                const DSpec& v = img_value(y, x);
                value[3 * i] += v.r;
                value[3 * i + 1] += v.g;
                value[3 * i + 2] += v.b;
                weight[i] += img_weight(y, x);
                auto add3 = [&](double* dst, const DSpec& q) {
                    if (!dst) return;
                    dst[3 * i] += q.r;
                    dst[3 * i + 1] += q.g;
                    dst[3 * i + 2] += q.b;
                };
                add3(value_sq, img_value_sq(y, x));
                add3(albedo, img_albedo(y, x));
                add3(normal, img_normal(y, x));
                if (denoise) denoise[i] += img_denoise(y, x);
            }
        return 0;
    } catch (const std::exception& e) {
        return fail(describe(e));
    }
}

// The film filter of rendering entry `index` evaluated at the offsets
// (x[i], y[i]) from a pixel centre, as the reference splats with it
// (FilmFilterApplier::FilmGrid::apply, render_target.h:384-395).
int ref_filter_eval(RefScene* s, int index, const float* x, const float* y, size_t n, float* out) {
    if (!s || (n && (!x || !y || !out))) return fail("invalid argument");
    if (index < 0 || size_t(index) >= s->renderings.size()) return fail("rendering index out of range");
    try {
        const ConfigGroup& r = *s->renderings[size_t(index)];
        RC<FilmFilter> film_filter;
        if (auto group = r.find_child_group("film_filter")) film_filter = s->context.create<FilmFilter>(*group);
        else film_filter = create_box_filter(real(0.5));
        for (size_t i = 0; i < n; ++i) out[i] = float(film_filter->eval(real(x[i]), real(y[i])));
        return 0;
    } catch (const std::exception& e) {
        return fail(describe(e));
    }
}

}  // extern "C"
