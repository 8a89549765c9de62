// pt_cuda for Atrc's factory: the renderer a maintainer of Atrc adds to its
// factory library so that a rendering entry with "type": "pt_cuda" renders
// on the GPU through libatrc_cuda.so, next to the CPU "pt" renderer.
//
// The file is written against the reference's own interfaces, which must be
// declared before it is included (in Atrc: the headers below; in this
// repository's tests: stand-ins with the same members):
//   agz::tracer::Renderer            src/tracer/include/agz/tracer/core/renderer.h:17-64
//   RenderTarget, FilmFilterApplier  src/tracer/include/agz/tracer/core/render_target.h:64-74, 212-221
//   Scene::get_camera                src/tracer/include/agz/tracer/core/scene.h:52
//   RendererInteractor               src/tracer/include/agz/tracer/core/renderer_interactor.h:17-65
//   EPS()                            src/tracer/include/agz/tracer/common.h:44
//   factory::Creator, CreatingContext src/factory/include/agz/factory/context.h:27-128
//   factory::config_to_json, json_to_string  src/factory/include/agz/factory/utility/config_cvt.h
//
// How it reaches the scene.  Atrc's Scene, Camera and FilmFilter are opaque
// interfaces (no enumeration of entities or camera parameters), so the
// renderer re-reads the JSON it was configured from, through the C ABI's
// loader, which mirrors Atrc's creators and defaults:
//   - the scene group is the creating context's `reference_root`, which the
//     CLI points at the "scene" group (src/cli/src/main.cpp:46-50);
//   - the renderer group is the one the factory hands to the creator, so each
//     entry of a "rendering" array keeps its own settings;
//   - cameras and film filters are recorded by decorators registered under
//     the reference's creator names: each wraps the original creator, taken
//     from a second, untouched CreatingContext, and remembers the config of
//     every object it creates.  A camera is looked up at render time by the
//     pointer Scene::get_camera() returns.  A film filter is created just
//     before the camera and the renderer of the same entry
//     (render_session.cpp:14-40), so the pt_cuda creator takes the filter
//     recorded since the previous renderer was created; without one the
//     entry uses the default box filter of radius 0.5, as the reference;
//   - the film size comes from FilmFilterApplier, eps from EPS().
//
// Cancellation.  Renderer::render_async / stop_async
// (src/tracer/src/core/core/renderer.cpp:5-38) signal through the
// std::atomic<bool> stop_rendering_ member; the renderer hands
// atrc_cuda_render a poll callback that loads it.  doing_rendering_ (the
// next member) is not read.
#pragma once

#include <cstdio>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "atrc_cuda.h"

namespace atrc_plugin {

using agz::tracer::Camera;
using agz::tracer::Config;
using agz::tracer::ConfigGroup;
using agz::tracer::FilmFilter;
using agz::tracer::FilmFilterApplier;
using agz::tracer::RC;
using agz::tracer::Renderer;
using agz::tracer::RendererInteractor;
using agz::tracer::RenderTarget;
using agz::tracer::Scene;
using agz::tracer::Spectrum;
using agz::tracer::Vec3;
using agz::tracer::real;
namespace factory = agz::tracer::factory;

inline std::string group_json(const ConfigGroup& g) {
    return factory::json_to_string(factory::config_to_json(g));
}

// Configs of the cameras and film filters created through the decorators.
class Records {
public:
    void camera(const Camera* cam, std::string json) {
        std::lock_guard<std::mutex> lk(m_);
        cameras_[cam] = std::move(json);
    }
    std::string camera_json(const Camera* cam) const {
        std::lock_guard<std::mutex> lk(m_);
        const auto it = cameras_.find(cam);
        return it == cameras_.end() ? std::string() : it->second;
    }
    void film_filter(std::string json) {
        std::lock_guard<std::mutex> lk(m_);
        pending_filter_ = std::move(json);
    }
    // the filter recorded since the last call (empty: the default box filter)
    std::string take_film_filter() {
        std::lock_guard<std::mutex> lk(m_);
        std::string f = std::move(pending_filter_);
        pending_filter_.clear();
        return f;
    }

private:
    mutable std::mutex m_;
    std::map<const Camera*, std::string> cameras_;
    std::string pending_filter_;
};

class RecordingCameraCreator : public factory::Creator<Camera> {
public:
    RecordingCameraCreator(const factory::Creator<Camera>* original, std::shared_ptr<Records> records)
        : original_(original), records_(std::move(records)) {}
    std::string name() const override { return original_->name(); }
    RC<Camera> create(const ConfigGroup& params, factory::CreatingContext& context, real film_aspect) const override {
        RC<Camera> cam = original_->create(params, context, film_aspect);
        records_->camera(cam.get(), group_json(params));
        return cam;
    }

private:
    const factory::Creator<Camera>* original_;
    std::shared_ptr<Records> records_;
};

class RecordingFilmFilterCreator : public factory::Creator<FilmFilter> {
public:
    RecordingFilmFilterCreator(const factory::Creator<FilmFilter>* original, std::shared_ptr<Records> records)
        : original_(original), records_(std::move(records)) {}
    std::string name() const override { return original_->name(); }
    RC<FilmFilter> create(const ConfigGroup& params, factory::CreatingContext& context) const override {
        RC<FilmFilter> f = original_->create(params, context);
        records_->film_filter(group_json(params));
        return f;
    }

private:
    const factory::Creator<FilmFilter>* original_;
    std::shared_ptr<Records> records_;
};

class PtCudaRenderer : public Renderer {
public:
    PtCudaRenderer(std::string scene_json, std::string renderer_json, std::string film_filter_json,
                   std::string scene_dir, std::shared_ptr<Records> records, int device = 0)
        : scene_json_(std::move(scene_json)), renderer_json_(std::move(renderer_json)),
          film_filter_json_(std::move(film_filter_json)), scene_dir_(std::move(scene_dir)),
          records_(std::move(records)), device_(device) {}

    ~PtCudaRenderer() override {
        stop_async();
        if (scene_) atrc_cuda_scene_destroy(scene_);
    }

    // The "rendering" entry this renderer belongs to, as the JSON the C ABI's
    // loader reads: {"scene": ..., "rendering": {width, height, eps, camera,
    // film_filter, renderer}}.
    std::string compose(const FilmFilterApplier& filter, const Scene& scene) const {
        const std::string cam = records_->camera_json(scene.get_camera());
        if (cam.empty()) throw std::runtime_error("pt_cuda: the scene's camera was not created through the factory");
        char num[64];
        std::string r = "{\"scene\": " + scene_json_ + ", \"rendering\": {";
        std::snprintf(num, sizeof(num), "\"width\": %d, \"height\": %d, ", filter.width(), filter.height());
        r += num;
        std::snprintf(num, sizeof(num), "\"eps\": \"%f\", ", double(agz::tracer::EPS()));
        r += num;
        r += "\"camera\": " + cam + ", ";
        if (!film_filter_json_.empty()) r += "\"film_filter\": " + film_filter_json_ + ", ";
        r += "\"renderer\": " + renderer_json_ + "}}";
        return r;
    }

    // Load the composed entry; the device scene is built once per renderer.
    AtrcRenderDesc prepare(const FilmFilterApplier& filter, const Scene& scene) {
        AtrcConfig* cfg = nullptr;
        check(atrc_config_load_string(compose(filter, scene).c_str(), scene_dir_.c_str(), &cfg));
        std::unique_ptr<AtrcConfig, void (*)(AtrcConfig*)> hold(cfg, atrc_config_destroy);
        AtrcRenderDesc desc{};
        char type[32] = {};
        check(atrc_config_rendering(cfg, 0, &desc, type, sizeof(type)));
        // use_mis = 0 selects trace_nomis in the reference's pt (pt.cpp:21-24),
        // which pt_cuda does not implement: refuse before building anything
        if (desc.renderer == ATRC_RENDERER_PT && !desc.use_mis)
            throw factory::CreatingObjectException(
                "pt_cuda: use_mis = 0 selects the reference's trace_nomis, which pt_cuda does not implement; "
                "render this entry with pt");
        if (!scene_) {
            const AtrcSceneDesc* sd = nullptr;
            check(atrc_config_scene(cfg, &sd));
            check(atrc_cuda_device_init(device_, nullptr));
            check(atrc_cuda_scene_create(sd, &scene_));  // BVH build and upload
        }
        return desc;
    }

    // Renderer::render (src/tracer/include/agz/tracer/core/renderer.h:33-35)
    RenderTarget render(FilmFilterApplier filter, Scene& scene, RendererInteractor& reporter) override {
        const AtrcRenderDesc desc = prepare(filter, scene);
        const int w = filter.width(), h = filter.height();
        const size_t n = size_t(w) * h;
        std::vector<double> value(3 * n), weight(n), albedo(3 * n), normal(3 * n), denoise(n);
        AtrcFilm film{value.data(), weight.data(), nullptr, albedo.data(), normal.data(), denoise.data(), 0, 0};
        struct Poll {
            PtCudaRenderer* self;
            RendererInteractor* reporter;
        } poll{this, &reporter};
        auto should_stop = [](void* u) -> int { return static_cast<Poll*>(u)->self->stop_rendering_.load() ? 1 : 0; };
        auto progress = [](double pct, void* u) { static_cast<Poll*>(u)->reporter->progress(pct, {}); };
        reporter.begin();
        reporter.new_stage();
        last_status_ = atrc_cuda_render(scene_, &desc, &film, should_stop, progress, &poll, nullptr);
        reporter.end_stage();
        reporter.end();
        if (last_status_ != ATRC_OK && last_status_ != ATRC_ERR_CANCELLED) check(last_status_);
        // value / weight (perpixel_renderer.cpp:180-191); a stopped render
        // returns the samples taken so far, as the reference's renderers do
        RenderTarget rt;
        rt.image.initialize(h, w);
        rt.albedo.initialize(h, w);
        rt.normal.initialize(h, w);
        rt.denoise.initialize(h, w);
        for (int y = 0; y < h; ++y)
            for (int x = 0; x < w; ++x) {
                const size_t i = size_t(y) * w + x;
                const double k = weight[i] > 0 ? 1 / weight[i] : 1;
                rt.image(y, x) = Spectrum(real(value[3 * i] * k), real(value[3 * i + 1] * k), real(value[3 * i + 2] * k));
                rt.albedo(y, x) =
                    Spectrum(real(albedo[3 * i] * k), real(albedo[3 * i + 1] * k), real(albedo[3 * i + 2] * k));
                rt.normal(y, x) = Vec3(real(normal[3 * i] * k), real(normal[3 * i + 1] * k), real(normal[3 * i + 2] * k));
                rt.denoise(y, x) = real(denoise[i] * k);
            }
        weight_sum_ = 0;
        for (double v : weight) weight_sum_ += v;
        return rt;
    }

    int last_status() const { return last_status_; }  // of the last render: ATRC_OK or ATRC_ERR_CANCELLED
    double last_weight_sum() const { return weight_sum_; }

private:
    static void check(int rc) {
        if (rc != ATRC_OK) throw factory::CreatingObjectException(std::string("pt_cuda: ") + atrc_last_error());
    }

    std::string scene_json_, renderer_json_, film_filter_json_, scene_dir_;
    std::shared_ptr<Records> records_;
    int device_;
    AtrcScene* scene_ = nullptr;
    int last_status_ = ATRC_OK;
    double weight_sum_ = 0;
};

class PtCudaCreator : public factory::Creator<Renderer> {
public:
    explicit PtCudaCreator(std::shared_ptr<Records> records) : records_(std::move(records)) {}
    std::string name() const override { return "pt_cuda"; }
    RC<Renderer> create(const ConfigGroup& params, factory::CreatingContext& context) const override {
        if (!context.reference_root)
            throw factory::CreatingObjectException("pt_cuda: the creating context has no reference_root");
        const std::string scene_dir = context.path_mapper ? context.path_mapper->map("${scene-directory}") : "";
        return std::make_shared<PtCudaRenderer>(group_json(*context.reference_root), group_json(params),
                                                records_->take_film_filter(), scene_dir, records_);
    }

private:
    std::shared_ptr<Records> records_;
};

// Register pt_cuda and the recording decorators in `context`, after it is
// constructed (src/factory/src/factory.cpp:18-53) and before the scene and
// the rendering entries are created.  `pristine` is a second, untouched
// CreatingContext that holds the original camera and film-filter creators;
// it must outlive `context`.
inline std::shared_ptr<Records> register_pt_cuda(factory::CreatingContext& context,
                                                 const factory::CreatingContext& pristine) {
    auto records = std::make_shared<Records>();
    for (const char* name : {"pinhole", "thin_lens"})
        if (const auto* c = pristine.factory<Camera>().get_creator(name))
            context.factory<Camera>().add_creator(std::make_unique<RecordingCameraCreator>(c, records));
    for (const char* name : {"box", "gaussian"})
        if (const auto* c = pristine.factory<FilmFilter>().get_creator(name))
            context.factory<FilmFilter>().add_creator(std::make_unique<RecordingFilmFilterCreator>(c, records));
    context.factory<Renderer>().add_creator(std::make_unique<PtCudaCreator>(records));
    return records;
}

}  // namespace atrc_plugin
