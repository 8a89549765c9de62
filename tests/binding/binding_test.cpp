// Drives the pt_cuda plugin (atrc_b200/csrc/plugin/pt_cuda_renderer.hpp) the
// way the reference's CLI and RenderSession drive a renderer
// (src/cli/src/main.cpp:46-70, src/factory/src/utility/render_session.cpp:14-96),
// on the stand-ins of reference_stubs.h.
//
//   binding_test compose <plan>  for every rendering entry of the plan: create
//                                the film filter, camera and renderer through
//                                the creating context, compose the entry's
//                                JSON and print the loaded AtrcRenderDesc as
//                                one JSON line (no GPU needed)
//   binding_test async <plan>    entry 0 on the GPU: a render_async that runs
//                                to the end (doing_rendering_ stays raised),
//                                then one stopped by stop_async after the
//                                second progress report; one JSON line
//
// Plan lines (written by the test):
//   scene_dir <dir>
//   scene <file with the scene group's JSON>
//   entry <width> <height> <eps> <camera type> <camera file> <filter type|-> <filter file|-> <renderer file>
#include "reference_stubs.h"

#include "pt_cuda_renderer.hpp"

#include <chrono>
#include <cstdio>
#include <fstream>
#include <sstream>
#include <thread>

using namespace agz::tracer;

namespace {

struct StandInCamera : Camera {};

class StandInCameraCreator : public factory::Creator<Camera> {
public:
    explicit StandInCameraCreator(std::string n) : n_(std::move(n)) {}
    std::string name() const override { return n_; }
    RC<Camera> create(const ConfigGroup&, factory::CreatingContext&, real) const override {
        return std::make_shared<StandInCamera>();
    }

private:
    std::string n_;
};

class StandInFilterCreator : public factory::Creator<FilmFilter> {
public:
    explicit StandInFilterCreator(std::string n) : n_(std::move(n)) {}
    std::string name() const override { return n_; }
    RC<FilmFilter> create(const ConfigGroup&, factory::CreatingContext&) const override {
        return std::make_shared<FilmFilter>(real(0.5));
    }

private:
    std::string n_;
};

class SceneDirMapper : public factory::PathMapper {
public:
    explicit SceneDirMapper(std::string d) : d_(std::move(d)) {}
    std::string map(const std::string& p) const override {
        const std::string key = "${scene-directory}";
        std::string r = p;
        for (size_t i = r.find(key); i != std::string::npos; i = r.find(key)) r.replace(i, key.size(), d_);
        return r;
    }

private:
    std::string d_;
};

class CountingReporter : public RendererInteractor {
public:
    explicit CountingReporter(const Renderer* r) : r_(r) {}
    void progress(double, const PreviewFunc&) override {
        ++calls;
        if (r_->is_doing_rendering()) doing_seen = true;
    }
    void begin() override {}
    void end() override {}
    void new_stage() override {}
    void end_stage() override {}
    std::atomic<int> calls{0};
    std::atomic<bool> doing_seen{false};

private:
    const Renderer* r_;
};

std::string read_file(const std::string& path) {
    std::ifstream f(path);
    if (!f) throw std::runtime_error("cannot read " + path);
    std::stringstream ss;
    ss << f.rdbuf();
    return ss.str();
}

struct Entry {
    int width = 0, height = 0;
    real eps = real(3e-4);
    ConfigGroup camera, filter, renderer;
    bool has_filter = false;
};

}  // namespace

agz::tracer::factory::CreatingContext::CreatingContext() {
    for (const char* n : {"pinhole", "thin_lens"}) factory<Camera>().add_creator(std::make_unique<StandInCameraCreator>(n));
    for (const char* n : {"box", "gaussian"}) factory<FilmFilter>().add_creator(std::make_unique<StandInFilterCreator>(n));
}

int main(int argc, char** argv) {
    if (argc != 3) {
        std::fprintf(stderr, "usage: binding_test compose|async <plan>\n");
        return 2;
    }
    const std::string mode = argv[1];
    try {
        std::ifstream plan(argv[2]);
        std::string scene_dir;
        ConfigGroup scene_group{"default", ""};
        std::vector<Entry> entries;
        for (std::string line; std::getline(plan, line);) {
            std::istringstream ls(line);
            std::string kind;
            ls >> kind;
            if (kind == "scene_dir") {
                ls >> scene_dir;
            } else if (kind == "scene") {
                std::string f;
                ls >> f;
                scene_group.json = read_file(f);
            } else if (kind == "entry") {
                Entry e;
                std::string ct, cf, ft, ff, rf;
                ls >> e.width >> e.height >> e.eps >> ct >> cf >> ft >> ff >> rf;
                e.camera = {ct, read_file(cf)};
                if (ft != "-") {
                    e.filter = {ft, read_file(ff)};
                    e.has_filter = true;
                }
                e.renderer = {"pt_cuda", read_file(rf)};
                entries.push_back(e);
            }
        }
        // the CLI's context, with pt_cuda registered beside the reference's
        // creators (src/cli/src/main.cpp:46-50)
        SceneDirMapper mapper(scene_dir);
        factory::CreatingContext pristine;
        factory::CreatingContext context;
        context.path_mapper = &mapper;
        context.reference_root = &scene_group;
        atrc_plugin::register_pt_cuda(context, pristine);
        Scene scene;
        std::string out;
        for (size_t i = 0; i < entries.size(); ++i) {
            const Entry& e = entries[i];
            // parse_rendering_settings order: film filter, camera, renderer
            set_eps(e.eps);
            RC<const FilmFilter> filter = e.has_filter ? context.create<FilmFilter>(e.filter)
                                                       : std::make_shared<FilmFilter>(real(0.5));
            RC<Camera> camera = context.create<Camera>(e.camera, real(e.width) / real(e.height));
            RC<Renderer> renderer = context.create<Renderer>(e.renderer);
            scene.set_camera(camera);
            auto* pt = dynamic_cast<atrc_plugin::PtCudaRenderer*>(renderer.get());
            if (!pt) throw std::runtime_error("pt_cuda creator returned another renderer");
            FilmFilterApplier applier(e.width, e.height, filter);
            if (mode == "compose") {
                AtrcConfig* cfg = nullptr;
                if (atrc_config_load_string(pt->compose(applier, scene).c_str(), scene_dir.c_str(), &cfg) != ATRC_OK)
                    throw std::runtime_error(atrc_last_error());
                AtrcRenderDesc d{};
                char type[32] = {};
                const int rc = atrc_config_rendering(cfg, 0, &d, type, sizeof(type));
                atrc_config_destroy(cfg);
                if (rc != ATRC_OK) throw std::runtime_error(atrc_last_error());
                char buf[1024];
                std::snprintf(buf, sizeof(buf),
                              "{\"entry\": %zu, \"type\": \"%s\", \"width\": %d, \"height\": %d, \"spp\": %d, "
                              "\"min_depth\": %d, \"max_depth\": %d, \"cont_prob\": %.17g, \"specular_depth\": %d, "
                              "\"use_mis\": %d, \"filter_type\": %d, \"filter_radius\": %.17g, \"filter_alpha\": %.17g, "
                              "\"eps\": %.17g, \"task_grid_size\": %d, \"fov\": %.17g, \"lens_radius\": %.17g, "
                              "\"focal_distance\": %.17g, \"pos\": [%.17g, %.17g, %.17g]}\n",
                              i, type, d.width, d.height, d.spp, d.min_depth, d.max_depth, double(d.cont_prob),
                              d.specular_depth, d.use_mis, d.filter_type, double(d.filter_radius),
                              double(d.filter_alpha), double(d.eps), d.task_grid_size, double(d.camera.fov),
                              double(d.camera.lens_radius), double(d.camera.focal_distance), double(d.camera.pos[0]),
                              double(d.camera.pos[1]), double(d.camera.pos[2]));
                out += buf;
            } else if (mode == "refuse") {
                // render each entry; report what it threw, if anything
                CountingReporter rep(renderer.get());
                std::string err;
                try {
                    renderer->render(applier, scene, rep);
                } catch (const std::exception& ex) {
                    err = ex.what();
                }
                for (char& ch : err)
                    if (ch == '"' || ch == '\\' || ch == '\n') ch = ' ';
                out += "{\"entry\": " + std::to_string(i) + ", \"error\": \"" + err + "\"}\n";
            } else if (mode == "async" && i == 0) {
                // 1. run to the end: doing_rendering_ is raised throughout
                CountingReporter full(renderer.get());
                renderer->render_async(applier, scene, full);
                RenderTarget rt = renderer->wait_async();
                const int full_status = pt->last_status();
                const double full_weight = pt->last_weight_sum();
                // 2. stopped by stop_async after the second progress report
                CountingReporter part(renderer.get());
                renderer->render_async(applier, scene, part);
                const auto t0 = std::chrono::steady_clock::now();
                while (part.calls < 2 && std::chrono::steady_clock::now() - t0 < std::chrono::seconds(120))
                    std::this_thread::sleep_for(std::chrono::milliseconds(1));
                renderer->stop_async();
                char buf[512];
                std::snprintf(buf, sizeof(buf),
                              "{\"full_status\": %d, \"full_weight\": %.17g, \"full_progress\": %d, "
                              "\"doing_seen\": %d, \"image_rows\": %d, \"stop_status\": %d, \"stop_weight\": %.17g, "
                              "\"stop_progress\": %d, \"doing_after\": %d}\n",
                              full_status, full_weight, int(full.calls), int(full.doing_seen), rt.image.h,
                              pt->last_status(), pt->last_weight_sum(), int(part.calls),
                              int(renderer->is_doing_rendering()));
                out += buf;
            }
        }
        std::fputs(out.c_str(), stdout);
        return 0;
    } catch (const std::exception& ex) {
        std::fprintf(stderr, "binding_test: %s\n", ex.what());
        return 1;
    }
}
