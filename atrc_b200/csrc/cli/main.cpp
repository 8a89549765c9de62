// atrc_cli -- command-line driver for pt_cuda, mirroring the reference's
// `CLI -d scene.json` / `CLI -s "<json>"` (src/cli/src/main.cpp:14-72,
// src/cli/src/params.cpp:6-43).  Every `rendering` entry of the configuration
// is rendered on the GPU through the C ABI and its `save_to_img` post
// processors run.  `--renderer pt_cuda` (or `--gpu`) renders entries written
// for the CPU `pt` and `ao` renderers unchanged.
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "../../../include/atrc_cuda.h"

namespace {

void usage() {
    std::printf(
        "usage: atrc_cli (-d scene.json | -s '<json>') [--renderer pt_cuda | --gpu] [--device N] [--quiet]\n"
        "  -d, --scene-filename  scene description file\n"
        "  -s, --scene           scene description text\n"
        "  --renderer pt_cuda    render entries whose renderer type is `pt` or `ao` on the GPU as well\n"
        "  --gpu                 the same as --renderer pt_cuda\n");
}

bool check(int rc, const char* what) {
    if (rc == ATRC_OK) return true;
    std::fprintf(stderr, "error: %s failed (%d): %s\n", what, rc, atrc_last_error());
    return false;
}

void progress(double pct, void*) {
    std::printf("\r  %.1f%%", pct);
    std::fflush(stdout);
}

}  // namespace

int main(int argc, char** argv) {
    std::string file, text, force;
    int device = 0;
    bool quiet = false;
    for (int i = 1; i < argc; ++i) {
        std::string a = argv[i];
        if ((a == "-d" || a == "--scene-filename") && i + 1 < argc) file = argv[++i];
        else if ((a == "-s" || a == "--scene") && i + 1 < argc) text = argv[++i];
        else if (a == "--renderer" && i + 1 < argc) force = argv[++i];
        else if (a == "--gpu") force = "pt_cuda";
        else if (a == "--device" && i + 1 < argc) device = std::atoi(argv[++i]);
        else if (a == "--quiet") quiet = true;
        else { usage(); return a == "-h" || a == "--help" ? 0 : 1; }
    }
    if (file.empty() && text.empty()) { usage(); return 1; }
    std::string scene_dir = std::filesystem::current_path().string();
    AtrcConfig* cfg = nullptr;
    if (!text.empty()) {
        if (!check(atrc_config_load_string(text.c_str(), scene_dir.c_str(), &cfg), "loading the scene")) return 1;
    } else {
        scene_dir = std::filesystem::absolute(std::filesystem::path(file)).parent_path().string();
        if (!check(atrc_config_load_file(file.c_str(), &cfg), "loading the scene")) return 1;
    }
    AtrcDeviceInfo info;
    if (!check(atrc_cuda_device_init(device, &info), "initialising the device")) return 1;
    if (!quiet) std::printf("device %d: %s, %d SMs\n", device, info.name, info.sm_count);
    const AtrcSceneDesc* sd = nullptr;
    atrc_config_scene(cfg, &sd);
    AtrcScene* scene = nullptr;
    auto t0 = std::chrono::steady_clock::now();
    if (!check(atrc_cuda_scene_create(sd, &scene), "creating the device scene")) return 1;
    if (!quiet)
        std::printf("scene: %u entities, built in %.2f s\n", sd->entity_count,
                    std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count());
    int n = 0;
    atrc_config_rendering_count(cfg, &n);
    int rc_all = 0;
    for (int r = 0; r < n; ++r) {
        AtrcRenderDesc desc;
        char type[32];
        atrc_config_rendering(cfg, r, &desc, type, sizeof(type));
        if (std::string(type) != "pt_cuda" && force != "pt_cuda") {
            std::fprintf(stderr, "rendering %d: renderer `%s` runs on the CPU reference; pass --gpu\n", r,
                         type);
            rc_all = 1;
            continue;
        }
        const size_t np = size_t(desc.width) * desc.height;
        std::vector<double> value(np * 3), weight(np);
        AtrcFilm film{};
        film.value = value.data();
        film.weight = weight.data();
        AtrcRenderStats st;
        if (!quiet) std::printf("rendering %d: %dx%d, %d spp\n", r, desc.width, desc.height, desc.spp);
        if (!check(atrc_cuda_render(scene, &desc, &film, nullptr, quiet ? nullptr : progress, nullptr, &st), "rendering")) {
            rc_all = 1;
            continue;
        }
        if (!quiet)
            std::printf("\n  %.3f s, %.1f Msamples/s, %.1f Mrays/s\n", st.seconds, st.samples / st.seconds / 1e6,
                        (st.rays_closest + st.rays_shadow) / st.seconds / 1e6);
        // the rendering's post processors, on the device, in order
        size_t need = 0;
        atrc_config_post_processors(cfg, r, nullptr, 0, &need);
        std::string pj(need, '\0');
        atrc_config_post_processors(cfg, r, pj.data(), need, nullptr);
        std::vector<char> log(4096, 0);
        if (!check(atrc_cuda_post_process(&film, desc.width, desc.height, pj.c_str(), scene_dir.c_str(), log.data(),
                                          log.size()),
                   "post processing"))
            rc_all = 1;
        else if (!quiet)
            std::printf("%s", log.data());
    }
    atrc_cuda_scene_destroy(scene);
    atrc_config_destroy(cfg);
    return rc_all;
}
