// Host half of the C ABI: configuration loading, error reporting and film
// resolution.  None of these functions touches a GPU.
#include <cstring>
#include <string>

#include "../../../include/atrc_cuda.h"
#include "scene_loader.h"

namespace atrc {

namespace {
thread_local std::string g_last_error;
}

void set_last_error(const std::string& msg) { g_last_error = msg; }

}  // namespace atrc

struct AtrcConfig {
    std::unique_ptr<atrc::LoadedConfig> cfg;
};

using atrc::set_last_error;

namespace {

template <class F>
int guarded_host(F&& f) {
    try {
        return f();
    } catch (const atrc::ConfigError& e) {
        set_last_error(e.what());
        return ATRC_ERR_CONFIG;
    } catch (const std::bad_alloc&) {
        set_last_error("host allocation failed");
        return ATRC_ERR_OUT_OF_MEMORY;
    } catch (const std::exception& e) {
        set_last_error(e.what());
        return ATRC_ERR_CONFIG;
    }
}

}  // namespace

extern "C" {

int atrc_abi_version(void) { return ATRC_ABI_VERSION; }

const char* atrc_last_error(void) { return atrc::g_last_error.c_str(); }

int atrc_abi_struct_sizes(uint64_t* sizes, int n) {
    const uint64_t s[17] = {sizeof(AtrcSceneDesc), sizeof(AtrcMeshDesc), sizeof(AtrcGeometryDesc),
                            sizeof(AtrcEntityDesc), sizeof(AtrcTexture2DDesc), sizeof(AtrcTexture3DDesc),
                            sizeof(AtrcMaterialDesc), sizeof(AtrcMediumDesc), sizeof(AtrcEnvDesc),
                            sizeof(AtrcRenderDesc), sizeof(AtrcFilm), sizeof(AtrcRenderStats), sizeof(AtrcRay),
                            sizeof(AtrcHit), sizeof(AtrcDeviceInfo), sizeof(AtrcTuning), sizeof(AtrcBvhBuildInfo)};
    for (int i = 0; sizes && i < n && i < 17; ++i) sizes[i] = s[i];
    return 17;
}

int atrc_config_load_file(const char* path, AtrcConfig** out) {
    if (!path || !out) { set_last_error("atrc_config_load_file: null argument"); return ATRC_ERR_INVALID_ARG; }
    *out = nullptr;
    return guarded_host([&] {
        auto c = std::make_unique<AtrcConfig>();
        c->cfg = atrc::load_config_file(path);
        *out = c.release();
        return int(ATRC_OK);
    });
}

int atrc_config_load_string(const char* json, const char* scene_dir, AtrcConfig** out) {
    if (!json || !out) { set_last_error("atrc_config_load_string: null argument"); return ATRC_ERR_INVALID_ARG; }
    *out = nullptr;
    return guarded_host([&] {
        auto c = std::make_unique<AtrcConfig>();
        c->cfg = atrc::load_config_string(json, scene_dir ? scene_dir : "");
        *out = c.release();
        return int(ATRC_OK);
    });
}

void atrc_config_destroy(AtrcConfig* cfg) { delete cfg; }

int atrc_config_scene(const AtrcConfig* cfg, const AtrcSceneDesc** out) {
    if (!cfg || !out) { set_last_error("atrc_config_scene: null argument"); return ATRC_ERR_INVALID_ARG; }
    *out = &cfg->cfg->scene;
    return ATRC_OK;
}

int atrc_config_rendering_count(const AtrcConfig* cfg, int* out) {
    if (!cfg || !out) { set_last_error("atrc_config_rendering_count: null argument"); return ATRC_ERR_INVALID_ARG; }
    *out = int(cfg->cfg->renderings.size());
    return ATRC_OK;
}

int atrc_config_rendering(const AtrcConfig* cfg, int index, AtrcRenderDesc* out, char* renderer_type, size_t cap) {
    if (!cfg || !out) { set_last_error("atrc_config_rendering: null argument"); return ATRC_ERR_INVALID_ARG; }
    if (index < 0 || size_t(index) >= cfg->cfg->renderings.size()) {
        set_last_error("atrc_config_rendering: index out of range");
        return ATRC_ERR_INVALID_ARG;
    }
    const auto& r = cfg->cfg->renderings[index];
    *out = r.desc;
    if (renderer_type && cap) {
        std::strncpy(renderer_type, r.renderer_type.c_str(), cap - 1);
        renderer_type[cap - 1] = '\0';
    }
    return ATRC_OK;
}

int atrc_config_post_processors(const AtrcConfig* cfg, int index, char* json_out, size_t cap, size_t* needed) {
    if (!cfg) { set_last_error("atrc_config_post_processors: null argument"); return ATRC_ERR_INVALID_ARG; }
    if (index < 0 || size_t(index) >= cfg->cfg->renderings.size()) {
        set_last_error("atrc_config_post_processors: index out of range");
        return ATRC_ERR_INVALID_ARG;
    }
    const std::string& s = cfg->cfg->renderings[index].post_processors_json;
    if (needed) *needed = s.size() + 1;
    if (json_out && cap) {
        std::strncpy(json_out, s.c_str(), cap - 1);
        json_out[cap - 1] = '\0';
    }
    return ATRC_OK;
}

int atrc_save_image(const char* filename, const char* ext, const float* rgb, int width, int height, float gamma) {
    if (!filename || !rgb || width <= 0 || height <= 0 || !(gamma > 0)) {
        set_last_error("atrc_save_image: invalid argument");
        return ATRC_ERR_INVALID_ARG;
    }
    return guarded_host([&] {
        std::string e = ext ? ext : "";
        const std::string fn = filename;
        if (e.empty()) {
            const size_t dot = fn.rfind('.');
            e = dot == std::string::npos ? "" : fn.substr(dot + 1);
        }
        if (e == "png") atrc::save_png8(fn, rgb, width, height, gamma);
        else if (e == "hdr") atrc::save_hdr_rgbe(fn, rgb, width, height);
        else if (e == "pfm") atrc::save_pfm(fn, rgb, width, height);
        else throw atrc::ConfigError("unsupported image extension: " + e + " (png, hdr, pfm)");
        return int(ATRC_OK);
    });
}

int atrc_save_png_bytes(const char* filename, const uint8_t* rgb8, int width, int height) {
    if (!filename || !rgb8 || width <= 0 || height <= 0) {
        set_last_error("atrc_save_png_bytes: invalid argument");
        return ATRC_ERR_INVALID_ARG;
    }
    return guarded_host([&] {
        atrc::write_png_bytes(filename, rgb8, width, height);
        return int(ATRC_OK);
    });
}

int atrc_film_resolve(const AtrcFilm* film, int width, int height, float* rgb) {
    if (!film || !film->value || !film->weight || !rgb || width <= 0 || height <= 0) {
        set_last_error("atrc_film_resolve: invalid argument");
        return ATRC_ERR_INVALID_ARG;
    }
    if (film->on_device) {
        set_last_error("atrc_film_resolve: host film expected");
        return ATRC_ERR_INVALID_ARG;
    }
    const size_t n = size_t(width) * height;
    for (size_t i = 0; i < n; ++i) {
        const double w = film->weight[i];
        const double r = w > 0 ? 1.0 / w : 1.0;  // perpixel_renderer.cpp:180-191
        for (int c = 0; c < 3; ++c) rgb[3 * i + c] = float(film->value[3 * i + c] * r);
    }
    return ATRC_OK;
}

}  // extern "C"
