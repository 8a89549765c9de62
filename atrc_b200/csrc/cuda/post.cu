// The output path on the device: film resolve, the reference's post
// processors and the 8-bit encoding of its image writers.
//
//  - resolve: value / weight per pixel (perpixel_renderer.cpp:180-191), the
//    G-buffer likewise;
//  - `gamma` (gamma.cpp:19-31): c^gamma; `aces` (aces.cpp:12-19,52-63):
//    the curve x (2.51 x + 0.03) / (x (2.43 x + 0.59) + 0.14) clamped to
//    [0, 1] of c * exposure;
//  - `save_to_img` (save_to_img.cpp:10-69) and `save_gbuffer_to_png`
//    (save_gbuffer.cpp:11-40): the film flipped vertically (row 0 is the
//    bottom of the picture) and uint8(clamp(c^gamma, 0, 1) * 255); normals
//    as (n + 1) / 2.
// Every kernel is one pass over the pixels (HBM-bound elementwise work).
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <filesystem>
#include <memory>
#include <string>
#include <vector>

#include "../../../include/atrc_cuda.h"
#include "../host/config.h"
#include "../host/scene_loader.h"
#include "cuda_util.h"

namespace atrc {
namespace {

__global__ void k_resolve(const double* __restrict__ sum, const double* __restrict__ weight, int channels, size_t n,
                          float* __restrict__ out) {
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) {
        const double w = weight[i];
        for (int c = 0; c < channels; ++c) out[i * channels + c] = w > 0 ? float(sum[i * channels + c] / w) : 0.0f;
    }
}

__device__ __forceinline__ float aces_curve(float x) {
    return fminf(fmaxf((x * (2.51f * x + 0.03f)) / (x * (2.43f * x + 0.59f) + 0.14f), 0.0f), 1.0f);
}

__global__ void k_post(float* __restrict__ rgb, size_t n, int type, float v) {
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) {
        const float c = rgb[i];
        rgb[i] = type == ATRC_POST_GAMMA ? powf(c, v) : type == ATRC_POST_ACES ? aces_curve(c * v) : (c + 1.0f) * 0.5f;
    }
}

// rows top to bottom (source row h - 1 - y), uint8(clamp(c^gamma, 0, 1) * 255)
__global__ void k_encode_ldr(const float* __restrict__ rgb, int w, int h, float gamma, uint8_t* __restrict__ out) {
    const size_t n = size_t(w) * h * 3;
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) {
        const size_t row = i / (size_t(w) * 3), col = i % (size_t(w) * 3);
        float v = powf(rgb[(size_t(h) - 1 - row) * size_t(w) * 3 + col], gamma);
        v = fminf(fmaxf(v, 0.0f), 1.0f);
        if (!(v == v)) v = 0.0f;
        out[i] = uint8_t(v * 255.0f);
    }
}

int grid_of(size_t n) { return int(std::min<size_t>((n + 255) / 256, 4096)); }

int pfail(int code, const std::string& m) {
    set_last_error(m);
    return code;
}

template <class F>
int pguarded(F&& f) {
    try {
        return f();
    } catch (const CudaError& e) {
        return pfail(ATRC_ERR_CUDA, e.what());
    } catch (const ConfigError& e) {
        return pfail(ATRC_ERR_CONFIG, e.what());
    } catch (const std::exception& e) {
        return pfail(ATRC_ERR_UNSUPPORTED, e.what());
    }
}

std::string replace_all(std::string s, const std::string& from, const std::string& to) {
    for (size_t p = s.find(from); p != std::string::npos; p = s.find(from, p + to.size())) s.replace(p, from.size(), to);
    return s;
}

}  // namespace
}  // namespace atrc

using namespace atrc;

extern "C" {

int atrc_cuda_film_resolve(const AtrcFilm* film, int width, int height, float* rgb, float* albedo, float* normal) {
    if (!film || !film->value || !film->weight || !rgb || width <= 0 || height <= 0)
        return pfail(ATRC_ERR_INVALID_ARG, "atrc_cuda_film_resolve: invalid argument");
    if (!film->on_device) return pfail(ATRC_ERR_INVALID_ARG, "atrc_cuda_film_resolve: the film must be on the device");
    return pguarded([&] {
        const size_t n = size_t(width) * height;
        k_resolve<<<grid_of(n), 256>>>(film->value, film->weight, 3, n, rgb);
        if (albedo && film->albedo) k_resolve<<<grid_of(n), 256>>>(film->albedo, film->weight, 3, n, albedo);
        if (normal && film->normal) k_resolve<<<grid_of(n), 256>>>(film->normal, film->weight, 3, n, normal);
        CK(cudaGetLastError());
        CK(cudaStreamSynchronize(0));
        return int(ATRC_OK);
    });
}

int atrc_cuda_post_apply(float* rgb, int width, int height, int32_t type, float value) {
    if (!rgb || width <= 0 || height <= 0 || type < ATRC_POST_GAMMA || type > ATRC_POST_NORMAL_TO_COLOR)
        return pfail(ATRC_ERR_INVALID_ARG, "atrc_cuda_post_apply: invalid argument");
    if (type == ATRC_POST_GAMMA && !(value > 0)) return pfail(ATRC_ERR_INVALID_ARG, "invalid gamma value");
    if (type == ATRC_POST_ACES && !(value >= 0)) return pfail(ATRC_ERR_INVALID_ARG, "invalid exposure value");
    return pguarded([&] {
        const size_t n = size_t(width) * height * 3;
        k_post<<<grid_of(n), 256>>>(rgb, n, type, value);
        CK(cudaGetLastError());
        CK(cudaStreamSynchronize(0));
        return int(ATRC_OK);
    });
}

int atrc_cuda_encode_ldr(const float* rgb, int width, int height, float gamma, uint8_t* out) {
    if (!rgb || !out || width <= 0 || height <= 0) return pfail(ATRC_ERR_INVALID_ARG, "atrc_cuda_encode_ldr: invalid argument");
    return pguarded([&] {
        const size_t n = size_t(width) * height * 3;
        k_encode_ldr<<<grid_of(n), 256>>>(rgb, width, height, gamma, out);
        CK(cudaGetLastError());
        CK(cudaStreamSynchronize(0));
        return int(ATRC_OK);
    });
}

int atrc_cuda_post_process(const AtrcFilm* film, int width, int height, const char* post_json, const char* scene_dir,
                           char* log, size_t log_cap) {
    if (!film || !film->value || !film->weight || !post_json || width <= 0 || height <= 0)
        return pfail(ATRC_ERR_INVALID_ARG, "atrc_cuda_post_process: invalid argument");
    if (log && log_cap) log[0] = 0;
    return pguarded([&] {
        std::string report;
        const size_t np = size_t(width) * height;
        // the film on the device (uploaded when the caller holds it on the host)
        AtrcFilm f = *film;
        DevBuf up;
        if (!film->on_device) {
            const bool a = film->albedo != nullptr, nn = film->normal != nullptr;
            up.alloc(np * 8 * (4 + (a ? 3 : 0) + (nn ? 3 : 0)));
            double* b = up.as<double>();
            CK(cudaMemcpy(b, film->value, np * 24, cudaMemcpyHostToDevice));
            CK(cudaMemcpy(b + np * 3, film->weight, np * 8, cudaMemcpyHostToDevice));
            f.value = b;
            f.weight = b + np * 3;
            f.albedo = a ? b + np * 4 : nullptr;
            f.normal = nn ? b + np * (a ? 7 : 4) : nullptr;
            if (a) CK(cudaMemcpy(f.albedo, film->albedo, np * 24, cudaMemcpyHostToDevice));
            if (nn) CK(cudaMemcpy(f.normal, film->normal, np * 24, cudaMemcpyHostToDevice));
            f.on_device = 1;
        }
        DevBuf img, ldr;
        img.alloc(np * 3 * 4);
        ldr.alloc(np * 3);
        int rc = atrc_cuda_film_resolve(&f, width, height, img.as<float>(), nullptr, nullptr);
        if (rc != ATRC_OK) return rc;
        const auto doc = parse_json_config(std::string("{\"p\": ") + post_json + "}");
        const ConfigArray& ops = doc->child_array("p");
        const std::string sd = scene_dir ? scene_dir : ".";
        auto map_path = [&](const std::string& s) {
            return replace_all(replace_all(s, "${scene-directory}", sd), "${working-directory}",
                               std::filesystem::current_path().string());
        };
        auto save_ldr = [&](const float* dev_rgb, float gamma, const std::string& fn) {
            std::filesystem::create_directories(std::filesystem::absolute(fn).parent_path());
            int r = atrc_cuda_encode_ldr(dev_rgb, width, height, gamma, ldr.as<uint8_t>());
            if (r != ATRC_OK) throw std::runtime_error(atrc_last_error());
            std::vector<uint8_t> bytes(np * 3);
            CK(cudaMemcpy(bytes.data(), ldr.p, np * 3, cudaMemcpyDeviceToHost));
            r = atrc_save_png_bytes(fn.c_str(), bytes.data(), width, height);
            if (r != ATRC_OK) throw std::runtime_error(atrc_last_error());
        };
        for (size_t k = 0; k < ops.size(); ++k) {
            const ConfigGroup& op = ops.at(k).as_group();
            const std::string t = op.child_str("type");
            if (ends_with(t, "//")) continue;  // commented out
            if (t == "gamma") {  // GammaCreator (post_processor_creators.cpp:26-45)
                const float g = op.find_child("gamma") ? op.child_real("gamma") : 1.0f / op.child_real("inv_gamma");
                rc = atrc_cuda_post_apply(img.as<float>(), width, height, ATRC_POST_GAMMA, g);
            } else if (t == "aces") {  // ACESCreator (post_processor_creators.cpp:9-24)
                rc = atrc_cuda_post_apply(img.as<float>(), width, height, ATRC_POST_ACES, op.child_real("exposure"));
            } else if (t == "save_to_img") {  // SaveImgCreator (post_processor_creators.cpp:110-150)
                const std::string fn = map_path(op.child_str("filename"));
                float gamma = 1;
                if (op.find_child("gamma")) gamma = op.child_real("gamma");
                else if (op.find_child("inv_gamma")) gamma = 1 / op.child_real("inv_gamma");
                std::string ext = op.child_str_or("ext", "");
                if (ext.empty()) ext = ends_with(fn, ".png") ? "png" : ends_with(fn, ".hdr") ? "hdr" :
                                       ends_with(fn, ".pfm") ? "pfm" : ends_with(fn, ".jpg") ? "jpg" : "";
                if (ext == "png") {
                    save_ldr(img.as<float>(), gamma, fn);
                } else if (ext == "hdr" || ext == "pfm") {
                    std::vector<float> host(np * 3);
                    CK(cudaMemcpy(host.data(), img.p, np * 12, cudaMemcpyDeviceToHost));
                    std::filesystem::create_directories(std::filesystem::absolute(fn).parent_path());
                    rc = atrc_save_image(fn.c_str(), ext.c_str(), host.data(), width, height, gamma);
                } else {
                    throw ConfigError("unknown image file format: " + fn + " (png, hdr, pfm)");
                }
                report += "saved " + fn + "\n";
            } else if (t == "save_gbuffer_to_png") {  // SaveGBufferCreator (post_processor_creators.cpp:87-108)
                for (const char* key : {"albedo", "normal"}) {
                    if (!op.find_child(key)) continue;
                    const double* src = std::string(key) == "albedo" ? f.albedo : f.normal;
                    if (!src) continue;  // not rendered with a G-buffer
                    DevBuf g;
                    g.alloc(np * 12);
                    k_resolve<<<grid_of(np), 256>>>(src, f.weight, 3, np, g.as<float>());
                    CK(cudaGetLastError());
                    if (std::string(key) == "normal")
                        rc = atrc_cuda_post_apply(g.as<float>(), width, height, ATRC_POST_NORMAL_TO_COLOR, 0);
                    const std::string fn = map_path(op.child_str(key));
                    save_ldr(g.as<float>(), 1.0f, fn);
                    report += "saved " + fn + "\n";
                }
            } else {
                // resize (third-party avir resampler) and oidn_denoiser
                // (optional Intel library) are not part of pt_cuda
                report += "skipped " + t + "\n";
            }
            if (rc != ATRC_OK) return rc;
        }
        if (log && log_cap) {
            std::strncpy(log, report.c_str(), log_cap - 1);
            log[log_cap - 1] = 0;
        }
        return int(ATRC_OK);
    });
}

}  // extern "C"
