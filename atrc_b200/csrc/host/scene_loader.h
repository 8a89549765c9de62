// Scene ingestion: Atrc JSON config -> flattened AtrcSceneDesc.
//
// Mirrors the reference's factory (src/factory/src/creator/*.cpp, the
// `reference` creator of src/factory/include/agz/factory/context.h:179-208)
// for every creator on the `pt` hot path.  Objects are recorded into flat
// tables instead of being built as virtual C++ objects, so that the device
// side can consume them.
#pragma once

#include <memory>
#include <string>
#include <vector>

#include "../../../include/atrc_cuda.h"
#include "config.h"

namespace atrc {

struct RenderingEntry {
    AtrcRenderDesc desc;
    std::string renderer_type;
    std::string post_processors_json;  // re-serialised `post_processors` array
};

struct LoadedConfig {
    std::shared_ptr<ConfigGroup> root;
    std::string scene_dir;

    // owned storage behind the POD descriptors
    std::vector<std::vector<float>> mesh_storage;
    std::vector<std::vector<float>> image_storage;
    std::vector<AtrcMeshDesc> meshes;
    std::vector<AtrcGeometryDesc> geometries;
    std::vector<AtrcEntityDesc> entities;
    std::vector<AtrcMaterialDesc> materials;
    std::vector<AtrcTexture2DDesc> textures2d;
    std::vector<AtrcTexture3DDesc> textures3d;
    std::vector<AtrcMediumDesc> media;
    AtrcSceneDesc scene{};

    std::vector<RenderingEntry> renderings;
};

// Parse a config.  Throws ConfigError (or std::runtime_error for I/O).
std::unique_ptr<LoadedConfig> load_config_string(const std::string& json,
                                                 const std::string& scene_dir);
std::unique_ptr<LoadedConfig> load_config_file(const std::string& path);

// ---- file formats (host) ---------------------------------------------------
// Returns RGB float texels, row 0 first; width/height out.
std::vector<float> load_rgb_image(const std::string& filename, int* width, int* height);
// `.bm` (src/factory/src/utility/bin_mesh.cpp:7-27) or Wavefront OBJ.
std::vector<float> load_triangle_mesh(const std::string& filename);
// Writers used by the CLI's post processors; `rgb` is a film (row 0 = bottom).
void save_pfm(const std::string& filename, const float* rgb, int w, int h);
void save_png8(const std::string& filename, const float* rgb, int w, int h, float gamma);
// 8-bit rows top to bottom.
void write_png_bytes(const std::string& filename, const uint8_t* rgb8, int w, int h);
void save_hdr_rgbe(const std::string& filename, const float* rgb, int w, int h);

}  // namespace atrc
