// Atrc JSON -> AtrcSceneDesc.  Each creator below cites the reference creator
// whose parameters, defaults and error behaviour it mirrors.
#include "scene_loader.h"

#include <climits>
#include <cmath>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <map>
#include <sstream>

namespace atrc {

namespace {

const float kPi = 3.14159265358979323846f;

std::string read_text_file(const std::string& path) {
    std::ifstream f(path, std::ios::binary);
    if (!f) throw ConfigError("failed to open file: " + path);
    std::stringstream ss;
    ss << f.rdbuf();
    return ss.str();
}

AtrcTransform to_desc(const Affine& a) {
    AtrcTransform t;
    std::memcpy(t.m, a.m, sizeof(t.m));
    std::memcpy(t.inv, a.inv, sizeof(t.inv));
    return t;
}

AtrcTransform identity_desc() {
    AtrcTransform t;
    affine_identity(t.m);
    affine_identity(t.inv);
    return t;
}

void json_escape(std::string& out, const std::string& s) {
    out += '"';
    for (char c : s) {
        if (c == '"' || c == '\\') { out += '\\'; out += c; }
        else if (c == '\n') out += "\\n";
        else out += c;
    }
    out += '"';
}

void node_to_json(const ConfigNode& n, std::string& out) {
    if (n.is_value()) { json_escape(out, n.as_value().as_str()); return; }
    if (n.is_array()) {
        const auto& a = n.as_array();
        out += '[';
        for (size_t i = 0; i < a.size(); ++i) {
            if (i) out += ',';
            node_to_json(a.at(i), out);
        }
        out += ']';
        return;
    }
    out += '{';
    bool first = true;
    for (auto& kv : n.as_group().children()) {
        if (!first) out += ',';
        first = false;
        json_escape(out, kv.first);
        out += ':';
        node_to_json(*kv.second, out);
    }
    out += '}';
}

// A flattened geometry chain (transform_wrapper / double_sided / leaf).
struct GeomRef {
    int leaf = -1;
    bool has_instance = false;
    Affine instance{};
    bool double_sided = false;
};

class SceneBuilder {
public:
    SceneBuilder(LoadedConfig& out, const ConfigGroup& scene_root, const std::string& scene_dir)
        : out_(out), scene_root_(scene_root), scene_dir_(scene_dir) {
        working_dir_ = std::filesystem::current_path().string();
        // medium 0 is the shared void medium (entity_creators.cpp:11-27)
        AtrcMediumDesc v{};
        v.type = ATRC_MED_VOID;
        v.max_scattering_count = INT_MAX;
        v.transform = identity_desc();
        v.density = v.albedo = v.g_tex = -1;
        out_.media.push_back(v);
    }

    // BasicPathMapper::map (context.h:157-177)
    std::string map_path(const std::string& s) const {
        std::string r = s;
        bool done = false;
        while (!done) {
            done = true;
            for (auto& p : {std::make_pair(std::string("${scene-directory}"), scene_dir_),
                            std::make_pair(std::string("${working-directory}"), working_dir_)}) {
                size_t pos;
                while ((pos = r.find(p.first)) != std::string::npos) {
                    r.replace(pos, p.first.size(), p.second);
                    done = false;
                }
            }
        }
        return std::filesystem::absolute(std::filesystem::path(r)).lexically_normal().string();
    }

    // ReferenceCreator<T>::create (context.h:179-208): names index the scene
    // root, the created object is shared by every reference with those names.
    const ConfigGroup& resolve_reference(const ConfigGroup& params, std::string* key) const {
        const ConfigArray& names = params.child_array("name");
        if (names.size() < 1) throw ConfigError("empty reference name sequence");
        const ConfigGroup* g = &scene_root_;
        std::string k;
        for (size_t i = 0; i < names.size(); ++i) {
            k += names.at_str(i);
            k += '\x1f';
            if (i + 1 < names.size()) g = &g->child_group(names.at_str(i));
        }
        *key = k;
        return g->child_group(names.at_str(names.size() - 1));
    }

    // ------------------------------------------------------------- textures
    int create_texture2d(const ConfigGroup& p) {
        const std::string type = p.child_str("type");
        if (type == "reference") {
            std::string key;
            const ConfigGroup& g = resolve_reference(p, &key);
            auto it = tex2d_refs_.find(key);
            if (it != tex2d_refs_.end()) return it->second;
            int r = create_texture2d(g);
            tex2d_refs_[key] = r;
            return r;
        }
        AtrcTexture2DDesc t{};
        t.tex3d = -1;
        // Texture2DCommonParams::from_params / full_transform (texture2d.h:8-53)
        const bool inv_u = p.child_int_or("inv_u", 0) != 0;
        const bool inv_v = p.child_int_or("inv_v", 0) != 0;
        const bool swap_uv = p.child_int_or("swap_uv", 0) != 0;
        Affine2 user = p.child_transform2_or_identity("transform");
        Affine2 full;
        full.m[0] = 1; full.m[1] = 0; full.m[2] = 0; full.m[3] = 0; full.m[4] = 1; full.m[5] = 0;
        auto mul = [](const Affine2& a, const Affine2& b) {
            Affine2 r;
            r.m[0] = a.m[0] * b.m[0] + a.m[1] * b.m[3];
            r.m[1] = a.m[0] * b.m[1] + a.m[1] * b.m[4];
            r.m[2] = a.m[0] * b.m[2] + a.m[1] * b.m[5] + a.m[2];
            r.m[3] = a.m[3] * b.m[0] + a.m[4] * b.m[3];
            r.m[4] = a.m[3] * b.m[1] + a.m[4] * b.m[4];
            r.m[5] = a.m[3] * b.m[2] + a.m[4] * b.m[5] + a.m[5];
            return r;
        };
        if (inv_v) { Affine2 f{{1, 0, 0, 0, -1, 1}}; full = mul(full, f); }
        if (inv_u) { Affine2 f{{-1, 0, 1, 0, 1, 0}}; full = mul(full, f); }
        if (swap_uv) { Affine2 f{{0, 1, 0, 1, 0, 0}}; full = mul(full, f); }
        full = mul(full, user);
        std::memcpy(t.uv_transform, full.m, sizeof(t.uv_transform));
        t.wrap_u = wrap_mode(p.child_str_or("wrap_u", "clamp"), "wrap_u");
        t.wrap_v = wrap_mode(p.child_str_or("wrap_v", "clamp"), "wrap_v");
        t.inv_gamma = p.child_real_or("inv_gamma", 1);
        if (type == "constant") {
            // Constant2D (constant2d.cpp:5-44): gamma applied once at creation
            Vec3 texel = p.child_spectrum("texel");
            if (t.inv_gamma != 1.0f) {
                texel.x = std::pow(texel.x, t.inv_gamma);
                texel.y = std::pow(texel.y, t.inv_gamma);
                texel.z = std::pow(texel.z, t.inv_gamma);
            }
            t.type = ATRC_TEX_CONSTANT;
            t.texel[0] = texel.x; t.texel[1] = texel.y; t.texel[2] = texel.z;
            t.inv_gamma = 1.0f;
        } else if (type == "checker_board") {  // CheckerBoardCreator (texture2d_creators.cpp:29-48)
            t.type = ATRC_TEX_CHECKER;
            t.grid_count = p.child_int("grid_count");
            if (t.grid_count <= 0) throw ConfigError("invalid grid_count value: " + std::to_string(t.grid_count));
            const Vec3 c1 = p.child_spectrum("color1"), c2 = p.child_spectrum("color2");
            t.texel[0] = c1.x; t.texel[1] = c1.y; t.texel[2] = c1.z;
            t.texel2[0] = c2.x; t.texel2[1] = c2.y; t.texel2[2] = c2.z;
        } else if (type == "solid_image") {
            // SolidImageCreator (texture2d_creators.cpp:148-163): a 3D
            // texture behind the 2D interface, without the 2D common
            // parameters (identity uv transform, clamp, no gamma)
            t.type = ATRC_TEX_SOLID;
            t.tex3d = create_texture3d(p.child_group("tex3d"));
            const float id[6] = {1, 0, 0, 0, 1, 0};
            std::memcpy(t.uv_transform, id, sizeof(id));
            t.wrap_u = t.wrap_v = ATRC_WRAP_CLAMP;
            t.inv_gamma = 1.0f;
        } else if (type == "hdr" || type == "image") {
            // HDRTexture (hdr.cpp:11-72) and ImageTexture (image.cpp): float
            // texels, 8-bit images as byte / 255 (from_color3b)
            const std::string fn = map_path(p.child_str("filename"));
            const std::string sampler = p.child_str_or("sample", "linear");
            if (sampler != "linear" && sampler != "nearest") throw ConfigError("invalid sample method");
            int w = 0, h = 0;
            auto data = load_rgb_image(fn, &w, &h);
            out_.image_storage.push_back(std::move(data));
            t.type = ATRC_TEX_IMAGE;
            t.width = w; t.height = h;
            t.data = out_.image_storage.back().data();
            t.nearest = sampler == "nearest";
        } else {
            throw ConfigError("unknown creator type name: " + type + " (texture2d)");
        }
        out_.textures2d.push_back(t);
        return int(out_.textures2d.size() - 1);
    }

    int constant_texture2d(float v) {
        AtrcTexture2DDesc t{};
        t.type = ATRC_TEX_CONSTANT;
        t.texel[0] = t.texel[1] = t.texel[2] = v;
        t.uv_transform[0] = 1; t.uv_transform[4] = 1;
        t.inv_gamma = 1;
        t.tex3d = -1;
        out_.textures2d.push_back(t);
        return int(out_.textures2d.size() - 1);
    }

    // helper::child_texture_or_constant (factory/help.h)
    int child_texture_or_constant(const ConfigGroup& p, const char* name, float v) {
        if (auto g = p.find_child_group(name)) return create_texture2d(*g);
        return constant_texture2d(v);
    }

    static int wrap_mode(const std::string& s, const char* what) {
        if (s == "clamp") return ATRC_WRAP_CLAMP;
        if (s == "repeat") return ATRC_WRAP_REPEAT;
        if (s == "mirror") return ATRC_WRAP_MIRROR;
        throw ConfigError(std::string("invalid ") + what + " value: " + s + " (expect clamp/repeat/mirror)");
    }

    int create_texture3d(const ConfigGroup& p) {
        const std::string type = p.child_str("type");
        if (type == "reference") {
            std::string key;
            const ConfigGroup& g = resolve_reference(p, &key);
            auto it = tex3d_refs_.find(key);
            if (it != tex3d_refs_.end()) return it->second;
            int r = create_texture3d(g);
            tex3d_refs_[key] = r;
            return r;
        }
        AtrcTexture3DDesc t{};
        // Texture3DCommonParams::full_transform (texture3d.h:46-99)
        const bool inv_u = p.child_int_or("inv_u", 0) != 0;
        const bool inv_v = p.child_int_or("inv_v", 0) != 0;
        const bool inv_w = p.child_int_or("inv_w", 0) != 0;
        int perm[3];
        p.child_vec3i_perm("uvw_perm", perm);
        Affine full = affine_from({1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0});
        if (inv_u) full = mul3(full, affine_from({-1, 0, 0, 1, 0, 1, 0, 0, 0, 0, 1, 0}));
        if (inv_v) full = mul3(full, affine_from({1, 0, 0, 0, 0, -1, 0, 1, 0, 0, 1, 0}));
        if (inv_w) full = mul3(full, affine_from({1, 0, 0, 0, 0, 1, 0, 0, 0, 0, -1, 1}));
        float pm[12] = {0};
        for (int r = 0; r < 3; ++r) {
            if (perm[r] < 0 || perm[r] >= 3) throw ConfigError("invalid uvw perm value");
            pm[4 * r + perm[r]] = 1;
        }
        full = mul3(full, affine_from({pm[0], pm[1], pm[2], pm[3], pm[4], pm[5], pm[6], pm[7], pm[8], pm[9], pm[10], pm[11]}));
        full = mul3(full, p.child_transform3_or_identity("transform"));
        std::memcpy(t.uvw_transform, full.m, sizeof(t.uvw_transform));
        t.uvw_perm[0] = 0; t.uvw_perm[1] = 1; t.uvw_perm[2] = 2;
        t.wrap[0] = wrap_mode(p.child_str_or("wrap_u", "clamp"), "wrap_u");
        t.wrap[1] = wrap_mode(p.child_str_or("wrap_v", "clamp"), "wrap_v");
        t.wrap[2] = wrap_mode(p.child_str_or("wrap_w", "clamp"), "wrap_w");
        t.inv_gamma = p.child_real_or("inv_gamma", 1);
        if (type == "constant") {
            Vec3 texel = p.child_spectrum("texel");
            t.type = ATRC_TEX_CONSTANT;
            t.texel[0] = texel.x; t.texel[1] = texel.y; t.texel[2] = texel.z;
            t.channels = 3;
            t.max_real = texel.x;
        } else if (type == "image3d") {
            // ImageTexture3D + texture3d_loader.cpp:11-37
            const std::string format = p.child_str("format");
            int ch;
            bool bytes;
            if (format == "real") { ch = 1; bytes = false; }
            else if (format == "spec") { ch = 3; bytes = false; }
            else if (format == "gray8") { ch = 1; bytes = true; }
            else if (format == "rgb8") { ch = 3; bytes = true; }
            else throw ConfigError("invalid image3d format: " + format);
            std::vector<float> data;
            int w = 0, h = 0, d = 0;
            if (auto n = p.find_child("binary_filename")) {
                std::ifstream f(map_path(n->as_value().as_str()), std::ios::binary);
                if (!f) throw ConfigError("failed to open 3d texture file");
                int32_t dims[3];
                f.read(reinterpret_cast<char*>(dims), sizeof(dims));
                if (!f) throw ConfigError("failed to read width/height/depth from file");
                w = dims[0]; h = dims[1]; d = dims[2];
                if (w <= 0 || h <= 0 || d <= 0) throw ConfigError("invalid 3d texture size");
                size_t n_el = size_t(w) * h * d * ch;
                data.resize(n_el);
                if (bytes) {
                    std::vector<uint8_t> b(n_el);
                    f.read(reinterpret_cast<char*>(b.data()), n_el);
                    for (size_t i = 0; i < n_el; ++i) data[i] = b[i] / 255.0f;
                } else {
                    f.read(reinterpret_cast<char*>(data.data()), n_el * sizeof(float));
                }
                if (!f) throw ConfigError("failed to parse texel data from file");
            } else if (auto n = p.find_child("ascii_filename")) {
                std::ifstream f(map_path(n->as_value().as_str()));
                if (!f) throw ConfigError("failed to open 3d texture file");
                f >> w >> h >> d;
                if (!f || w <= 0 || h <= 0 || d <= 0) throw ConfigError("failed to read width/height/depth from file");
                size_t n_el = size_t(w) * h * d * ch;
                data.resize(n_el);
                for (size_t i = 0; i < n_el; ++i) {
                    float v;
                    f >> v;
                    if (!f) throw ConfigError("failed to parse texel data from file");
                    data[i] = bytes ? v / 255.0f : v;
                }
            } else {
                throw ConfigError("image3d: binary_filename or ascii_filename expected "
                                  "(image slices are not supported by pt_cuda)");
            }
            float mx = -INFINITY;
            for (size_t i = 0; i < data.size(); i += ch) mx = std::fmax(mx, data[i]);
            out_.image_storage.push_back(std::move(data));
            t.type = ATRC_TEX_IMAGE;
            t.width = w; t.height = h; t.depth = d; t.channels = ch;
            t.data = out_.image_storage.back().data();
            const std::string sampler = p.child_str_or("sampler", "linear");
            t.nearest = sampler == "nearest";
            t.max_real = mx;
        } else {
            throw ConfigError("unknown creator type name: " + type + " (texture3d)");
        }
        out_.textures3d.push_back(t);
        return int(out_.textures3d.size() - 1);
    }

    // -------------------------------------------------------------- geometry
    GeomRef create_geometry(const ConfigGroup& p) {
        const std::string type = p.child_str("type");
        if (type == "reference") {
            std::string key;
            const ConfigGroup& g = resolve_reference(p, &key);
            auto it = geom_refs_.find(key);
            if (it != geom_refs_.end()) return it->second;
            GeomRef r = create_geometry(g);
            geom_refs_[key] = r;
            return r;
        }
        if (type == "transform_wrapper") {
            // TransformWrapperCreator (geometry_creators.cpp:100-117)
            GeomRef in = create_geometry(p.child_group("internal"));
            Affine t = p.child_transform3("transform");
            if (in.has_instance) {
                // nested wrappers collapse into one instance transform
                in.instance = mul3(t, in.instance);
            } else {
                in.instance = t;
                in.has_instance = true;
            }
            return in;
        }
        if (type == "double_sided") {
            GeomRef in = create_geometry(p.child_group("internal"));
            in.double_sided = true;
            return in;
        }
        AtrcGeometryDesc g{};
        g.mesh = -1;
        if (type == "triangle_bvh" || type == "triangle_bvh_noembree" || type == "triangle_bvh_embree") {
            g.type = ATRC_GEOM_TRIANGLE_BVH;
            g.transform = to_desc(p.child_transform3("transform"));
            const std::string fn = map_path(p.child_str("filename"));
            auto it = mesh_files_.find(fn);
            if (it != mesh_files_.end()) {
                g.mesh = it->second;
            } else {
                auto tris = load_triangle_mesh(fn);
                if (tris.empty()) throw ConfigError("empty mesh: " + fn);
                out_.mesh_storage.push_back(std::move(tris));
                AtrcMeshDesc m;
                m.triangle_count = out_.mesh_storage.back().size() / 24;
                m.vertices = out_.mesh_storage.back().data();
                out_.meshes.push_back(m);
                g.mesh = int(out_.meshes.size() - 1);
                mesh_files_[fn] = g.mesh;
            }
        } else if (type == "quad" || type == "triangle") {
            g.type = type == "quad" ? ATRC_GEOM_QUAD : ATRC_GEOM_TRIANGLE;
            g.transform = to_desc(p.child_transform3("transform"));
            const char* names[4] = {"A", "B", "C", "D"};
            const char* tnames[4] = {"tA", "tB", "tC", "tD"};
            int n = type == "quad" ? 4 : 3;
            for (int i = 0; i < n; ++i) {
                Vec3 v = p.child_vec3(names[i]);
                Vec2 t = p.child_vec2_or(tnames[i], Vec2(0));
                g.p[i][0] = v.x; g.p[i][1] = v.y; g.p[i][2] = v.z;
                g.uv[i][0] = t.x; g.uv[i][1] = t.y;
            }
        } else if (type == "sphere" || type == "disk") {
            g.type = type == "sphere" ? ATRC_GEOM_SPHERE : ATRC_GEOM_DISK;
            g.transform = to_desc(p.child_transform3("transform"));
            g.radius = p.child_real("radius");
        } else {
            throw ConfigError("unknown creator type name: " + type + " (geometry)");
        }
        out_.geometries.push_back(g);
        GeomRef r;
        r.leaf = int(out_.geometries.size() - 1);
        return r;
    }

    // -------------------------------------------------------------- material
    int create_material(const ConfigGroup& p) {
        const std::string type = p.child_str("type");
        if (type == "reference") {
            std::string key;
            const ConfigGroup& g = resolve_reference(p, &key);
            auto it = mat_refs_.find(key);
            if (it != mat_refs_.end()) return it->second;
            int r = create_material(g);
            mat_refs_[key] = r;
            return r;
        }
        AtrcMaterialDesc m{};
        for (int i = 0; i < ATRC_DISNEY_SLOT_COUNT; ++i) m.tex[i] = -1;
        m.normal_map = -1;
        m.bssrdf[0] = m.bssrdf[1] = m.bssrdf[2] = -1;
        if (type == "ideal_diffuse") {
            // material_creators.cpp (IdealDiffuseCreator)
            m.type = ATRC_MAT_IDEAL_DIFFUSE;
            m.tex[0] = create_texture2d(p.child_group("albedo"));
            if (auto n = p.find_child_group("normal_map")) m.normal_map = create_texture2d(*n);
        } else if (type == "ideal_black") {
            m.type = ATRC_MAT_IDEAL_BLACK;
        } else if (type == "invisible_surface") {
            m.type = ATRC_MAT_INVISIBLE_SURFACE;
        } else if (type == "disney") {
            // DisneyCreator (material_creators.cpp:56-113)
            m.type = ATRC_MAT_DISNEY;
            m.tex[ATRC_DISNEY_BASE_COLOR] = create_texture2d(p.child_group("base_color"));
            m.tex[ATRC_DISNEY_METALLIC] = create_texture2d(p.child_group("metallic"));
            m.tex[ATRC_DISNEY_ROUGHNESS] = create_texture2d(p.child_group("roughness"));
            m.tex[ATRC_DISNEY_TRANSMISSION] = child_texture_or_constant(p, "transmission", 0);
            if (auto n = p.find_child_group("transmission_roughness"))
                m.tex[ATRC_DISNEY_TRANSMISSION_ROUGHNESS] = create_texture2d(*n);
            else
                m.tex[ATRC_DISNEY_TRANSMISSION_ROUGHNESS] = m.tex[ATRC_DISNEY_ROUGHNESS];
            m.tex[ATRC_DISNEY_IOR] = child_texture_or_constant(p, "ior", 1.5f);
            m.tex[ATRC_DISNEY_SPECULAR_SCALE] = child_texture_or_constant(p, "specular_scale", 1);
            m.tex[ATRC_DISNEY_SPECULAR_TINT] = child_texture_or_constant(p, "specular_tint", 0);
            m.tex[ATRC_DISNEY_ANISOTROPIC] = child_texture_or_constant(p, "anisotropic", 0);
            m.tex[ATRC_DISNEY_SHEEN] = child_texture_or_constant(p, "sheen", 0);
            m.tex[ATRC_DISNEY_SHEEN_TINT] = child_texture_or_constant(p, "sheen_tint", 0);
            m.tex[ATRC_DISNEY_CLEARCOAT] = child_texture_or_constant(p, "clearcoat", 0);
            m.tex[ATRC_DISNEY_CLEARCOAT_GLOSS] = child_texture_or_constant(p, "clearcoat_gloss", 1);
            if (auto n = p.find_child_group("normal_map")) m.normal_map = create_texture2d(*n);
            // init_bssrdf_surface (material_creators.cpp:20-45): subsurface
            // scattering when bssrdf_dmfp is given; A defaults to the base
            // colour and eta to the ior
            if (p.find_child("bssrdf_dmfp")) {
                m.bssrdf[1] = create_texture2d(p.child_group("bssrdf_dmfp"));
                m.bssrdf[0] = p.find_child_group("bssrdf_A") ? create_texture2d(p.child_group("bssrdf_A"))
                                                             : m.tex[ATRC_DISNEY_BASE_COLOR];
                m.bssrdf[2] = p.find_child_group("bssrdf_eta") ? create_texture2d(p.child_group("bssrdf_eta"))
                                                               : m.tex[ATRC_DISNEY_IOR];
            }
        } else if (type == "mirror") {  // MirrorCreator (material_creators.cpp:270-289)
            m.type = ATRC_MAT_MIRROR;
            m.tex[0] = create_texture2d(p.child_group("color_map"));
            m.tex[1] = create_texture2d(p.child_group("eta"));
            m.tex[2] = create_texture2d(p.child_group("k"));
        } else if (type == "glass") {  // GlassCreator (material_creators.cpp:139-180)
            m.type = ATRC_MAT_GLASS;
            const int ior = create_texture2d(p.child_group("ior"));
            int refl = -1, refr = -1;
            if (auto n = p.find_child_group("color_map")) refl = refr = create_texture2d(*n);
            if (auto n = p.find_child_group("color_reflection_map")) refl = create_texture2d(*n);
            if (auto n = p.find_child_group("color_refraction_map")) refr = create_texture2d(*n);
            if (refl < 0 || refr < 0) throw ConfigError("empty color reflection/refraction map");
            m.tex[0] = refl;
            m.tex[1] = refr;
            m.tex[2] = ior;
        } else if (type == "metal") {  // MetalCreator (material_creators.cpp:235-268)
            m.type = ATRC_MAT_METAL;
            m.tex[0] = create_texture2d(p.child_group("color"));
            // the reference's create_metal(color, eta, k, ...) forwards its
            // arguments in that order to Metal(color, k, eta, ...)
            // (metal.cpp:23-27, 65-78), so the conductor Fresnel it renders
            // with takes the "k" map as the index of refraction and the "eta"
            // map as the absorption: the same swap here keeps parity
            m.tex[2] = create_texture2d(p.child_group("eta"));
            m.tex[1] = create_texture2d(p.child_group("k"));
            m.tex[3] = create_texture2d(p.child_group("roughness"));
            m.tex[4] = create_texture2d(p.child_group("anisotropic"));
            if (auto n = p.find_child_group("normal_map")) m.normal_map = create_texture2d(*n);
        } else if (type == "phong") {  // PhongCreator (material_creators.cpp:326-345)
            m.type = ATRC_MAT_PHONG;
            m.tex[0] = create_texture2d(p.child_group("d"));
            m.tex[1] = create_texture2d(p.child_group("s"));
            m.tex[2] = create_texture2d(p.child_group("ns"));
            if (auto n = p.find_child_group("normal_map")) m.normal_map = create_texture2d(*n);
        } else {
            throw ConfigError("material type '" + type + "' is not supported by pt_cuda");
        }
        out_.materials.push_back(m);
        return int(out_.materials.size() - 1);
    }

    // ---------------------------------------------------------------- medium
    int create_medium(const ConfigGroup& p) {
        const std::string type = p.child_str("type");
        if (type == "reference") {
            std::string key;
            const ConfigGroup& g = resolve_reference(p, &key);
            auto it = med_refs_.find(key);
            if (it != med_refs_.end()) return it->second;
            int r = create_medium(g);
            med_refs_[key] = r;
            return r;
        }
        AtrcMediumDesc m{};
        m.transform = identity_desc();
        m.density = m.albedo = m.g_tex = -1;
        m.max_scattering_count = p.child_int_or("max_scattering_count", INT_MAX);
        if (type == "void") {
            return 0;
        } else if (type == "homogeneous") {
            m.type = ATRC_MED_HOMOGENEOUS;
            Vec3 a = p.child_spectrum("sigma_a"), s = p.child_spectrum("sigma_s");
            m.sigma_a[0] = a.x; m.sigma_a[1] = a.y; m.sigma_a[2] = a.z;
            m.sigma_s[0] = s.x; m.sigma_s[1] = s.y; m.sigma_s[2] = s.z;
            m.g = p.child_real("g");
        } else if (type == "heterogeneous") {
            m.type = ATRC_MED_HETEROGENEOUS;
            m.transform = to_desc(p.child_transform3("transform"));
            m.density = create_texture3d(p.child_group("density"));
            m.albedo = create_texture3d(p.child_group("albedo"));
            m.g_tex = create_texture3d(p.child_group("g"));
            m.white_for_indirect = p.child_int_or("white_for_indirect", 0) != 0;
        } else {
            throw ConfigError("unknown creator type name: " + type + " (medium)");
        }
        out_.media.push_back(m);
        return int(out_.media.size() - 1);
    }

    // ---------------------------------------------------------------- entity
    void create_entity(const ConfigGroup& p) {
        const std::string type = p.child_str("type");
        if (type != "geometric")
            throw ConfigError("unknown creator type name: " + type + " (entity)");
        // GeometricEntityCreator (entity_creators.cpp:29-60)
        GeomRef g = create_geometry(p.child_group("geometry"));
        AtrcEntityDesc e{};
        e.geometry = g.leaf;
        e.has_instance = g.has_instance;
        e.instance = g.has_instance ? to_desc(g.instance) : identity_desc();
        e.double_sided = g.double_sided;
        e.material = create_material(p.child_group("material"));
        e.medium_in = p.find_child_group("med_in") ? create_medium(p.child_group("med_in")) : 0;
        e.medium_out = p.find_child_group("med_out") ? create_medium(p.child_group("med_out")) : 0;
        Vec3 er = p.child_spectrum_or("emit_radiance", Vec3(0));
        e.emit_radiance[0] = er.x; e.emit_radiance[1] = er.y; e.emit_radiance[2] = er.z;
        e.no_denoise = p.child_int_or("no_denoise", 0) != 0;
        e.power = p.child_real_or("power", -1);
        out_.entities.push_back(e);
    }

    void build_scene() {
        const ConfigGroup& p = scene_root_;
        const std::string type = p.child_str("type");
        if (type != "default") throw ConfigError("unknown creator type name: " + type + " (scene)");
        // DefaultSceneCreator (scene_creators.cpp:24-65)
        if (auto ents = p.find_child_array("entities")) {
            for (size_t i = 0; i < ents->size(); ++i) {
                const ConfigGroup& g = ents->at(i).as_group();
                if (ends_with(g.child_str("type"), "//")) continue;
                create_entity(g);
            }
        }
        AtrcEnvDesc env{};
        env.type = ATRC_ENV_NONE;
        env.tex = -1;
        if (auto g = p.find_child_group("env")) {
            const std::string et = g->child_str("type");
            env.power = g->child_real_or("power", -1);
            if (et == "ibl") {
                env.type = ATRC_ENV_IBL;
                env.tex = create_texture2d(g->child_group("tex"));
                env.no_importance_sampling = g->child_int_or("no_importance_sampling", 0) != 0;
            } else if (et == "native_sky") {
                env.type = ATRC_ENV_NATIVE_SKY;
                Vec3 t = g->child_spectrum("top"), b = g->child_spectrum("bottom");
                env.top[0] = t.x; env.top[1] = t.y; env.top[2] = t.z;
                env.bottom[0] = b.x; env.bottom[1] = b.y; env.bottom[2] = b.z;
            } else {
                throw ConfigError("unknown creator type name: " + et + " (envir_light)");
            }
        }
        int agg = ATRC_AGG_NATIVE, leaf = 5;
        if (auto g = p.find_child_group("aggregate")) {
            const std::string at = g->child_str("type");
            if (at == "bvh") {
                agg = ATRC_AGG_BVH;
                leaf = g->child_int_or("max_leaf_size", 5);
                if (leaf < 1) throw ConfigError("invalid max_leaf_size value");
            } else if (at != "native") {
                throw ConfigError("unknown creator type name: " + at + " (aggregate)");
            }
        }
        // pt_cuda-only key: builder of the device scene's mesh trees
        int builder = ATRC_BVH_SAH;
        if (p.find_child("bvh_builder")) {
            const std::string b = p.child_str("bvh_builder");
            if (b == "sah") builder = ATRC_BVH_SAH;
            else if (b == "ploc") builder = ATRC_BVH_PLOC;
            else if (b == "auto") builder = ATRC_BVH_AUTO;
            else throw ConfigError("invalid bvh_builder value: " + b + " (expect sah/ploc/auto)");
        }
        AtrcSceneDesc& s = out_.scene;
        s.abi_version = ATRC_ABI_VERSION;
        s.aggregate = agg;
        s.aggregate_max_leaf_size = leaf;
        s.bvh_builder = builder;
        s.meshes = out_.meshes.data(); s.mesh_count = uint32_t(out_.meshes.size());
        s.geometries = out_.geometries.data(); s.geometry_count = uint32_t(out_.geometries.size());
        s.entities = out_.entities.data(); s.entity_count = uint32_t(out_.entities.size());
        s.materials = out_.materials.data(); s.material_count = uint32_t(out_.materials.size());
        s.textures2d = out_.textures2d.data(); s.texture2d_count = uint32_t(out_.textures2d.size());
        s.textures3d = out_.textures3d.data(); s.texture3d_count = uint32_t(out_.textures3d.size());
        s.media = out_.media.data(); s.medium_count = uint32_t(out_.media.size());
        s.env = env;
    }

    // ------------------------------------------------------------- rendering
    RenderingEntry parse_rendering(const ConfigGroup& r) {
        // parse_rendering_settings (render_session.cpp:14-66)
        RenderingEntry e;
        AtrcRenderDesc& d = e.desc;
        std::memset(&d, 0, sizeof(d));
        d.width = r.child_int("width");
        d.height = r.child_int("height");
        if (d.width <= 0 || d.height <= 0) throw ConfigError("invalid film size");
        d.filter_type = ATRC_FILTER_BOX;
        d.filter_radius = 0.5f;
        if (auto f = r.find_child_group("film_filter")) {
            const std::string ft = f->child_str("type");
            if (ft == "box") {
                d.filter_type = ATRC_FILTER_BOX;
                d.filter_radius = f->child_real("radius");
            } else if (ft == "gaussian") {
                d.filter_type = ATRC_FILTER_GAUSSIAN;
                d.filter_radius = f->child_real("radius");
                d.filter_alpha = f->child_real("alpha");
            } else {
                throw ConfigError("unknown creator type name: " + ft + " (film_filter)");
            }
        }
        d.eps = 3e-4f;
        if (auto n = r.find_child("eps")) d.eps = n->as_value().as_real();
        parse_camera(r.child_group("camera"), float(d.width) / float(d.height), &d.camera);
        const ConfigGroup& rp = r.child_group("renderer");
        e.renderer_type = rp.child_str("type");
        if (e.renderer_type != "pt" && e.renderer_type != "pt_cuda" && e.renderer_type != "ao")
            throw ConfigError("renderer type '" + e.renderer_type + "' is not supported (pt, pt_cuda, ao)");
        d.spp = rp.child_int("spp");
        if (d.spp <= 0) throw ConfigError("invalid spp value");
        d.renderer = e.renderer_type == "ao" ? ATRC_RENDERER_AO : ATRC_RENDERER_PT;
        // AORendererCreator (renderer_creators.cpp:19-38)
        d.ao_sample_count = rp.child_int_or("ao_sample_count", 5);
        if (d.renderer == ATRC_RENDERER_AO && d.ao_sample_count <= 0)
            throw ConfigError("invalid ao_sample_count value");
        d.ao_max_distance = rp.child_real_or("max_occlusion_distance", 1);
        {
            const Vec3 lo = rp.child_spectrum_or("low_color", Vec3(0, 0, 0));
            const Vec3 hi = rp.child_spectrum_or("high_color", Vec3(1, 1, 1));
            const Vec3 bg = rp.child_spectrum_or("background_color", Vec3(0, 0, 0));
            const float l3[3] = {lo.x, lo.y, lo.z}, h3[3] = {hi.x, hi.y, hi.z}, b3[3] = {bg.x, bg.y, bg.z};
            for (int k = 0; k < 3; ++k) {
                d.ao_low[k] = l3[k];
                d.ao_high[k] = h3[k];
                d.ao_background[k] = b3[k];
            }
        }
        // PathTracingRendererCreator (renderer_creators.cpp:115-151)
        d.min_depth = rp.child_int_or("min_depth", 5);
        d.max_depth = rp.child_int_or("max_depth", 10);
        d.cont_prob = rp.child_real_or("cont_prob", 0.9f);
        d.use_mis = rp.child_int_or("use_mis", 1) != 0;
        d.specular_depth = rp.child_int_or("specular_depth", 20);
        d.task_grid_size = rp.child_int_or("task_grid_size", 32);
        if (d.task_grid_size <= 0) throw ConfigError("invalid task_grid_size value");
        // pt_cuda-only keys (defaults keep `pt` configs valid)
        d.seed = uint64_t(rp.child_int_or("seed", 42));
        d.path_pool = rp.child_int_or("path_pool", 0);
        d.sort_mode = rp.child_int_or("sort_mode", ATRC_SORT_AUTO);
        d.disney_fixed = rp.child_int_or("disney_fixed", 0) != 0;
        d.isect_mode = rp.child_int_or("watertight", 0) != 0 ? ATRC_ISECT_WATERTIGHT : ATRC_ISECT_FAST;
        if (d.sort_mode < ATRC_SORT_AUTO || d.sort_mode > ATRC_SORT_MATERIAL)
            throw ConfigError("invalid sort_mode value (-1 auto, 0 none, 1 material type, 2 material)");
        d.first_spp = 0;
        d.spp_count = 0;
        if (auto n = r.find_child("post_processors")) node_to_json(*n, e.post_processors_json);
        else e.post_processors_json = "[]";
        return e;
    }

    void parse_camera(const ConfigGroup& c, float aspect, AtrcCameraDesc* cam) {
        const std::string type = c.child_str("type");
        if (type == "reference") {
            std::string key;
            const ConfigGroup& g = resolve_reference(c, &key);
            parse_camera(g, aspect, cam);
            return;
        }
        Vec3 pos = c.child_vec3("pos"), dst = c.child_vec3("dst"), up = c.child_vec3("up");
        cam->pos[0] = pos.x; cam->pos[1] = pos.y; cam->pos[2] = pos.z;
        cam->dst[0] = dst.x; cam->dst[1] = dst.y; cam->dst[2] = dst.z;
        cam->up[0] = up.x; cam->up[1] = up.y; cam->up[2] = up.z;
        if (type == "thin_lens") {
            // PerspectiveCameraCreator (camera_creators.cpp:40-64)
            cam->fov = c.child_real("fov") / 180.0f * kPi;
            cam->lens_radius = c.child_real_or("lens_radius", 0);
            cam->focal_distance = c.child_real_or("focal_distance", 1);
        } else if (type == "pinhole") {
            // PinholeCameraCreator (camera_creators.cpp:13-36)
            const float width = c.child_real("width");
            const float height = width / aspect;
            const float dist = c.child_real("dist");
            cam->fov = 2 * std::atan(height / (2 * dist));
            cam->lens_radius = 0;
            cam->focal_distance = 1;
        } else {
            throw ConfigError("unknown creator type name: " + type + " (camera)");
        }
    }

private:
    static Affine affine_from(std::initializer_list<float> v) {
        float m[12];
        int i = 0;
        for (float x : v) m[i++] = x;
        Affine a;
        std::memcpy(a.m, m, sizeof(m));
        affine_identity(a.inv);
        return a;
    }
    static Affine mul3(const Affine& a, const Affine& b) {
        Affine r;
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 4; ++j) {
                double s = 0;
                for (int k = 0; k < 3; ++k) s += double(a.m[4 * i + k]) * b.m[4 * k + j];
                if (j == 3) s += a.m[4 * i + 3];
                r.m[4 * i + j] = float(s);
            }
        // inverse of a general affine 3x4
        const float* m = r.m;
        double A = double(m[5]) * m[10] - double(m[6]) * m[9];
        double B = -(double(m[4]) * m[10] - double(m[6]) * m[8]);
        double C = double(m[4]) * m[9] - double(m[5]) * m[8];
        double det = m[0] * A + m[1] * B + m[2] * C;
        if (det == 0.0) throw ConfigError("singular transform");
        double id = 1.0 / det;
        double inv3[9] = {A * id, -(double(m[1]) * m[10] - double(m[2]) * m[9]) * id, (double(m[1]) * m[6] - double(m[2]) * m[5]) * id,
                          B * id, (double(m[0]) * m[10] - double(m[2]) * m[8]) * id, -(double(m[0]) * m[6] - double(m[2]) * m[4]) * id,
                          C * id, -(double(m[0]) * m[9] - double(m[1]) * m[8]) * id, (double(m[0]) * m[5] - double(m[1]) * m[4]) * id};
        for (int row = 0; row < 3; ++row) {
            for (int c = 0; c < 3; ++c) r.inv[4 * row + c] = float(inv3[3 * row + c]);
            r.inv[4 * row + 3] = float(-(inv3[3 * row] * m[3] + inv3[3 * row + 1] * m[7] + inv3[3 * row + 2] * m[11]));
        }
        return r;
    }

    LoadedConfig& out_;
    const ConfigGroup& scene_root_;
    std::string scene_dir_, working_dir_;
    std::map<std::string, GeomRef> geom_refs_;
    std::map<std::string, int> mat_refs_, tex2d_refs_, tex3d_refs_, med_refs_;
    std::map<std::string, int> mesh_files_;
};

}  // namespace

std::unique_ptr<LoadedConfig> load_config_string(const std::string& json, const std::string& scene_dir) {
    auto out = std::make_unique<LoadedConfig>();
    out->root = parse_json_config(json);
    out->scene_dir = scene_dir.empty() ? std::filesystem::current_path().string() : scene_dir;
    const ConfigGroup& scene = out->root->child_group("scene");
    SceneBuilder b(*out, scene, out->scene_dir);
    b.build_scene();
    const ConfigNode& rendering = out->root->child("rendering");
    if (rendering.is_group()) {
        out->renderings.push_back(b.parse_rendering(rendering.as_group()));
    } else {
        const ConfigArray& a = rendering.as_array();
        for (size_t i = 0; i < a.size(); ++i) out->renderings.push_back(b.parse_rendering(a.at(i).as_group()));
    }
    return out;
}

std::unique_ptr<LoadedConfig> load_config_file(const std::string& path) {
    std::string text = read_text_file(path);
    std::string dir = std::filesystem::absolute(std::filesystem::path(path)).parent_path().string();
    return load_config_string(text, dir);
}

}  // namespace atrc
