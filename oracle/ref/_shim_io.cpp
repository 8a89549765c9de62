// agz-utils compatibility shim: image and mesh file I/O (see
// agz-utils/_shim.h).  Images come back with row 0 = the top row of the
// picture, as agz-utils' loaders return them; the reference's textures then
// read row y = v * height.
//   float RGB: Portable Float Map (.pfm, rows stored bottom-up) and Radiance
//              RGBE (.hdr, flat or new-style run-length scanlines, -Y H +X)
//   8-bit:     PNG (8-bit gray / gray+alpha / RGB / RGBA, not interlaced;
//              zlib inflate, the five scanline filters) and binary PPM (P6)
//   meshes:    OBJ (v / vt / vn, polygons as fans, negative indices) and STL
//              (binary, or ASCII "facet normal ... vertex ...")
#include <zlib.h>

#include <fstream>
#include <sstream>

#include "agz-utils/_shim.h"

namespace agz {
namespace {

using texture::texture2d_t;

std::vector<unsigned char> read_all(const std::string& fn) {
    std::ifstream f(fn, std::ios::binary);
    if (!f) throw std::runtime_error("failed to open file: " + fn);
    return std::vector<unsigned char>(std::istreambuf_iterator<char>(f), {});
}

std::string lower_ext(const std::string& fn) {
    std::string e = std::filesystem::path(fn).extension().string();
    for (auto& c : e) c = char(std::tolower(c));
    return e;
}

texture2d_t<math::color3f> load_pfm(const std::string& fn) {
    const auto d = read_all(fn);
    std::string hdr;
    size_t pos = 0;
    int fields = 0;
    std::string tok[4];
    // "PF" / "Pf", width, height, scale, each ended by whitespace
    while (fields < 4 && pos < d.size()) {
        while (pos < d.size() && std::isspace(d[pos])) ++pos;
        while (pos < d.size() && !std::isspace(d[pos])) tok[fields] += char(d[pos++]);
        ++fields;
    }
    ++pos;  // the single whitespace after the scale
    if (fields < 4 || (tok[0] != "PF" && tok[0] != "Pf")) throw std::runtime_error("not a PFM file: " + fn);
    const int ch = tok[0] == "PF" ? 3 : 1;
    const int w = std::stoi(tok[1]), h = std::stoi(tok[2]);
    const float scale = std::stof(tok[3]);
    if (w <= 0 || h <= 0 || pos + size_t(w) * h * ch * 4 > d.size()) throw std::runtime_error("bad PFM: " + fn);
    texture2d_t<math::color3f> img(h, w);
    const bool big_endian = scale > 0;
    for (int y = 0; y < h; ++y)
        for (int x = 0; x < w; ++x)
            for (int c = 0; c < 3; ++c) {
                const size_t at = pos + ((size_t(h - 1 - y) * w + x) * ch + (ch == 3 ? c : 0)) * 4;
                unsigned char b[4] = {d[at], d[at + 1], d[at + 2], d[at + 3]};
                if (big_endian) {
                    std::swap(b[0], b[3]);
                    std::swap(b[1], b[2]);
                }
                float v;
                std::memcpy(&v, b, 4);
                img(y, x)[c] = v;
            }
    return img;
}

texture2d_t<math::color3f> load_radiance(const std::string& fn) {
    const auto d = read_all(fn);
    size_t pos = 0;
    auto line = [&] {
        std::string s;
        while (pos < d.size() && d[pos] != '\n') s += char(d[pos++]);
        ++pos;
        return s;
    };
    if (line().rfind("#?", 0) != 0) throw std::runtime_error("not a Radiance file: " + fn);
    for (std::string s = line(); !s.empty(); s = line())
        if (s.rfind("FORMAT=", 0) == 0 && s != "FORMAT=32-bit_rle_rgbe")
            throw std::runtime_error("unsupported Radiance format: " + s);
    std::istringstream res(line());
    std::string a, b;
    int h = 0, w = 0;
    res >> a >> h >> b >> w;
    if (a != "-Y" || b != "+X" || w <= 0 || h <= 0) throw std::runtime_error("unsupported Radiance orientation: " + fn);
    texture2d_t<math::color3f> img(h, w);
    std::vector<unsigned char> scan(size_t(w) * 4);
    for (int y = 0; y < h; ++y) {
        if (pos + 4 > d.size()) throw std::runtime_error("truncated Radiance file: " + fn);
        const bool rle = w >= 8 && w < 32768 && d[pos] == 2 && d[pos + 1] == 2 && ((d[pos + 2] << 8) | d[pos + 3]) == w;
        if (rle) {
            pos += 4;
            for (int c = 0; c < 4; ++c)
                for (int x = 0; x < w;) {
                    if (pos >= d.size()) throw std::runtime_error("truncated Radiance file: " + fn);
                    int n = d[pos++];
                    if (n > 128) {
                        n -= 128;
                        const unsigned char v = d[pos++];
                        for (int k = 0; k < n && x < w; ++k) scan[size_t(x++) * 4 + c] = v;
                    } else {
                        for (int k = 0; k < n && x < w; ++k) scan[size_t(x++) * 4 + c] = d[pos++];
                    }
                }
        } else {
            if (pos + size_t(w) * 4 > d.size()) throw std::runtime_error("truncated Radiance file: " + fn);
            std::memcpy(scan.data(), &d[pos], size_t(w) * 4);
            pos += size_t(w) * 4;
        }
        for (int x = 0; x < w; ++x) {
            const unsigned char* p = &scan[size_t(x) * 4];
            const float f = p[3] ? std::ldexp(1.0f, int(p[3]) - (128 + 8)) : 0.0f;
            img(y, x) = math::color3f(p[0] * f, p[1] * f, p[2] * f);
        }
    }
    return img;
}

// 8-bit PNG -> channels-per-pixel samples, row 0 = top.
std::vector<unsigned char> decode_png(const std::string& fn, int* w, int* h, int* channels) {
    const auto d = read_all(fn);
    static const unsigned char sig[8] = {137, 80, 78, 71, 13, 10, 26, 10};
    if (d.size() < 8 || std::memcmp(d.data(), sig, 8) != 0) throw std::runtime_error("not a PNG file: " + fn);
    auto be32 = [&](size_t at) { return (uint32_t(d[at]) << 24) | (uint32_t(d[at + 1]) << 16) | (uint32_t(d[at + 2]) << 8) | d[at + 3]; };
    size_t pos = 8;
    int depth = 0, ctype = -1, interlace = 0;
    std::vector<unsigned char> idat;
    while (pos + 12 <= d.size()) {
        const uint32_t len = be32(pos);
        const std::string type(reinterpret_cast<const char*>(&d[pos + 4]), 4);
        if (pos + 12 + len > d.size()) throw std::runtime_error("truncated PNG: " + fn);
        const unsigned char* body = &d[pos + 8];
        if (type == "IHDR") {
            *w = int(be32(pos + 8));
            *h = int(be32(pos + 12));
            depth = body[8];
            ctype = body[9];
            interlace = body[12];
        } else if (type == "IDAT") {
            idat.insert(idat.end(), body, body + len);
        } else if (type == "IEND") {
            break;
        }
        pos += 12 + len;
    }
    const int ch = ctype == 0 ? 1 : ctype == 4 ? 2 : ctype == 2 ? 3 : ctype == 6 ? 4 : 0;
    if (depth != 8 || ch == 0 || interlace != 0 || *w <= 0 || *h <= 0)
        throw std::runtime_error("unsupported PNG (8-bit gray / RGB (+ alpha), not interlaced): " + fn);
    *channels = ch;
    const size_t stride = size_t(*w) * ch;
    std::vector<unsigned char> raw((stride + 1) * *h);
    uLongf raw_len = uLongf(raw.size());
    if (uncompress(raw.data(), &raw_len, idat.data(), uLong(idat.size())) != Z_OK || raw_len != raw.size())
        throw std::runtime_error("corrupt PNG data: " + fn);
    std::vector<unsigned char> out(stride * *h);
    for (int y = 0; y < *h; ++y) {
        const unsigned char f = raw[(stride + 1) * y];
        const unsigned char* src = &raw[(stride + 1) * y + 1];
        unsigned char* dst = &out[stride * y];
        const unsigned char* up = y > 0 ? &out[stride * (y - 1)] : nullptr;
        for (size_t i = 0; i < stride; ++i) {
            const int a = i >= size_t(ch) ? dst[i - ch] : 0, b = up ? up[i] : 0, c = (up && i >= size_t(ch)) ? up[i - ch] : 0;
            int pred = 0;
            switch (f) {
            case 0: pred = 0; break;
            case 1: pred = a; break;
            case 2: pred = b; break;
            case 3: pred = (a + b) / 2; break;
            case 4: {  // Paeth
                const int p = a + b - c, pa = std::abs(p - a), pb = std::abs(p - b), pc = std::abs(p - c);
                pred = (pa <= pb && pa <= pc) ? a : (pb <= pc ? b : c);
                break;
            }
            default: throw std::runtime_error("bad PNG filter: " + fn);
            }
            dst[i] = (unsigned char)(src[i] + pred);
        }
    }
    return out;
}

std::vector<unsigned char> decode_ppm(const std::string& fn, int* w, int* h) {
    const auto d = read_all(fn);
    size_t pos = 0;
    auto token = [&] {
        std::string t;
        while (pos < d.size()) {
            if (d[pos] == '#') {
                while (pos < d.size() && d[pos] != '\n') ++pos;
            } else if (std::isspace(d[pos])) {
                ++pos;
            } else {
                break;
            }
        }
        while (pos < d.size() && !std::isspace(d[pos])) t += char(d[pos++]);
        return t;
    };
    if (token() != "P6") throw std::runtime_error("not a binary PPM: " + fn);
    *w = std::stoi(token());
    *h = std::stoi(token());
    if (std::stoi(token()) != 255) throw std::runtime_error("PPM max value must be 255: " + fn);
    ++pos;
    if (pos + size_t(*w) * *h * 3 > d.size()) throw std::runtime_error("truncated PPM: " + fn);
    return std::vector<unsigned char>(d.begin() + long(pos), d.begin() + long(pos + size_t(*w) * *h * 3));
}

}  // namespace

namespace img {

texture2d_t<math::color3f> load_rgb_from_hdr_file(const std::string& filename) {
    return lower_ext(filename) == ".pfm" ? load_pfm(filename) : load_radiance(filename);
}

texture2d_t<math::color3b> load_rgb_from_file(const std::string& filename) {
    int w = 0, h = 0, ch = 3;
    const auto px = lower_ext(filename) == ".ppm" ? decode_ppm(filename, &w, &h) : decode_png(filename, &w, &h, &ch);
    texture2d_t<math::color3b> img(h, w);
    for (int y = 0; y < h; ++y)
        for (int x = 0; x < w; ++x) {
            const unsigned char* p = &px[(size_t(y) * w + x) * ch];
            img(y, x) = ch >= 3 ? math::color3b(p[0], p[1], p[2]) : math::color3b(p[0], p[0], p[0]);
        }
    return img;
}

texture2d_t<uint8_t> load_gray_from_file(const std::string& filename) {
    const auto rgb = load_rgb_from_file(filename);
    texture2d_t<uint8_t> img(rgb.height(), rgb.width());
    for (int y = 0; y < rgb.height(); ++y)
        for (int x = 0; x < rgb.width(); ++x) {
            const auto& c = rgb(y, x);
            img(y, x) = uint8_t((int(c.r) + int(c.g) + int(c.b)) / 3);
        }
    return img;
}

void save_rgb_to_png_file(const std::string& filename, const texture2d_t<math::color3b>&) {
    throw std::runtime_error("the agz-utils shim does not write images (" + filename + ")");
}
void save_rgb_to_jpg_file(const std::string& filename, const texture2d_t<math::color3b>&) {
    throw std::runtime_error("the agz-utils shim does not write images (" + filename + ")");
}
void save_rgb_to_hdr_file(const std::string& filename, const texture2d_t<math::color3f>&) {
    throw std::runtime_error("the agz-utils shim does not write images (" + filename + ")");
}

}  // namespace img

namespace mesh {

namespace {

math::vec3 face_normal(const math::vec3& a, const math::vec3& b, const math::vec3& c) {
    return cross(b - a, c - a).normalize();
}

std::vector<triangle_t> load_obj(const std::string& fn) {
    std::ifstream f(fn);
    if (!f) throw std::runtime_error("failed to open mesh: " + fn);
    std::vector<math::vec3> pos, nor;
    std::vector<math::vec2> uv;
    std::vector<triangle_t> out;
    struct Ref { int p, t, n; };
    auto fix = [](int i, size_t n) { return i < 0 ? int(n) + i : i - 1; };
    for (std::string line; std::getline(f, line);) {
        std::istringstream ls(line);
        std::string k;
        ls >> k;
        if (k == "v") { math::vec3 v; ls >> v.x >> v.y >> v.z; pos.push_back(v); }
        else if (k == "vt") { math::vec2 t; ls >> t.x >> t.y; uv.push_back(t); }
        else if (k == "vn") { math::vec3 v; ls >> v.x >> v.y >> v.z; nor.push_back(v); }
        else if (k == "f") {
            std::vector<Ref> refs;
            for (std::string w; ls >> w;) {
                Ref r{0, 0, 0};
                std::string part[3];
                int idx = 0;
                for (char ch : w) {
                    if (ch == '/') ++idx;
                    else if (idx < 3) part[idx] += ch;
                }
                r.p = fix(std::stoi(part[0]), pos.size());
                r.t = part[1].empty() ? -1 : fix(std::stoi(part[1]), uv.size());
                r.n = part[2].empty() ? -1 : fix(std::stoi(part[2]), nor.size());
                refs.push_back(r);
            }
            for (size_t i = 1; i + 1 < refs.size(); ++i) {
                const Ref tri[3] = {refs[0], refs[i], refs[i + 1]};
                triangle_t t;
                const math::vec3 fnrm = face_normal(pos.at(tri[0].p), pos.at(tri[1].p), pos.at(tri[2].p));
                for (int k2 = 0; k2 < 3; ++k2) {
                    t.vertices[k2].position = pos.at(tri[k2].p);
                    t.vertices[k2].normal = tri[k2].n >= 0 ? nor.at(tri[k2].n) : fnrm;
                    t.vertices[k2].tex_coord = tri[k2].t >= 0 ? uv.at(tri[k2].t) : math::vec2();
                }
                out.push_back(t);
            }
        }
    }
    return out;
}

std::vector<triangle_t> load_stl(const std::string& fn) {
    const auto d = read_all(fn);
    std::vector<triangle_t> out;
    if (d.size() >= 84) {
        uint32_t n;
        std::memcpy(&n, &d[80], 4);
        if (d.size() == 84 + size_t(n) * 50) {
            for (uint32_t i = 0; i < n; ++i) {
                float v[12];
                std::memcpy(v, &d[84 + size_t(i) * 50], 48);
                triangle_t t;
                for (int k = 0; k < 3; ++k) {
                    t.vertices[k].position = math::vec3(v[3 + 3 * k], v[4 + 3 * k], v[5 + 3 * k]);
                    t.vertices[k].normal = math::vec3(v[0], v[1], v[2]);
                }
                out.push_back(t);
            }
            return out;
        }
    }
    std::istringstream s(std::string(d.begin(), d.end()));
    math::vec3 n;
    std::vector<math::vec3> vs;
    for (std::string w; s >> w;) {
        if (w == "normal") s >> n.x >> n.y >> n.z;
        else if (w == "vertex") {
            math::vec3 p;
            s >> p.x >> p.y >> p.z;
            vs.push_back(p);
            if (vs.size() == 3) {
                triangle_t t;
                for (int k = 0; k < 3; ++k) { t.vertices[k].position = vs[k]; t.vertices[k].normal = n; }
                out.push_back(t);
                vs.clear();
            }
        }
    }
    return out;
}

}  // namespace

std::vector<triangle_t> load_from_file(const std::string& filename) {
    const std::string e = lower_ext(filename);
    if (e == ".obj") return load_obj(filename);
    if (e == ".stl") return load_stl(filename);
    throw std::runtime_error("unsupported mesh format: " + filename);
}

}  // namespace mesh
}  // namespace agz
