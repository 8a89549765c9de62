// Host file formats: float images (.pfm, Radiance .hdr), meshes (.bm, .obj)
// and image writers for the output post processors.
//
// The reference reads these through agz-utils (img::load_rgb_from_hdr_file,
// mesh::load_from_file), which is absent from its checkout; the formats are
// implemented here from their public specifications.  `.bm` follows
// src/factory/src/utility/bin_mesh.cpp:7-27 (size_t count, then per triangle
// three {position[3], normal[3], tex_coord[2]} float vertices).
#include <zlib.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <iterator>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "scene_loader.h"

namespace atrc {

namespace {

bool has_ext(const std::string& fn, const char* ext) {
    size_t n = std::strlen(ext);
    if (fn.size() < n) return false;
    for (size_t i = 0; i < n; ++i)
        if (std::tolower((unsigned char)fn[fn.size() - n + i]) != ext[i]) return false;
    return true;
}

// Portable float map: "PF\n<w> <h>\n<scale>\n" then rows bottom-to-top.
std::vector<float> load_pfm(const std::string& fn, int* w, int* h) {
    std::ifstream f(fn, std::ios::binary);
    if (!f) throw ConfigError("failed to open image: " + fn);
    std::string magic;
    f >> magic;
    int ch;
    if (magic == "PF") ch = 3;
    else if (magic == "Pf") ch = 1;
    else throw ConfigError("not a PFM file: " + fn);
    double scale;
    f >> *w >> *h >> scale;
    f.get();
    if (!f || *w <= 0 || *h <= 0) throw ConfigError("bad PFM header: " + fn);
    const bool little = scale < 0;
    std::vector<float> raw(size_t(*w) * *h * ch);
    f.read(reinterpret_cast<char*>(raw.data()), raw.size() * sizeof(float));
    if (!f) throw ConfigError("truncated PFM: " + fn);
    if (!little) {
        for (auto& v : raw) {
            uint32_t u;
            std::memcpy(&u, &v, 4);
            u = __builtin_bswap32(u);
            std::memcpy(&v, &u, 4);
        }
    }
    std::vector<float> out(size_t(*w) * *h * 3);
    for (int y = 0; y < *h; ++y) {
        const int src_row = *h - 1 - y;  // PFM stores the bottom row first
        for (int x = 0; x < *w; ++x)
            for (int c = 0; c < 3; ++c)
                out[(size_t(y) * *w + x) * 3 + c] = raw[(size_t(src_row) * *w + x) * ch + (ch == 3 ? c : 0)];
    }
    return out;
}

// Radiance RGBE (.hdr), flat or new-style run-length encoded scanlines.
std::vector<float> load_rgbe(const std::string& fn, int* w, int* h) {
    std::ifstream f(fn, std::ios::binary);
    if (!f) throw ConfigError("failed to open image: " + fn);
    std::string line;
    std::getline(f, line);
    if (line.rfind("#?", 0) != 0) throw ConfigError("not a Radiance HDR file: " + fn);
    while (std::getline(f, line) && !line.empty()) {
        if (line.rfind("FORMAT=", 0) == 0 && line != "FORMAT=32-bit_rle_rgbe")
            throw ConfigError("unsupported HDR format: " + line);
    }
    std::getline(f, line);
    char ya[4], xa[4];
    if (std::sscanf(line.c_str(), "%3s %d %3s %d", ya, h, xa, w) != 4 || std::string(ya) != "-Y" || std::string(xa) != "+X")
        throw ConfigError("unsupported HDR orientation: " + line);
    if (*w <= 0 || *h <= 0 || *w > 65536 || *h > 65536) throw ConfigError("bad HDR size: " + line);
    std::vector<float> out(size_t(*w) * *h * 3);
    std::vector<uint8_t> scan(size_t(*w) * 4);
    for (int y = 0; y < *h; ++y) {
        uint8_t hdr[4];
        f.read(reinterpret_cast<char*>(hdr), 4);
        if (!f) throw ConfigError("truncated HDR: " + fn);
        if (*w >= 8 && *w < 32768 && hdr[0] == 2 && hdr[1] == 2 && ((hdr[2] << 8) | hdr[3]) == *w) {
            for (int c = 0; c < 4; ++c) {
                int x = 0;
                while (x < *w) {
                    int cnt = f.get();
                    if (cnt == EOF) throw ConfigError("truncated HDR: " + fn);
                    if (cnt == 0 || x + (cnt > 128 ? cnt - 128 : cnt) > *w)
                        throw ConfigError("bad HDR run length: " + fn);
                    if (cnt > 128) {
                        cnt -= 128;
                        const int v = f.get();
                        if (v == EOF) throw ConfigError("truncated HDR: " + fn);
                        for (int k = 0; k < cnt; ++k) scan[size_t(x++) * 4 + c] = uint8_t(v);
                    } else {
                        for (int k = 0; k < cnt; ++k) {
                            const int v = f.get();
                            if (v == EOF) throw ConfigError("truncated HDR: " + fn);
                            scan[size_t(x++) * 4 + c] = uint8_t(v);
                        }
                    }
                }
            }
        } else {
            std::memcpy(scan.data(), hdr, 4);
            f.read(reinterpret_cast<char*>(scan.data() + 4), (size_t(*w) - 1) * 4);
            if (!f) throw ConfigError("truncated HDR: " + fn);
        }
        for (int x = 0; x < *w; ++x) {
            const uint8_t* p = &scan[size_t(x) * 4];
            float s = p[3] ? std::ldexp(1.0f, int(p[3]) - 136) : 0.0f;
            for (int c = 0; c < 3; ++c) out[(size_t(y) * *w + x) * 3 + c] = p[c] * s;
        }
    }
    return out;
}

uint32_t crc32_table[256];
bool crc_init = false;

uint32_t crc32(const uint8_t* d, size_t n, uint32_t c = 0xFFFFFFFFu) {
    if (!crc_init) {
        for (uint32_t i = 0; i < 256; ++i) {
            uint32_t v = i;
            for (int k = 0; k < 8; ++k) v = (v & 1) ? 0xEDB88320u ^ (v >> 1) : v >> 1;
            crc32_table[i] = v;
        }
        crc_init = true;
    }
    for (size_t i = 0; i < n; ++i) c = crc32_table[(c ^ d[i]) & 0xFF] ^ (c >> 8);
    return c;
}

void put_be32(std::vector<uint8_t>& v, uint32_t x) {
    v.push_back(uint8_t(x >> 24)); v.push_back(uint8_t(x >> 16));
    v.push_back(uint8_t(x >> 8)); v.push_back(uint8_t(x));
}

void png_chunk(std::ofstream& f, const char* type, const std::vector<uint8_t>& data) {
    std::vector<uint8_t> buf;
    put_be32(buf, uint32_t(data.size()));
    buf.insert(buf.end(), type, type + 4);
    buf.insert(buf.end(), data.begin(), data.end());
    uint32_t c = crc32(buf.data() + 4, buf.size() - 4) ^ 0xFFFFFFFFu;
    put_be32(buf, c);
    f.write(reinterpret_cast<const char*>(buf.data()), buf.size());
}

}  // namespace

// 8-bit PNG (gray, gray+alpha, RGB, RGBA; not interlaced) -> RGB floats
// byte / 255, row 0 = top.  The IDAT stream is inflated with zlib and the
// five scanline filters of the PNG specification are undone.
std::vector<float> load_png(const std::string& fn, int* w, int* h) {
    std::ifstream f(fn, std::ios::binary);
    if (!f) throw ConfigError("failed to open file: " + fn);
    std::vector<uint8_t> data((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
    static const uint8_t sig[8] = {137, 80, 78, 71, 13, 10, 26, 10};
    if (data.size() < 8 || std::memcmp(data.data(), sig, 8) != 0) throw ConfigError("not a PNG file: " + fn);
    auto be32 = [&](size_t o) {
        return (uint32_t(data[o]) << 24) | (uint32_t(data[o + 1]) << 16) | (uint32_t(data[o + 2]) << 8) | data[o + 3];
    };
    uint32_t W = 0, H = 0;
    int depth = 0, ctype = -1, interlace = 0;
    std::vector<uint8_t> idat;
    for (size_t pos = 8; pos + 12 <= data.size();) {
        const uint32_t n = be32(pos);
        if (pos + 12 + n > data.size()) throw ConfigError("truncated PNG chunk: " + fn);
        const std::string kind(reinterpret_cast<const char*>(&data[pos + 4]), 4);
        const uint8_t* body = &data[pos + 8];
        if (kind == "IHDR" && n >= 13) {
            W = be32(pos + 8);
            H = be32(pos + 12);
            depth = body[8];
            ctype = body[9];
            interlace = body[12];
        } else if (kind == "IDAT") {
            idat.insert(idat.end(), body, body + n);
        } else if (kind == "IEND") {
            break;
        }
        pos += 12 + n;
    }
    const int ch = ctype == 0 ? 1 : ctype == 4 ? 2 : ctype == 2 ? 3 : ctype == 6 ? 4 : 0;
    if (depth != 8 || ch == 0 || interlace != 0 || W == 0 || H == 0 || W > (1u << 16) || H > (1u << 16))
        throw ConfigError("unsupported PNG (8-bit gray / RGB / RGBA, not interlaced): " + fn);
    const size_t stride = size_t(W) * ch;
    std::vector<uint8_t> raw(size_t(H) * (stride + 1));
    uLongf got = uLongf(raw.size());
    if (uncompress(raw.data(), &got, idat.data(), uLong(idat.size())) != Z_OK || got != raw.size())
        throw ConfigError("corrupt PNG data: " + fn);
    std::vector<uint8_t> img(size_t(H) * stride);
    for (uint32_t y = 0; y < H; ++y) {
        const uint8_t ft = raw[y * (stride + 1)];
        const uint8_t* src = &raw[y * (stride + 1) + 1];
        uint8_t* dst = &img[y * stride];
        const uint8_t* up = y ? &img[(y - 1) * stride] : nullptr;
        for (size_t i = 0; i < stride; ++i) {
            const int a = i >= size_t(ch) ? dst[i - ch] : 0, b = up ? up[i] : 0, c = (up && i >= size_t(ch)) ? up[i - ch] : 0;
            int v = src[i];
            if (ft == 1) v += a;
            else if (ft == 2) v += b;
            else if (ft == 3) v += (a + b) / 2;
            else if (ft == 4) {
                const int pp = a + b - c, pa = std::abs(pp - a), pb = std::abs(pp - b), pc = std::abs(pp - c);
                v += (pa <= pb && pa <= pc) ? a : (pb <= pc ? b : c);
            } else if (ft != 0) {
                throw ConfigError("corrupt PNG filter: " + fn);
            }
            dst[i] = uint8_t(v);
        }
    }
    *w = int(W);
    *h = int(H);
    std::vector<float> out(size_t(W) * H * 3);
    for (size_t k = 0; k < size_t(W) * H; ++k)
        for (int c = 0; c < 3; ++c) out[k * 3 + c] = float(img[k * ch + (ch >= 3 ? c : 0)]) / 255.0f;
    return out;
}

// Binary PPM (P6, maxval 255) -> RGB floats byte / 255, row 0 = top.
std::vector<float> load_ppm(const std::string& fn, int* w, int* h) {
    std::ifstream f(fn, std::ios::binary);
    if (!f) throw ConfigError("failed to open file: " + fn);
    std::string magic;
    int W = 0, H = 0, maxval = 0;
    f >> magic >> W >> H >> maxval;
    f.get();
    if (magic != "P6" || W <= 0 || H <= 0 || maxval != 255) throw ConfigError("unsupported PPM (P6, 8-bit): " + fn);
    std::vector<uint8_t> bytes(size_t(W) * H * 3);
    f.read(reinterpret_cast<char*>(bytes.data()), std::streamsize(bytes.size()));
    if (!f) throw ConfigError("truncated PPM: " + fn);
    *w = W;
    *h = H;
    std::vector<float> out(bytes.size());
    for (size_t k = 0; k < bytes.size(); ++k) out[k] = float(bytes[k]) / 255.0f;
    return out;
}

std::vector<float> load_rgb_image(const std::string& fn, int* w, int* h) {
    if (has_ext(fn, ".pfm")) return load_pfm(fn, w, h);
    if (has_ext(fn, ".hdr")) return load_rgbe(fn, w, h);
    if (has_ext(fn, ".png")) return load_png(fn, w, h);
    if (has_ext(fn, ".ppm")) return load_ppm(fn, w, h);
    throw ConfigError("unsupported image format (pt_cuda reads .pfm, .hdr, .png and .ppm): " + fn);
}

// STL triangle soup, binary (80-byte header, uint32 count, 50 bytes per
// facet: normal, three vertices, attribute word) or ASCII (solid / facet
// normal / outer loop / vertex x3).  A file is binary when its size is
// 84 + 50 * count, whatever its first bytes say.  Vertex normals are the
// facet normal, or the winding normal where the file's is zero; uv = 0.
static std::vector<float> load_stl(const std::string& fn) {
    std::ifstream f(fn, std::ios::binary);
    if (!f) throw ConfigError("failed to open file: " + fn);
    std::vector<char> data((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
    std::vector<float> out;
    auto emit = [&](Vec3 n, const Vec3* v) {
        const Vec3 w = cross(v[1] - v[0], v[2] - v[0]);
        if (!(dot(n, n) > 0) || !std::isfinite(n.x + n.y + n.z)) n = dot(w, w) > 0 ? normalize(w) : Vec3(0, 0, 1);
        else n = normalize(n);
        for (int k = 0; k < 3; ++k) out.insert(out.end(), {v[k].x, v[k].y, v[k].z, n.x, n.y, n.z, 0.0f, 0.0f});
    };
    uint32_t count = 0;
    if (data.size() >= 84) std::memcpy(&count, data.data() + 80, 4);
    if (data.size() >= 84 && data.size() == 84 + size_t(count) * 50) {
        out.reserve(size_t(count) * 24);
        for (uint32_t t = 0; t < count; ++t) {
            float r[12];
            std::memcpy(r, data.data() + 84 + size_t(t) * 50, sizeof(r));
            const Vec3 v[3] = {Vec3(r[3], r[4], r[5]), Vec3(r[6], r[7], r[8]), Vec3(r[9], r[10], r[11])};
            emit(Vec3(r[0], r[1], r[2]), v);
        }
        return out;
    }
    std::istringstream ss(std::string(data.begin(), data.end()));
    std::string tok;
    if (!(ss >> tok) || tok != "solid") throw ConfigError("not an STL file: " + fn);
    Vec3 n, v[3];
    int nv = 0;
    while (ss >> tok) {
        if (tok == "facet") {
            std::string kw;
            ss >> kw >> n.x >> n.y >> n.z;
            if (!ss || kw != "normal") throw ConfigError("bad STL facet: " + fn);
            nv = 0;
        } else if (tok == "vertex") {
            if (nv >= 3) throw ConfigError("STL facet with more than three vertices: " + fn);
            ss >> v[nv].x >> v[nv].y >> v[nv].z;
            if (!ss) throw ConfigError("bad STL vertex: " + fn);
            ++nv;
        } else if (tok == "endfacet") {
            if (nv != 3) throw ConfigError("STL facet without three vertices: " + fn);
            emit(n, v);
        }
    }
    return out;
}

std::vector<float> load_triangle_mesh(const std::string& fn) {
    if (has_ext(fn, ".bm")) {
        std::ifstream f(fn, std::ios::binary);
        if (!f) throw ConfigError("failed to open file: " + fn);
        uint64_t count = 0;
        f.read(reinterpret_cast<char*>(&count), sizeof(count));
        if (!f) throw ConfigError("failed to load triangle count from " + fn);
        std::vector<float> v(size_t(count) * 24);
        f.read(reinterpret_cast<char*>(v.data()), v.size() * sizeof(float));
        if (!f) throw ConfigError("failed to load triangle data from " + fn);
        return v;
    }
    if (has_ext(fn, ".obj")) {
        std::ifstream f(fn);
        if (!f) throw ConfigError("failed to open file: " + fn);
        std::vector<float> pos, nor, uv, out;
        std::string line;
        auto fix = [](int i, size_t n) -> long { return i > 0 ? long(i) - 1 : long(n) + i; };
        while (std::getline(f, line)) {
            std::istringstream ss(line);
            std::string tag;
            ss >> tag;
            if (tag == "v") { float x, y, z; ss >> x >> y >> z; pos.insert(pos.end(), {x, y, z}); }
            else if (tag == "vn") { float x, y, z; ss >> x >> y >> z; nor.insert(nor.end(), {x, y, z}); }
            else if (tag == "vt") { float x, y; ss >> x >> y; uv.insert(uv.end(), {x, y}); }
            else if (tag == "f") {
                struct Idx { long p = -1, t = -1, n = -1; };
                std::vector<Idx> poly;
                std::string tok;
                while (ss >> tok) {
                    Idx id;
                    int a = 0, b = 0, c = 0;
                    if (std::sscanf(tok.c_str(), "%d/%d/%d", &a, &b, &c) == 3) { id.p = fix(a, pos.size() / 3); id.t = fix(b, uv.size() / 2); id.n = fix(c, nor.size() / 3); }
                    else if (std::sscanf(tok.c_str(), "%d//%d", &a, &c) == 2) { id.p = fix(a, pos.size() / 3); id.n = fix(c, nor.size() / 3); }
                    else if (std::sscanf(tok.c_str(), "%d/%d", &a, &b) == 2) { id.p = fix(a, pos.size() / 3); id.t = fix(b, uv.size() / 2); }
                    else if (std::sscanf(tok.c_str(), "%d", &a) == 1) { id.p = fix(a, pos.size() / 3); }
                    else throw ConfigError("bad OBJ face: " + line);
                    poly.push_back(id);
                }
                for (size_t k = 1; k + 1 < poly.size(); ++k) {
                    const Idx tri[3] = {poly[0], poly[k], poly[k + 1]};
                    Vec3 P[3];
                    for (int i = 0; i < 3; ++i) {
                        if (tri[i].p < 0 || size_t(tri[i].p) >= pos.size() / 3) throw ConfigError("OBJ index out of range");
                        P[i] = Vec3(pos[tri[i].p * 3], pos[tri[i].p * 3 + 1], pos[tri[i].p * 3 + 2]);
                    }
                    Vec3 fn_ = normalize(cross(P[1] - P[0], P[2] - P[0]));
                    for (int i = 0; i < 3; ++i) {
                        Vec3 n = fn_;
                        if (tri[i].n >= 0 && size_t(tri[i].n) < nor.size() / 3)
                            n = Vec3(nor[tri[i].n * 3], nor[tri[i].n * 3 + 1], nor[tri[i].n * 3 + 2]);
                        float u = 0, v = 0;
                        if (tri[i].t >= 0 && size_t(tri[i].t) < uv.size() / 2) { u = uv[tri[i].t * 2]; v = uv[tri[i].t * 2 + 1]; }
                        out.insert(out.end(), {P[i].x, P[i].y, P[i].z, n.x, n.y, n.z, u, v});
                    }
                }
            }
        }
        return out;
    }
    if (has_ext(fn, ".stl")) return load_stl(fn);
    throw ConfigError("unsupported mesh format (pt_cuda reads .bm, .obj and .stl): " + fn);
}

void save_pfm(const std::string& fn, const float* rgb, int w, int h) {
    // PFM stores the bottom row first, which is film row 0
    std::ofstream f(fn, std::ios::binary);
    if (!f) throw ConfigError("failed to open output: " + fn);
    f << "PF\n" << w << " " << h << "\n-1.0\n";
    for (int y = 0; y < h; ++y) f.write(reinterpret_cast<const char*>(rgb + size_t(y) * w * 3), size_t(w) * 3 * sizeof(float));
}

void save_png8(const std::string& fn, const float* rgb, int w, int h, float gamma) {
    // Texels map as uint8(clamp(c^gamma, 0, 1) * 255), rows written top to
    // bottom (save_to_img.cpp:36-49 flips the film vertically).
    std::vector<uint8_t> bytes(size_t(w) * h * 3);
    for (int y = 0; y < h; ++y) {
        const int src = h - 1 - y;
        for (int x = 0; x < w * 3; ++x) {
            float v = std::pow(rgb[size_t(src) * w * 3 + x], gamma);
            v = std::fmin(std::fmax(v, 0.0f), 1.0f);
            if (!(v == v)) v = 0;
            bytes[size_t(y) * w * 3 + x] = uint8_t(v * 255.0f);
        }
    }
    write_png_bytes(fn, bytes.data(), w, h);
}

void write_png_bytes(const std::string& fn, const uint8_t* rgb8, int w, int h) {
    // 8-bit RGB PNG with stored (uncompressed) deflate blocks, rows as given
    std::vector<uint8_t> raw;
    raw.reserve(size_t(h) * (size_t(w) * 3 + 1));
    for (int y = 0; y < h; ++y) {
        raw.push_back(0);
        raw.insert(raw.end(), rgb8 + size_t(y) * w * 3, rgb8 + size_t(y + 1) * w * 3);
    }
    std::vector<uint8_t> z = {0x78, 0x01};
    size_t off = 0;
    while (off < raw.size() || raw.empty()) {
        size_t n = std::min<size_t>(65535, raw.size() - off);
        bool last = off + n >= raw.size();
        z.push_back(last ? 1 : 0);
        z.push_back(uint8_t(n)); z.push_back(uint8_t(n >> 8));
        z.push_back(uint8_t(~n)); z.push_back(uint8_t((~n) >> 8));
        z.insert(z.end(), raw.begin() + off, raw.begin() + off + n);
        off += n;
        if (raw.empty()) break;
    }
    uint32_t a = 1, b = 0;
    for (uint8_t c : raw) { a = (a + c) % 65521; b = (b + a) % 65521; }
    put_be32(z, (b << 16) | a);
    std::ofstream f(fn, std::ios::binary);
    if (!f) throw ConfigError("failed to open output: " + fn);
    const uint8_t sig[8] = {137, 80, 78, 71, 13, 10, 26, 10};
    f.write(reinterpret_cast<const char*>(sig), 8);
    std::vector<uint8_t> ihdr;
    put_be32(ihdr, uint32_t(w));
    put_be32(ihdr, uint32_t(h));
    ihdr.insert(ihdr.end(), {8, 2, 0, 0, 0});
    png_chunk(f, "IHDR", ihdr);
    png_chunk(f, "IDAT", z);
    png_chunk(f, "IEND", {});
}

// One component of a scanline in the new-style run-length encoding: runs of
// 4 or more equal bytes as (128 + length, byte), up to 127 long; everything
// else as literals (length, bytes...), up to 128 long.
static void rle_component(std::ofstream& f, const uint8_t* v, int n) {
    int x = 0;
    while (x < n) {
        int run = 1;
        while (x + run < n && run < 127 && v[x + run] == v[x]) ++run;
        if (run >= 4) {
            const uint8_t rec[2] = {uint8_t(128 + run), v[x]};
            f.write(reinterpret_cast<const char*>(rec), 2);
            x += run;
            continue;
        }
        // literals up to the next run of 4 (or 128 bytes)
        int lit = 0;
        while (x + lit < n && lit < 128) {
            int r = 1;
            while (x + lit + r < n && r < 4 && v[x + lit + r] == v[x + lit]) ++r;
            if (r >= 4) break;
            ++lit;
        }
        const uint8_t cnt = uint8_t(lit);
        f.write(reinterpret_cast<const char*>(&cnt), 1);
        f.write(reinterpret_cast<const char*>(v + x), lit);
        x += lit;
    }
}

void save_hdr_rgbe(const std::string& fn, const float* rgb, int w, int h) {
    std::ofstream f(fn, std::ios::binary);
    if (!f) throw ConfigError("failed to open output: " + fn);
    f << "#?RADIANCE\nFORMAT=32-bit_rle_rgbe\n\n-Y " << h << " +X " << w << "\n";
    // scanlines of 8 to 32767 pixels are run-length encoded, as Radiance
    // writes them: a flat scanline whose first pixel reads (2, 2, w >> 8,
    // w & 255) would otherwise be taken for an encoded one
    const bool rle = w >= 8 && w < 32768;
    std::vector<uint8_t> line(static_cast<size_t>(w) * 4), comp(static_cast<size_t>(w));
    for (int y = 0; y < h; ++y) {
        const size_t row = size_t(h - 1 - y) * w;  // top row first
        for (int x = 0; x < w; ++x) {
            const float* c = rgb + 3 * (row + x);
            const float r = std::fmax(c[0], 0.f), g = std::fmax(c[1], 0.f), b = std::fmax(c[2], 0.f);
            const float m = std::fmax(r, std::fmax(g, b));
            uint8_t* e = &line[size_t(x) * 4];
            e[0] = e[1] = e[2] = e[3] = 0;
            if (m > 1e-32f) {
                int ex;
                const float s = std::frexp(m, &ex) * 256.0f / m;
                if (ex > 127) {  // beyond RGBE's range: the largest value
                    e[0] = e[1] = e[2] = e[3] = 255;
                } else {
                    e[0] = uint8_t(r * s); e[1] = uint8_t(g * s); e[2] = uint8_t(b * s); e[3] = uint8_t(ex + 128);
                }
            }
        }
        if (!rle) {
            f.write(reinterpret_cast<const char*>(line.data()), std::streamsize(line.size()));
            continue;
        }
        const uint8_t head[4] = {2, 2, uint8_t(w >> 8), uint8_t(w & 255)};
        f.write(reinterpret_cast<const char*>(head), 4);
        for (int c = 0; c < 4; ++c) {
            for (int x = 0; x < w; ++x) comp[size_t(x)] = line[size_t(x) * 4 + c];
            rle_component(f, comp.data(), w);
        }
    }
    if (!f) throw ConfigError("failed to write: " + fn);
}

}  // namespace atrc
