// AtrcSceneDesc -> device layout.  The per-triangle data follows the
// reference's construction exactly (same float operations in the same order)
// so that device hits are bit-identical to the reference's:
//   - TriangleBVH::load bakes positions with local_to_world
//     (src/tracer/src/core/geometry/triangle_bvh.cpp:533-558), then stores
//     A, B-A, C-A, z = normalize(cross(B-A, C-A)) flipped toward the mean
//     vertex normal, x = dpdu (triangle_bvh.cpp:267-299);
//   - Quad bakes A..D and splits into ABC / ACD (quad.cpp:134-157);
//   - Triangle keeps local vertices and moves rays to local space
//     (triangle.cpp:31-51, 108-125).
#include "scene_build.h"

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <stdexcept>

namespace atrc {

namespace {

const float kPi = 3.14159265358979323846f;

struct Bound {
    Vec3 lo{3.402823466e38f}, hi{-3.402823466e38f};
    void add(Vec3 p) { lo = vmin(lo, p); hi = vmax(hi, p); }
    void add(const Bound& b) { add(b.lo); add(b.hi); }
};

void widen_degenerate(Bound& b) {
    for (int i = 0; i < 3; ++i)
        if (b.lo[i] >= b.hi[i]) b.lo[i] = b.hi[i] - 0.1f * std::fabs(b.hi[i]);
}

Vec3 V(const float* p) { return Vec3(p[0], p[1], p[2]); }

float tri_area(Vec3 ba, Vec3 ca) { return length(cross(ba, ca)) / 2; }

// from_z convention shared with the device: x from the axis least aligned
Vec3 from_z_x(Vec3 z) {
    Vec3 zz = normalize(z);
    Vec3 t = std::fabs(zz.x) > 0.9f ? Vec3(0, 1, 0) : Vec3(1, 0, 0);
    Vec3 y = normalize(cross(zz, t));
    return cross(y, zz);
}

// triangle_aux.h:76-88
Vec3 dpdu_as_ex(Vec3 ba, Vec3 ca, Vec2 tba, Vec2 tca, Vec3 nor) {
    const float m00 = tba.x, m01 = tba.y, m10 = tca.x, m11 = tca.y;
    const float det = m00 * m11 - m01 * m10;
    if (!det) return from_z_x(nor);
    const float inv_det = 1 / det;
    return normalize(m11 * inv_det * ba - m01 * inv_det * ca);
}

// A triangle in leaf order: A, B - A, C - A for Moller-Trumbore (the edges
// as the reference computes them) and the exact vertices B, C for the
// watertight test, which needs every shared vertex bit-identical in the
// triangles that share it (A + (B - A) does not round back to B).
void put_tri(HostScene* hs, Vec3 a, Vec3 ba, Vec3 ca, Vec3 b, Vec3 c, const dev::TriShade& sh, uint32_t orig) {
    const float t[12] = {a.x, a.y, a.z, 0, ba.x, ba.y, ba.z, 0, ca.x, ca.y, ca.z, 0};
    hs->tris.insert(hs->tris.end(), t, t + 12);
    const float v[8] = {b.x, b.y, b.z, 0, c.x, c.y, c.z, 0};
    hs->tri_bc.insert(hs->tri_bc.end(), v, v + 8);
    hs->tri_shade.push_back(sh);
    hs->tri_orig.push_back(orig);
}

void set3(float* d, Vec3 v) { d[0] = v.x; d[1] = v.y; d[2] = v.z; }
void set2(float* d, Vec2 v) { d[0] = v.x; d[1] = v.y; }

// Walker alias table (Vose), built in double precision.
void build_alias(const std::vector<double>& w, std::vector<float>* prob, std::vector<int32_t>* alias) {
    const size_t n = w.size();
    size_t base = prob->size();
    prob->resize(base + n);
    alias->resize(base + n);
    double sum = 0;
    for (double x : w) sum += x;
    std::vector<double> p(n);
    std::vector<size_t> small, large;
    for (size_t i = 0; i < n; ++i) {
        p[i] = sum > 0 ? w[i] * double(n) / sum : 1.0;
        (p[i] < 1 ? small : large).push_back(i);
    }
    while (!small.empty() && !large.empty()) {
        size_t s = small.back(); small.pop_back();
        size_t l = large.back(); large.pop_back();
        (*prob)[base + s] = float(p[s]);
        (*alias)[base + s] = int32_t(l);
        p[l] = (p[l] + p[s]) - 1.0;
        (p[l] < 1 ? small : large).push_back(l);
    }
    for (size_t i : large) { (*prob)[base + i] = 1; (*alias)[base + i] = int32_t(i); }
    for (size_t i : small) { (*prob)[base + i] = 1; (*alias)[base + i] = int32_t(i); }
}

struct LeafInfo {
    int kind = dev::LEAF_TRIANGLES;
    int32_t root = 0;
    int32_t tri_first = 0, tri_count = 0;
    Bound bound;           // in the leaf's own world (baked) space
    float area = 0;        // leaf surface area (reference Geometry::surface_area)
    float abc_prob = 0;
    int32_t alias_first = -1;
    std::vector<double> tri_areas;  // for the alias table (pool order)
};

// Sample a texture on the host (for the environment importance table).
struct HostTex {
    const AtrcTexture2DDesc* d;
    Vec3 texel(int x, int y) const {
        const float* p = d->data + (size_t(y) * d->width + x) * 3;
        return Vec3(p[0], p[1], p[2]);
    }
    static float wrap(int mode, float x) {
        if (mode == ATRC_WRAP_REPEAT) return std::fmin(std::fmax(x - std::floor(x), 0.f), 1.f);
        if (mode == ATRC_WRAP_MIRROR) {
            const int ip = int(x >= 0 ? x : std::floor(x));
            float r = (ip & 1) ? 1 - x + ip : x - ip;
            return std::fmin(std::fmax(r, 0.f), 1.f);
        }
        return std::fmin(std::fmax(x, 0.f), 1.f);
    }
    Vec3 sample(float u, float v) const {
        if (d->type == ATRC_TEX_CONSTANT) return Vec3(d->texel[0], d->texel[1], d->texel[2]);
        const float* m = d->uv_transform;
        float tu = m[0] * u + m[1] * v + m[2], tv = m[3] * u + m[4] * v + m[5];
        tu = wrap(d->wrap_u, tu);
        tv = wrap(d->wrap_v, tv);
        Vec3 r;
        if (d->type == ATRC_TEX_CHECKER) {
            const float gs = 1.0f / float(d->grid_count);
            const int ui = int(std::fmin(std::fmax(tu, 0.f), 1.f) / gs), vi = int(std::fmin(std::fmax(tv, 0.f), 1.f) / gs);
            r = ((ui + vi) & 1) ? Vec3(d->texel[0], d->texel[1], d->texel[2]) : Vec3(d->texel2[0], d->texel2[1], d->texel2[2]);
        } else if (d->nearest) {
            r = texel(std::min(int(tu * d->width), d->width - 1), std::min(int(tv * d->height), d->height - 1));
        } else {
            float fx = tu * d->width - 0.5f, fy = tv * d->height - 0.5f;
            float flx = std::floor(fx), fly = std::floor(fy);
            int x0 = int(flx), y0 = int(fly);
            float ax = fx - flx, ay = fy - fly;
            int x1 = std::max(std::min(x0 + 1, d->width - 1), 0), y1 = std::max(std::min(y0 + 1, d->height - 1), 0);
            x0 = std::max(x0, 0); y0 = std::max(y0, 0);
            Vec3 a = texel(x0, y0) * (1 - ax) + texel(x1, y0) * ax;
            Vec3 b = texel(x0, y1) * (1 - ax) + texel(x1, y1) * ax;
            r = a * (1 - ay) + b * ay;
        }
        if (d->inv_gamma != 1) r = Vec3(std::pow(r.x, d->inv_gamma), std::pow(r.y, d->inv_gamma), std::pow(r.z, d->inv_gamma));
        return r;
    }
};

float lum(Vec3 c) { return 0.2126f * c.x + 0.7152f * c.y + 0.0722f * c.z; }

}  // namespace

void build_host_scene(const AtrcSceneDesc& d, HostScene* hs, int device) {
    if (d.abi_version != ATRC_ABI_VERSION) throw std::runtime_error("scene description ABI version mismatch");
    if (d.bvh_builder < ATRC_BVH_SAH || d.bvh_builder > ATRC_BVH_AUTO) throw std::runtime_error("invalid bvh_builder");
    *hs = HostScene();
    // ------------------------------------------------------------- leaves
    std::vector<LeafInfo> leaves(d.geometry_count);
    for (uint32_t gi = 0; gi < d.geometry_count; ++gi) {
        const AtrcGeometryDesc& g = d.geometries[gi];
        LeafInfo& L = leaves[gi];
        const float* m = g.transform.m;
        std::vector<BuildPrim> prims;
        std::vector<Vec3> ta, tba, tca, tb, tc;
        std::vector<dev::TriShade> tsh;
        std::vector<uint32_t> torig;
        // (a, b, c): the exact vertices; ba = b - a and ca = c - a as computed
        // by the caller
        auto add_tri = [&](Vec3 a, Vec3 ba, Vec3 ca, Vec3 b_exact, Vec3 c_exact, const dev::TriShade& sh,
                           uint32_t orig) {
            BuildPrim bp;
            Vec3 b = a + ba, c = a + ca;
            Vec3 lo = vmin(a, vmin(b, c)), hi = vmax(a, vmax(b, c));
            lo = vmin(lo, vmin(b_exact, c_exact));
            hi = vmax(hi, vmax(b_exact, c_exact));
            bp.lo[0] = lo.x; bp.lo[1] = lo.y; bp.lo[2] = lo.z;
            bp.hi[0] = hi.x; bp.hi[1] = hi.y; bp.hi[2] = hi.z;
            prims.push_back(bp);
            ta.push_back(a); tba.push_back(ba); tca.push_back(ca);
            tb.push_back(b_exact); tc.push_back(c_exact);
            tsh.push_back(sh);
            torig.push_back(orig);
        };
        if (g.type == ATRC_GEOM_TRIANGLE_BVH) {
            if (g.mesh < 0 || uint32_t(g.mesh) >= d.mesh_count) throw std::runtime_error("bad mesh index");
            const AtrcMeshDesc& mesh = d.meshes[g.mesh];
            if (mesh.triangle_count == 0) throw std::runtime_error("empty mesh");
            L.area = 0;
            for (uint64_t t = 0; t < mesh.triangle_count; ++t) {
                const float* v = mesh.vertices + t * 24;
                Vec3 p[3], n[3];
                Vec2 uv[3];
                for (int k = 0; k < 3; ++k) {
                    p[k] = apply_point_rn(m, V(v + 8 * k));
                    n[k] = apply_vector_rn(m, V(v + 8 * k + 3));
                    uv[k] = Vec2(v[8 * k + 6], v[8 * k + 7]);
                }
                L.area += tri_area(p[1] - p[0], p[2] - p[0]);
                Vec3 a = p[0], ba = p[1] - p[0], ca = p[2] - p[0];
                Vec3 na = normalize(n[0]), nb = normalize(n[1]), nc = normalize(n[2]);
                dev::TriShade sh{};
                Vec3 z = normalize(cross(ba, ca));
                if (dot(na + nb + nc, z) < 0) z = -z;
                Vec2 tba2 = uv[1] - uv[0], tca2 = uv[2] - uv[0];
                Vec3 x = dpdu_as_ex(ba, ca, tba2, tca2, z);
                set3(sh.x, x); set3(sh.z, z);
                set3(sh.n_a, na); set3(sh.n_ba, nb - na); set3(sh.n_ca, nc - na);
                set2(sh.t_a, uv[0]); set2(sh.t_ba, tba2); set2(sh.t_ca, tca2);
                add_tri(a, ba, ca, p[1], p[2], sh, uint32_t(t));
            }
        } else if (g.type == ATRC_GEOM_QUAD) {
            Vec3 A = apply_point_rn(m, V(g.p[0])), B = apply_point_rn(m, V(g.p[1]));
            Vec3 C = apply_point_rn(m, V(g.p[2])), D = apply_point_rn(m, V(g.p[3]));
            Vec3 ba = B - A, ca = C - A, da = D - A;
            Vec2 ta2(g.uv[0][0], g.uv[0][1]);
            Vec2 tba2 = Vec2(g.uv[1][0], g.uv[1][1]) - ta2;
            Vec2 tca2 = Vec2(g.uv[2][0], g.uv[2][1]) - ta2;
            Vec2 tda2 = Vec2(g.uv[3][0], g.uv[3][1]) - ta2;
            Vec3 z = normalize(cross(ba, ca));
            Vec3 x_abc = dpdu_as_ex(ba, ca, tba2, tca2, z);
            Vec3 x_acd = dpdu_as_ex(ca, da, tca2, tda2, z);
            float a1 = tri_area(ba, ca), a2 = tri_area(ca, da);
            L.area = a1 + a2;
            L.abc_prob = a1 / L.area;
            dev::TriShade s1{}, s2{};
            set3(s1.x, x_abc); set3(s1.z, z); set3(s1.n_a, z);
            set2(s1.t_a, ta2); set2(s1.t_ba, tba2); set2(s1.t_ca, tca2);
            set3(s2.x, x_acd); set3(s2.z, z); set3(s2.n_a, z);
            set2(s2.t_a, ta2); set2(s2.t_ba, tca2); set2(s2.t_ca, tda2);
            // n_a = z with zero deltas: the shading frame equals the
            // geometric frame (quad.cpp:36,48 user_coord = geometry_coord)
            s1.pad[0] = 1.0f;  // marks "user frame = geometric frame"
            s2.pad[0] = 1.0f;
            add_tri(A, ba, ca, B, C, s1, 0);
            add_tri(A, ca, da, C, D, s2, 1);
            L.bound = Bound();
            L.bound.add(A); L.bound.add(A + ba); L.bound.add(A + ca); L.bound.add(A + da);
            widen_degenerate(L.bound);
        } else if (g.type == ATRC_GEOM_TRIANGLE) {
            Vec3 a = V(g.p[0]), ba = V(g.p[1]) - a, ca = V(g.p[2]) - a;
            Vec2 ta2(g.uv[0][0], g.uv[0][1]);
            Vec2 tba2 = Vec2(g.uv[1][0], g.uv[1][1]) - ta2;
            Vec2 tca2 = Vec2(g.uv[2][0], g.uv[2][1]) - ta2;
            Vec3 z = normalize(cross(ba, ca));
            Vec3 x = dpdu_as_ex(ba, ca, tba2, tca2, z);
            L.area = tri_area(apply_vector_rn(m, ba), apply_vector_rn(m, ca));
            dev::TriShade s{};
            set3(s.x, x); set3(s.z, z); set3(s.n_a, z);
            set2(s.t_a, ta2); set2(s.t_ba, tba2); set2(s.t_ca, tca2);
            s.pad[0] = 1.0f;
            add_tri(a, ba, ca, V(g.p[1]), V(g.p[2]), s, 0);
            L.bound = Bound();
            L.bound.add(apply_point_rn(m, a)); L.bound.add(apply_point_rn(m, a + ba)); L.bound.add(apply_point_rn(m, a + ca));
            widen_degenerate(L.bound);
        } else if (g.type == ATRC_GEOM_SPHERE || g.type == ATRC_GEOM_DISK) {
            if (!(g.radius > 0)) throw std::runtime_error("invalid sphere/disk radius");
            L.kind = g.type == ATRC_GEOM_SPHERE ? dev::LEAF_SPHERE : dev::LEAF_DISK;
            const float ratio = length(apply_vector_rn(m, Vec3(1, 0, 0)));
            L.bound = Bound();
            if (g.type == ATRC_GEOM_SPHERE) {
                const float wr = ratio * g.radius;
                Vec3 o = apply_point_rn(m, Vec3(0.0f));
                L.bound.lo = o - Vec3(wr + 3e-4f);
                L.bound.hi = o + Vec3(wr + 3e-4f);
                L.area = 4 * kPi * wr * wr;
            } else {
                const float vs = std::min(0.1f * g.radius, 0.01f);
                for (int k = 0; k < 8; ++k)
                    L.bound.add(apply_point_rn(m, Vec3(k & 1 ? g.radius : -g.radius, k & 2 ? g.radius : -g.radius, k & 4 ? vs : -vs)));
                L.area = ratio * ratio * kPi * g.radius * g.radius;
            }
            continue;
        } else {
            throw std::runtime_error("unknown geometry type");
        }
        // bottom-level BVH over this leaf's triangles
        const bool ploc = device >= 0 && (d.bvh_builder == ATRC_BVH_PLOC ||
                                          (d.bvh_builder == ATRC_BVH_AUTO && prims.size() >= (size_t(1) << 18)));
        WideBvh bvh;
        if (ploc) {
            bvh = ploc_wide_device(prims, device);
        } else {
            BvhResult bin = build_bvh(prims, 4);
            bvh.root = collapse_bvh4(bin, &bvh.nodes);
            bvh.order = std::move(bin.order);
            std::copy(bin.bound_lo, bin.bound_lo + 3, bvh.bound_lo);
            std::copy(bin.bound_hi, bin.bound_hi + 3, bvh.bound_hi);
        }
        hs->max_blas_depth = std::max(hs->max_blas_depth, bvh4_depth(bvh.nodes, bvh.root));
        const int32_t tri_off = int32_t(hs->tri_shade.size());
        const int32_t first_node = int32_t(hs->nodes.size());
        // into the scene's node array: interior links shift by the nodes
        // already there, leaf links by the triangles already there
        auto place = [&](int32_t link) -> int32_t {
            if (link == kEmptyLink) return link;
            if (link >= 0) return link + first_node;
            uint32_t enc = uint32_t(~link);
            return leaf_link((enc >> 4) + uint32_t(tri_off), (enc & 15) + 1);
        };
        if (hs->nodes.size() + bvh.nodes.size() >= size_t(INT32_MAX)) throw std::runtime_error("too many BVH nodes");
        for (Bvh4Node w : bvh.nodes) {
            for (int32_t& l : w.link) l = place(l);
            hs->nodes.push_back(w);
        }
        L.root = place(bvh.root);
        if (bvh.order.size() != prims.size()) throw std::runtime_error("BVH leaf order does not cover the triangles");
        validate_bvh4(hs->nodes, L.root, uint32_t(tri_off), uint32_t(prims.size()));
        L.tri_first = tri_off;
        L.tri_count = int32_t(prims.size());
        if (g.type == ATRC_GEOM_TRIANGLE_BVH) {
            L.bound = Bound();
            L.bound.lo = Vec3(bvh.bound_lo[0], bvh.bound_lo[1], bvh.bound_lo[2]);
            L.bound.hi = Vec3(bvh.bound_hi[0], bvh.bound_hi[1], bvh.bound_hi[2]);
            widen_degenerate(L.bound);
        }
        std::vector<uint8_t> placed(prims.size(), 0);
        for (uint32_t k : bvh.order) {
            if (k >= prims.size() || placed[k]) throw std::runtime_error("BVH leaf order is not a permutation");
            placed[k] = 1;
            put_tri(hs, ta[k], tba[k], tca[k], tb[k], tc[k], tsh[k], torig[k]);
            L.tri_areas.push_back(double(tri_area(tba[k], tca[k])));
        }
    }

    // leaf links encode (first << 4 | count - 1) in 31 bits; the two most
    // negative links are reserved as traversal markers
    if (hs->tri_shade.size() >= (size_t(1) << 27) - 2)
        throw std::runtime_error("scene has too many triangles for one device scene (limit 134M)");

    // ------------------------------------------------------------ entities
    std::vector<bool> leaf_needs_alias(d.geometry_count, false);
    std::vector<Bound> ent_bounds(d.entity_count);
    for (uint32_t ei = 0; ei < d.entity_count; ++ei) {
        const AtrcEntityDesc& e = d.entities[ei];
        if (e.geometry < 0 || uint32_t(e.geometry) >= d.geometry_count) throw std::runtime_error("bad geometry index");
        if (e.material < 0 || uint32_t(e.material) >= d.material_count) throw std::runtime_error("bad material index");
        if (e.medium_in < 0 || uint32_t(e.medium_in) >= d.medium_count || e.medium_out < 0 ||
            uint32_t(e.medium_out) >= d.medium_count)
            throw std::runtime_error("bad medium index");
        const AtrcGeometryDesc& g = d.geometries[e.geometry];
        const LeafInfo& L = leaves[e.geometry];
        dev::Entity de{};
        de.kind = L.kind;
        de.blas_root = L.root;
        de.tri_first = L.tri_first;
        de.tri_count = L.tri_count;
        de.geom_type = g.type;
        de.material = e.material;
        de.med_in = e.medium_in;
        de.med_out = e.medium_out;
        de.flags = 0;
        if (e.has_instance) de.flags |= dev::ENT_WRAP;
        if (g.type == ATRC_GEOM_TRIANGLE || g.type == ATRC_GEOM_SPHERE || g.type == ATRC_GEOM_DISK) de.flags |= dev::ENT_LOCAL;
        if (e.double_sided) de.flags |= dev::ENT_DOUBLE_SIDED;
        if (e.no_denoise) de.flags |= dev::ENT_NO_DENOISE;
        const bool light = e.emit_radiance[0] != 0 || e.emit_radiance[1] != 0 || e.emit_radiance[2] != 0;
        if (light) de.flags |= dev::ENT_LIGHT;
        std::memcpy(de.wrap_m, e.instance.m, sizeof(de.wrap_m));
        std::memcpy(de.wrap_inv, e.instance.inv, sizeof(de.wrap_inv));
        std::memcpy(de.local_m, g.transform.m, sizeof(de.local_m));
        std::memcpy(de.local_inv, g.transform.inv, sizeof(de.local_inv));
        set3(de.emit, Vec3(e.emit_radiance[0], e.emit_radiance[1], e.emit_radiance[2]));
        de.radius = g.radius;
        const float ratio = length(apply_vector_rn(g.transform.m, Vec3(1, 0, 0)));
        de.world_radius = ratio * g.radius;
        de.wrap_scale = e.has_instance ? length(apply_vector_rn(e.instance.m, Vec3(0, 0, 1))) : 1.0f;
        de.leaf_area = L.area;
        de.area = L.area * (e.has_instance ? de.wrap_scale * de.wrap_scale : 1.0f) * (e.double_sided ? 2.0f : 1.0f);
        de.quad_abc_prob = L.abc_prob;
        de.alias_first = -1;
        if (light && g.type == ATRC_GEOM_TRIANGLE_BVH) leaf_needs_alias[e.geometry] = true;
        hs->entities.push_back(de);
        // world bound (transform_wrapper.cpp:13-27)
        Bound b;
        if (e.has_instance) {
            Vec3 lo = L.bound.lo, hi = L.bound.hi;
            for (int k = 0; k < 8; ++k)
                b.add(apply_point_rn(e.instance.m, Vec3(k & 4 ? hi.x : lo.x, k & 2 ? hi.y : lo.y, k & 1 ? hi.z : lo.z)));
        } else {
            b = L.bound;
        }
        ent_bounds[ei] = b;
    }
    // triangle-area alias tables for mesh lights
    std::vector<int32_t> leaf_alias(d.geometry_count, -1);
    for (uint32_t gi = 0; gi < d.geometry_count; ++gi) {
        if (!leaf_needs_alias[gi]) continue;
        leaf_alias[gi] = int32_t(hs->alias_prob.size());
        std::vector<float> p;
        std::vector<int32_t> a;
        build_alias(leaves[gi].tri_areas, &p, &a);
        hs->alias_prob.insert(hs->alias_prob.end(), p.begin(), p.end());
        hs->alias_idx.insert(hs->alias_idx.end(), a.begin(), a.end());
    }
    for (uint32_t ei = 0; ei < d.entity_count; ++ei)
        hs->entities[ei].alias_first = leaf_alias[d.entities[ei].geometry];

    // ---------------------------------------------------------------- TLAS
    if (d.entity_count > 0) {
        std::vector<BuildPrim> eprims(d.entity_count);
        for (uint32_t ei = 0; ei < d.entity_count; ++ei) {
            for (int k = 0; k < 3; ++k) {
                eprims[ei].lo[k] = ent_bounds[ei].lo[k];
                eprims[ei].hi[k] = ent_bounds[ei].hi[k];
            }
        }
        BvhResult tl = build_bvh(eprims, 1);  // one entity per top-level leaf
        hs->tlas_depth = tl.max_depth;
        hs->scene.tlas_root = collapse_bvh4(tl, &hs->nodes);
        validate_bvh4(hs->nodes, hs->scene.tlas_root, 0, uint32_t(d.entity_count));
        hs->tlas_order = tl.order;
    } else {
        hs->scene.tlas_root = 0;
    }
    hs->scene.entity_count = int32_t(d.entity_count);
    Bound world;
    for (auto& b : ent_bounds) world.add(b);
    for (int k = 0; k < 3; ++k) { hs->scene.scene_lo[k] = world.lo[k]; hs->scene.scene_hi[k] = world.hi[k]; }

    // ------------------------------------------------------------ textures
    for (uint32_t i = 0; i < d.texture2d_count; ++i) {
        const AtrcTexture2DDesc& t = d.textures2d[i];
        dev::Texture2D dt{};
        dt.type = t.type;
        dt.width = t.width;
        dt.height = t.height;
        dt.nearest = t.nearest;
        std::memcpy(dt.texel, t.texel, sizeof(dt.texel));
        dt.inv_gamma = t.inv_gamma;
        std::memcpy(dt.uv, t.uv_transform, sizeof(dt.uv));
        dt.wrap_u = t.wrap_u;
        dt.wrap_v = t.wrap_v;
        dt.data_offset = -1;
        if (t.type == ATRC_TEX_CHECKER) {
            if (t.grid_count <= 0) throw std::runtime_error("invalid grid_count value");
            std::memcpy(dt.texel2, t.texel2, sizeof(dt.texel2));
            dt.grid_size = 1.0f / float(t.grid_count);
        }
        if (t.type == ATRC_TEX_IMAGE) {
            if (t.width <= 0 || t.height <= 0 || !t.data) throw std::runtime_error("invalid image texture");
            dt.data_offset = int64_t(hs->texels.size());
            hs->texels.insert(hs->texels.end(), t.data, t.data + size_t(t.width) * t.height * 3);
        }
        dt.tex3d = -1;
        if (t.type == ATRC_TEX_SOLID) {
            if (t.tex3d < 0 || uint32_t(t.tex3d) >= d.texture3d_count) throw std::runtime_error("bad solid_image texture");
            dt.tex3d = t.tex3d;
        } else if (t.type != ATRC_TEX_CONSTANT && t.type != ATRC_TEX_IMAGE && t.type != ATRC_TEX_CHECKER) {
            throw std::runtime_error("unknown texture2d type");
        }
        hs->tex2d.push_back(dt);
    }
    for (uint32_t i = 0; i < d.texture3d_count; ++i) {
        const AtrcTexture3DDesc& t = d.textures3d[i];
        dev::Texture3D dt{};
        dt.type = t.type;
        dt.width = t.width; dt.height = t.height; dt.depth = t.depth;
        dt.channels = t.channels;
        dt.nearest = t.nearest;
        std::memcpy(dt.wrap, t.wrap, sizeof(dt.wrap));
        std::memcpy(dt.texel, t.texel, sizeof(dt.texel));
        dt.inv_gamma = t.inv_gamma;
        dt.max_real = t.max_real;
        std::memcpy(dt.uvw, t.uvw_transform, sizeof(dt.uvw));
        dt.data_offset = -1;
        if (t.type == ATRC_TEX_IMAGE) {
            if (!t.data || t.width <= 0 || t.height <= 0 || t.depth <= 0) throw std::runtime_error("invalid 3d texture");
            dt.data_offset = int64_t(hs->texels.size());
            hs->texels.insert(hs->texels.end(), t.data, t.data + size_t(t.width) * t.height * t.depth * t.channels);
        }
        hs->tex3d.push_back(dt);
    }

    // ----------------------------------------------------------- materials
    for (uint32_t i = 0; i < d.material_count; ++i) {
        const AtrcMaterialDesc& m = d.materials[i];
        dev::Material dm{};
        dm.type = m.type;
        std::memcpy(dm.tex, m.tex, sizeof(dm.tex));
        dm.normal_map = m.normal_map;
        // texture slots each type reads; Lambert and Disney materials whose
        // textures are all constant are folded into c[]
        int slots = 0;
        switch (m.type) {
            case ATRC_MAT_DISNEY: slots = ATRC_DISNEY_SLOT_COUNT; break;
            case ATRC_MAT_IDEAL_DIFFUSE: slots = 1; break;
            case ATRC_MAT_MIRROR: case ATRC_MAT_GLASS: case ATRC_MAT_PHONG: slots = 3; break;
            case ATRC_MAT_METAL: slots = 5; break;
            case ATRC_MAT_IDEAL_BLACK: case ATRC_MAT_INVISIBLE_SURFACE: break;
            default: throw std::runtime_error("unknown material type");
        }
        bool all_const = m.normal_map < 0;
        for (int s = 0; s < slots; ++s) {
            if (m.tex[s] < 0 || uint32_t(m.tex[s]) >= d.texture2d_count) throw std::runtime_error("bad texture index");
            if (d.textures2d[m.tex[s]].type != ATRC_TEX_CONSTANT) all_const = false;
        }
        if (m.normal_map >= 0 && uint32_t(m.normal_map) >= d.texture2d_count) throw std::runtime_error("bad texture index");
        const bool sss = m.bssrdf[1] >= 0;
        if (sss) hs->scene.has_subsurface = 1;
        for (int s = 0; s < 3; ++s) {
            dm.bssrdf[s] = sss ? m.bssrdf[s] : -1;
            if (sss && (m.type != ATRC_MAT_DISNEY || m.bssrdf[s] < 0 || uint32_t(m.bssrdf[s]) >= d.texture2d_count))
                throw std::runtime_error("bad subsurface texture index (Disney materials only)");
        }
        if (m.type != ATRC_MAT_DISNEY && m.type != ATRC_MAT_IDEAL_DIFFUSE) all_const = false;
        dm.all_constant = all_const;
        if (all_const && slots > 0) {
            auto T = [&](int s) { return d.textures2d[m.tex[s]].texel; };
            const float* bc = T(0);
            dm.c[0] = bc[0]; dm.c[1] = bc[1]; dm.c[2] = bc[2];
            if (m.type == ATRC_MAT_DISNEY) {
                dm.c[3] = T(ATRC_DISNEY_METALLIC)[0];
                dm.c[4] = T(ATRC_DISNEY_ROUGHNESS)[0];
                dm.c[5] = T(ATRC_DISNEY_TRANSMISSION)[0];
                dm.c[6] = T(ATRC_DISNEY_TRANSMISSION_ROUGHNESS)[0];
                dm.c[7] = T(ATRC_DISNEY_IOR)[0];
                const float* ss = T(ATRC_DISNEY_SPECULAR_SCALE);
                dm.c[8] = ss[0]; dm.c[9] = ss[1]; dm.c[10] = ss[2];
                dm.c[11] = T(ATRC_DISNEY_SPECULAR_TINT)[0];
                dm.c[12] = T(ATRC_DISNEY_ANISOTROPIC)[0];
                dm.c[13] = T(ATRC_DISNEY_SHEEN)[0];
                dm.c[14] = T(ATRC_DISNEY_SHEEN_TINT)[0];
                dm.c[15] = T(ATRC_DISNEY_CLEARCOAT)[0];
                dm.cc_gloss = T(ATRC_DISNEY_CLEARCOAT_GLOSS)[0];
            }
        }
        hs->materials.push_back(dm);
    }

    // --------------------------------------------------------------- media
    bool has_media = false;
    for (uint32_t i = 0; i < d.medium_count; ++i) {
        const AtrcMediumDesc& m = d.media[i];
        dev::Medium dm{};
        dm.type = m.type;
        dm.max_scattering_count = m.max_scattering_count;
        for (int k = 0; k < 3; ++k) {
            dm.sigma_a[k] = m.sigma_a[k];
            dm.sigma_s[k] = m.sigma_s[k];
            dm.sigma_t[k] = m.sigma_a[k] + m.sigma_s[k];
        }
        dm.g = m.g;
        std::memcpy(dm.inv, m.transform.inv, sizeof(dm.inv));
        dm.density = m.density;
        dm.albedo = m.albedo;
        dm.g_tex = m.g_tex;
        dm.white_for_indirect = m.white_for_indirect;
        if (m.type == ATRC_MED_HETEROGENEOUS) {
            if (m.density < 0 || uint32_t(m.density) >= d.texture3d_count || m.albedo < 0 ||
                uint32_t(m.albedo) >= d.texture3d_count || m.g_tex < 0 || uint32_t(m.g_tex) >= d.texture3d_count)
                throw std::runtime_error("bad 3d texture index");
            // heterogeneous.cpp:37-41 (EPS floor uses the default epsilon)
            dm.max_density = std::max(d.textures3d[m.density].max_real, 3e-4f);
            dm.inv_max_density = 1 / dm.max_density;
        }
        if (m.type == ATRC_MED_HOMOGENEOUS && (m.g <= -1 || m.g >= 1)) throw std::runtime_error("invalid g value");
        if (m.type != ATRC_MED_VOID) has_media = true;
        hs->media.push_back(dm);
    }
    if (hs->media.empty()) {
        dev::Medium v{};
        v.type = ATRC_MED_VOID;
        v.max_scattering_count = 0x7fffffff;
        hs->media.push_back(v);
    }
    hs->scene.medium_count = int32_t(hs->media.size());
    hs->scene.has_media = has_media;

    // --------------------------------------------------------------- lights
    int nl = 0;
    dev::Env& env = hs->scene.env;
    env.type = d.env.type;
    env.tex = d.env.tex;
    if (d.env.type != ATRC_ENV_NONE) {
        hs->scene.light_entity[nl++] = -1;
        set3(env.top, Vec3(d.env.top[0], d.env.top[1], d.env.top[2]));
        set3(env.bottom, Vec3(d.env.bottom[0], d.env.bottom[1], d.env.bottom[2]));
        // EnvirLight::preprocess (light.cpp:6-14)
        if (d.entity_count) {
            env.radius = 1.1f * length(world.hi - world.lo) / 2;
            Vec3 c = 0.5f * (world.lo + world.hi);
            set3(env.centre, c);
        } else {
            env.radius = 1;
        }
        if (d.env.type == ATRC_ENV_IBL) {
            if (d.env.tex < 0 || uint32_t(d.env.tex) >= d.texture2d_count) throw std::runtime_error("bad env texture");
            // EnvironmentLightSampler (env_sampler.h:15-104), table in FP64
            const AtrcTexture2DDesc& td = d.textures2d[d.env.tex];
            if (td.type == ATRC_TEX_SOLID) throw std::runtime_error("solid_image is not supported as an environment map");
            const bool uniform = d.env.no_importance_sampling || td.type == ATRC_TEX_CONSTANT;
            const int tw = uniform ? 1 : td.width, th = uniform ? 1 : td.height;
            const int pw = std::min(tw, 200), ph = std::min(th, 200);
            HostTex ht{&td};
            std::vector<double> probs(size_t(pw) * ph);
            double sum = 0;
            for (int y = 0; y < ph; ++y) {
                const double y0 = double(y) / ph, y1 = double(y + 1) / ph;
                const int ys0 = std::max(0, int(std::floor(y0 * th) - 1));
                const int ys1 = std::min(th - 1, int(std::floor(y1 * th) + 1));
                for (int x = 0; x < pw; ++x) {
                    const double x0 = double(x) / pw, x1 = double(x + 1) / pw;
                    const int xs0 = std::max(0, int(std::floor(x0 * tw) - 1));
                    const int xs1 = std::min(tw - 1, int(std::floor(x1 * tw) + 1));
                    double pl = 0;
                    for (int ys = ys0; ys <= ys1; ++ys)
                        for (int xs = xs0; xs <= xs1; ++xs)
                            pl += uniform ? 1.0 : double(lum(ht.sample((xs + 0.5f) / tw, (ys + 0.5f) / th)));
                    const double da = std::fabs(2 * M_PI * (x1 - x0) * (std::cos(M_PI * y1) - std::cos(M_PI * y0)));
                    probs[size_t(y) * pw + x] = pl * da;
                    sum += pl * da;
                }
            }
            if (sum > 3e-4) for (auto& p : probs) p /= sum;
            hs->env_probs.resize(probs.size());
            for (size_t i = 0; i < probs.size(); ++i) hs->env_probs[i] = float(probs[i]);
            build_alias(probs, &hs->env_alias_prob, &hs->env_alias_idx);
            env.pw = pw;
            env.ph = ph;
        }
    }
    for (uint32_t ei = 0; ei < d.entity_count; ++ei) {
        if (hs->entities[ei].flags & dev::ENT_LIGHT) {
            if (nl >= dev::kMaxLights)
                throw std::runtime_error("pt_cuda supports at most " + std::to_string(dev::kMaxLights) + " lights");
            hs->scene.light_entity[nl++] = int32_t(ei);
        }
    }
    hs->scene.light_count = nl;
}

}  // namespace atrc
