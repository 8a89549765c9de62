"""Known-answer scenes shared by the oracle and the GPU known-answer tests."""
from __future__ import annotations

import json
import math
from pathlib import Path

import numpy as np


def furnace(width=24, height=24, spp=64, renderer="pt", albedo=1.0, max_depth=64) -> dict:
    """A Lambertian sphere of albedo 1 under a uniform sky of radiance 1.
    The sphere is convex, so every reflected ray escapes: each pixel's
    expected value is exactly 1 (the sphere reflects all it receives)."""
    return {"scene": {"type": "default",
                      "entities": [{"type": "geometric",
                                    "geometry": {"type": "sphere", "radius": 1, "transform": []},
                                    "material": {"type": "ideal_diffuse",
                                                 "albedo": {"type": "constant", "texel": [albedo]}}}],
                      "env": {"type": "native_sky", "top": [1], "bottom": [1]}},
            "rendering": {"camera": {"type": "thin_lens", "pos": [0, -4, 0], "dst": [0, 0, 0], "up": [0, 0, 1],
                                     "fov": 40},
                          "width": width, "height": height,
                          "renderer": {"type": renderer, "spp": spp, "max_depth": max_depth, "min_depth": 5},
                          "reporter": {"type": "noout"}}}


def slab(tmp: Path, sigma_a=0.7, thickness=2.0, renderer="pt", spp=16) -> tuple[dict, float]:
    """A purely absorbing homogeneous slab (sigma_s = 0) between a narrow
    camera and a uniform sky of radiance 1: the centre pixel sees exp(-sigma_a d)."""
    from atrc_b200.scenes import _box_mesh, write_bm
    p, n, uv = _box_mesh((0.5, 0.5, 0.5))
    write_bm(tmp / "unitbox.bm", p + 0.5, n, uv)
    cfg = {"scene": {"type": "default",
                     "entities": [{"type": "geometric",
                                   "geometry": {"type": "triangle_bvh", "filename": "${scene-directory}/unitbox.bm",
                                                "transform": [{"type": "translate", "offset": [-2, -thickness / 2, -2]},
                                                              {"type": "scale", "ratio": [4, thickness, 4]}]},
                                   "material": {"type": "invisible_surface"},
                                   "med_in": {"type": "homogeneous", "sigma_a": [sigma_a], "sigma_s": [0], "g": 0}}],
                     "env": {"type": "native_sky", "top": [1], "bottom": [1]}},
           "rendering": {"camera": {"type": "thin_lens", "pos": [0, -6, 0], "dst": [0, 0, 0], "up": [0, 0, 1],
                                    "fov": 2},
                         "width": 9, "height": 9, "renderer": {"type": renderer, "spp": spp, "max_depth": 16},
                         "reporter": {"type": "noout"}}}
    return cfg, math.exp(-sigma_a * thickness)


def edge_rays():
    """Rays aimed exactly at vertices, edges and the shared diagonal of a quad
    made of two triangles (Moller-Trumbore's inclusive bounds count them)."""
    from atrc_b200 import RAY_DTYPE
    targets = [(-1, -1), (1, -1), (1, 1), (-1, 1), (0, 0), (0.5, 0.5), (0, -1), (1, 0), (-0.25, 0.25),
               (1.00001, 0), (-1.00001, 0.3), (0.3, 0.2)]
    r = np.zeros(len(targets), RAY_DTYPE)
    for i, (x, y) in enumerate(targets):
        r[i]["o"] = (x, y, 2.0)
        r[i]["d"] = (0, 0, -1)
        r[i]["t_max"] = np.inf
    return r, np.array([abs(x) <= 1 and abs(y) <= 1 for x, y in targets])


def edge_scene() -> dict:
    return {"scene": {"type": "default",
                      "entities": [{"type": "geometric",
                                    "geometry": {"type": "quad", "A": [-1, -1, 0], "B": [1, -1, 0], "C": [1, 1, 0],
                                                 "D": [-1, 1, 0], "transform": []},
                                    "material": {"type": "ideal_black"}}]},
            "rendering": {"camera": {"type": "thin_lens", "pos": [0, 0, 3], "dst": [0, 0, 0], "up": [0, 1, 0],
                                     "fov": 40},
                          "width": 4, "height": 4, "renderer": {"type": "pt", "spp": 1}, "reporter": {"type": "noout"}}}


def material_probe(material: dict) -> dict:
    return {"scene": {"type": "default",
                      "entities": [{"type": "geometric",
                                    "geometry": {"type": "quad", "A": [-1, -1, 0], "B": [1, -1, 0], "C": [1, 1, 0],
                                                 "D": [-1, 1, 0], "transform": []},
                                    "material": material}]},
            "rendering": {"camera": {"type": "thin_lens", "pos": [0, 0, 3], "dst": [0, 0, 0], "up": [0, 1, 0],
                                     "fov": 40},
                          "width": 4, "height": 4, "renderer": {"type": "pt", "spp": 1}, "reporter": {"type": "noout"}}}


def dumps(cfg: dict) -> str:
    return json.dumps(cfg)


def feature_scene(tmp: Path, renderer="pt", spp=256, width=48, height=36, gaussian=False) -> dict:
    """Every pt feature the benchmark workloads leave out, in one small scene:
    sphere / disk / single triangle / double-sided geometry, nested instances,
    image textures with repeat wrap and uv transforms, a normal map, Disney
    transmission, clearcoat, sheen and anisotropy, sphere and disk area lights,
    the native sky, a thin-lens camera with depth of field and (optionally)
    the Gaussian film filter."""
    from atrc_b200.scenes import _box_mesh, write_bm, write_pfm
    rng = np.random.default_rng(77)
    write_pfm(tmp / "checker.pfm", np.kron(rng.uniform(0.1, 0.9, (4, 4, 3)), np.ones((8, 8, 1))).astype(np.float32))
    nm = np.zeros((16, 16, 3), np.float32)
    yy, xx = np.mgrid[0:16, 0:16] / 16.0
    nm[..., 0] = 0.5 + 0.3 * np.sin(6 * xx)
    nm[..., 1] = 0.5 + 0.3 * np.cos(6 * yy)
    nm[..., 2] = 0.9
    write_pfm(tmp / "normal.pfm", nm)
    p, n, uv = _box_mesh((0.4, 0.4, 0.4))
    write_bm(tmp / "box.bm", p, n, uv)

    def const(v):
        return {"type": "constant", "texel": list(np.atleast_1d(v).astype(float))}

    checker = {"type": "hdr", "filename": "${scene-directory}/checker.pfm", "wrap_u": "repeat", "wrap_v": "mirror",
               "transform": [{"type": "scale", "ratio": 3}, {"type": "rotate", "deg": 20}]}
    ents = [
        {"type": "geometric", "geometry": {"type": "quad", "A": [-4, -4, -1], "B": [4, -4, -1], "C": [4, 4, -1],
                                           "D": [-4, 4, -1], "tA": [0, 0], "tB": [1, 0], "tC": [1, 1], "tD": [0, 1],
                                           "transform": []},
         "material": {"type": "ideal_diffuse", "albedo": checker,
                      "normal_map": {"type": "hdr", "filename": "${scene-directory}/normal.pfm", "wrap_u": "repeat",
                                     "wrap_v": "repeat"}}},
        {"type": "geometric", "geometry": {"type": "sphere", "radius": 0.7,
                                           "transform": [{"type": "translate", "offset": [-1.2, 0.3, -0.3]}]},
         "material": {"type": "disney", "base_color": const([0.8, 0.8, 0.9]), "metallic": const(0),
                      "roughness": const(0.3), "transmission": const(0.8), "ior": const(1.45)}},
        {"type": "geometric", "geometry": {"type": "double_sided",
                                           "internal": {"type": "disk", "radius": 0.6,
                                                        "transform": [{"type": "translate", "offset": [1.2, 0.6, 0]},
                                                                      {"type": "rotate_x", "deg": 70}]}},
         "material": {"type": "disney", "base_color": const([0.7, 0.3, 0.2]), "metallic": const(0.3),
                      "roughness": const(0.5), "clearcoat": const(0.8), "sheen": const(0.6),
                      "sheen_tint": const(0.5), "anisotropic": const(0.6), "specular_tint": const(0.4)}},
        {"type": "geometric", "geometry": {"type": "triangle", "A": [-0.5, 0, 0], "B": [0.5, 0, 0], "C": [0, 0, 0.9],
                                           "tA": [0, 0], "tB": [1, 0], "tC": [0.5, 1],
                                           "transform": [{"type": "translate", "offset": [0.2, 1.2, -1]},
                                                         {"type": "rotate_z", "deg": 15}]},
         "material": {"type": "ideal_diffuse", "albedo": checker}},
        {"type": "geometric", "geometry": {"type": "transform_wrapper", "transform": [{"type": "translate", "offset": [0, -0.6, -0.55]}],
                                           "internal": {"type": "transform_wrapper",
                                                        "transform": [{"type": "rotate", "axis": [1, 1, 0], "deg": 30}],
                                                        "internal": {"type": "triangle_bvh",
                                                                     "filename": "${scene-directory}/box.bm",
                                                                     "transform": []}}},
         "material": {"type": "ideal_diffuse", "albedo": const([0.3, 0.6, 0.4])}},
        {"type": "geometric", "geometry": {"type": "sphere", "radius": 0.25,
                                           "transform": [{"type": "translate", "offset": [0.5, -0.3, 1.6]}]},
         "material": {"type": "ideal_black"}, "emit_radiance": [6, 5, 4]},
        {"type": "geometric", "geometry": {"type": "disk", "radius": 0.4,
                                           "transform": [{"type": "translate", "offset": [-1.5, -0.5, 2.0]},
                                                         {"type": "rotate_x", "deg": 180}]},
         "material": {"type": "ideal_black"}, "emit_radiance": [3, 4, 6]},
    ]
    cfg = {"scene": {"type": "default", "entities": ents,
                     "env": {"type": "native_sky", "top": [0.4, 0.5, 0.8], "bottom": [0.1, 0.08, 0.05]}},
           "rendering": {"camera": {"type": "thin_lens", "pos": [0, -5, 1.2], "dst": [0, 0, -0.2], "up": [0, 0, 1],
                                    "fov": 50, "lens_radius": 0.05, "focal_distance": 5},
                         "width": width, "height": height,
                         "renderer": {"type": renderer, "spp": spp, "max_depth": 12, "min_depth": 3},
                         "reporter": {"type": "noout"}}}
    if gaussian:
        cfg["rendering"]["film_filter"] = {"type": "gaussian", "radius": 1.5, "alpha": 2}
    return cfg


def write_png8(path: Path, rgb: np.ndarray) -> None:
    """(H, W, 3) uint8 -> 8-bit RGB PNG, filter 0 on every row, rows top first."""
    import struct
    import zlib
    h, w, _ = rgb.shape
    raw = b"".join(b"\x00" + rgb[y].astype(np.uint8).tobytes() for y in range(h))

    def chunk(kind, body):
        return struct.pack(">I", len(body)) + kind + body + struct.pack(">I", zlib.crc32(kind + body) & 0xFFFFFFFF)

    path.write_bytes(b"\x89PNG\r\n\x1a\n" + chunk(b"IHDR", struct.pack(">IIBBBBB", w, h, 8, 2, 0, 0, 0)) +
                     chunk(b"IDAT", zlib.compress(raw)) + chunk(b"IEND", b""))


def materials_scene(tmp: Path, renderer="pt", spp=256, width=48, height=36) -> dict:
    """The wider material set in one small scene: a mirror sphere, a glass
    sphere, an anisotropic normal-mapped metal sphere, a phong box, a
    checker_board floor (phong) and an 8-bit PNG image texture on the back
    wall, lit by a sphere light and the native sky."""
    from atrc_b200.scenes import _box_mesh, write_bm, write_pfm
    rng = np.random.default_rng(91)
    write_png8(tmp / "wall.png", np.kron(rng.integers(20, 235, (4, 6, 3)), np.ones((6, 6, 1), np.int64)))
    nm = np.zeros((16, 16, 3), np.float32)
    yy, xx = np.mgrid[0:16, 0:16] / 16.0
    nm[..., 0] = 0.5 + 0.25 * np.sin(5 * xx)
    nm[..., 1] = 0.5 + 0.25 * np.cos(7 * yy)
    nm[..., 2] = 0.9
    write_pfm(tmp / "bumps.pfm", nm)
    p, n, uv = _box_mesh((0.35, 0.35, 0.35))
    write_bm(tmp / "box.bm", p, n, uv)

    def const(v):
        return {"type": "constant", "texel": list(np.atleast_1d(v).astype(float))}

    checker = {"type": "checker_board", "grid_count": 8, "color1": [0.8, 0.75, 0.7], "color2": [0.15, 0.2, 0.3]}
    ents = [
        {"type": "geometric", "geometry": {"type": "quad", "A": [-4, -4, -1], "B": [4, -4, -1], "C": [4, 4, -1],
                                           "D": [-4, 4, -1], "tA": [0, 0], "tB": [1, 0], "tC": [1, 1], "tD": [0, 1],
                                           "transform": []},
         "material": {"type": "phong", "d": checker, "s": const(0.25), "ns": const(30)}},
        {"type": "geometric", "geometry": {"type": "quad", "A": [-4, 3, -1], "B": [4, 3, -1], "C": [4, 3, 3],
                                           "D": [-4, 3, 3], "tA": [0, 0], "tB": [1, 0], "tC": [1, 1], "tD": [0, 1],
                                           "transform": []},
         "material": {"type": "ideal_diffuse",
                      "albedo": {"type": "image", "filename": "${scene-directory}/wall.png", "sample": "nearest"}}},
        {"type": "geometric", "geometry": {"type": "sphere", "radius": 0.55,
                                           "transform": [{"type": "translate", "offset": [-1.3, 0.4, -0.45]}]},
         "material": {"type": "mirror", "color_map": const([0.9, 0.85, 0.8]), "eta": const([0.2, 0.9, 1.1]),
                      "k": const([3.9, 2.4, 2.2])}},
        {"type": "geometric", "geometry": {"type": "sphere", "radius": 0.5,
                                           "transform": [{"type": "translate", "offset": [0.0, -0.4, -0.5]}]},
         "material": {"type": "glass", "ior": const(1.5), "color_reflection_map": const(1.0),
                      "color_refraction_map": const([0.9, 0.95, 1.0])}},
        {"type": "geometric", "geometry": {"type": "sphere", "radius": 0.5,
                                           "transform": [{"type": "translate", "offset": [1.3, 0.5, -0.5]}]},
         "material": {"type": "metal", "color": const([0.95, 0.8, 0.5]), "eta": const([0.2, 0.4, 1.4]),
                      "k": const([3.9, 2.4, 1.9]), "roughness": const(0.35), "anisotropic": const(0.6),
                      "normal_map": {"type": "hdr", "filename": "${scene-directory}/bumps.pfm",
                                     "wrap_u": "repeat", "wrap_v": "repeat"}}},
        {"type": "geometric", "geometry": {"type": "transform_wrapper",
                                           "transform": [{"type": "translate", "offset": [0.9, -1.0, -0.65]},
                                                         {"type": "rotate_z", "deg": 25}],
                                           "internal": {"type": "triangle_bvh", "filename": "${scene-directory}/box.bm",
                                                        "transform": []}},
         "material": {"type": "phong", "d": const([0.2, 0.5, 0.3]), "s": const([0.6, 0.6, 0.6]), "ns": const(8)}},
        {"type": "geometric", "geometry": {"type": "sphere", "radius": 0.3,
                                           "transform": [{"type": "translate", "offset": [-0.4, -0.8, 1.8]}]},
         "material": {"type": "ideal_black"}, "emit_radiance": [8, 7, 6]},
    ]
    return {"scene": {"type": "default", "entities": ents,
                      "env": {"type": "native_sky", "top": [0.4, 0.5, 0.8], "bottom": [0.1, 0.08, 0.05]}},
            "rendering": {"camera": {"type": "thin_lens", "pos": [0, -5, 1.0], "dst": [0, 0, -0.3], "up": [0, 0, 1],
                                     "fov": 50},
                          "width": width, "height": height,
                          "renderer": {"type": renderer, "spp": spp, "max_depth": 12, "min_depth": 3},
                          "reporter": {"type": "noout"}}}


def ao_slab(h=0.5, dist=1.0, spp=256, count=5, looking_up=False) -> dict:
    """`ao` between two large parallel quads h apart, seen from between them.
    A cosine-distributed ray from the floor meets the ceiling after
    h / cos(theta), so it is unblocked within `dist` iff cos(theta) < h / dist:
    the expected unblocked fraction is (h / dist)^2 (with the eps trims:
    ((h - eps) / (dist - eps))^2)."""
    def quad(z):
        return {"type": "geometric", "geometry": {"type": "quad", "A": [-100, -100, z], "B": [100, -100, z],
                                                  "C": [100, 100, z], "D": [-100, 100, z], "transform": []},
                "material": {"type": "ideal_diffuse", "albedo": {"type": "constant", "texel": [0.5]}}}
    ents = [quad(0.0), quad(h)] if not looking_up else [quad(0.0)]
    # the view stays clear of the quads' diagonal edge, where the (not
    # watertight) reference triangle test can let a ray through
    dst = [0.3, 0.1, 1] if looking_up else [0.3, 0.1, 0]
    return {"scene": {"type": "default", "entities": ents},
            "rendering": {"camera": {"type": "thin_lens", "pos": [0.3, 0.1, 0.5 * h], "dst": dst, "up": [0, 1, 0],
                                     "fov": 20},
                          "width": 8, "height": 8,
                          "renderer": {"type": "ao", "spp": spp, "ao_sample_count": count,
                                       "max_occlusion_distance": dist, "low_color": [0.1, 0.2, 0.3],
                                       "high_color": [0.9, 0.8, 0.7], "background_color": [0.05, 0.06, 0.07]},
                          "reporter": {"type": "noout"}}}


def subsurface_plane(A=(0.5, 0.5, 0.5), dmfp=(0.1, 0.1, 0.1), ior=1.3, spp=16) -> dict:
    """A large flat quad of Disney material with subsurface scattering
    (bssrdf_dmfp; A from bssrdf_A), seen straight down."""
    def const(v):
        return {"type": "constant", "texel": list(map(float, np.atleast_1d(v)))}
    mat = {"type": "disney", "base_color": const([0.8, 0.8, 0.8]), "metallic": const(0), "roughness": const(0.5),
           "transmission": const(1.0), "ior": const(ior), "bssrdf_dmfp": const(list(dmfp)), "bssrdf_A": const(list(A))}
    return {"scene": {"type": "default",
                      "entities": [{"type": "geometric",
                                    "geometry": {"type": "quad", "A": [-50, -50, 0], "B": [50, -50, 0],
                                                 "C": [50, 50, 0], "D": [-50, 50, 0], "transform": []},
                                    "material": mat}]},
            "rendering": {"camera": {"type": "thin_lens", "pos": [0.3, 0.1, 2], "dst": [0.3, 0.1, 0], "up": [0, 1, 0],
                                     "fov": 20},
                          "width": 4, "height": 4, "renderer": {"type": "pt", "spp": spp},
                          "reporter": {"type": "noout"}}}


def subsurface_scene(tmp: Path, spp=256, width=40, height=30) -> dict:
    """Disney materials with subsurface scattering on a sphere and a mesh
    box over a diffuse floor, lit by a sphere light and the native sky."""
    from atrc_b200.scenes import _box_mesh, write_bm
    p, n, uv = _box_mesh((0.45, 0.45, 0.45))
    write_bm(tmp / "sss_box.bm", p, n, uv)

    def const(v):
        return {"type": "constant", "texel": list(map(float, np.atleast_1d(v)))}

    def skin(color, A, dmfp, trans=0.8):
        return {"type": "disney", "base_color": const(color), "metallic": const(0), "roughness": const(0.4),
                "transmission": const(trans), "ior": const(1.4), "bssrdf_dmfp": const(dmfp), "bssrdf_A": const(A)}
    ents = [
        {"type": "geometric", "geometry": {"type": "quad", "A": [-4, -4, -1], "B": [4, -4, -1], "C": [4, 4, -1],
                                           "D": [-4, 4, -1], "transform": []},
         "material": {"type": "ideal_diffuse", "albedo": const([0.6, 0.6, 0.6])}},
        {"type": "geometric", "geometry": {"type": "sphere", "radius": 0.6,
                                           "transform": [{"type": "translate", "offset": [-0.7, 0.2, -0.4]}]},
         "material": skin([0.9, 0.6, 0.5], [0.9, 0.55, 0.4], [0.3, 0.15, 0.08])},
        {"type": "geometric", "geometry": {"type": "transform_wrapper",
                                           "transform": [{"type": "translate", "offset": [0.8, -0.2, -0.55]},
                                                         {"type": "rotate_z", "deg": 30}],
                                           "internal": {"type": "triangle_bvh",
                                                        "filename": "${scene-directory}/sss_box.bm",
                                                        "transform": []}},
         "material": skin([0.5, 0.7, 0.9], [0.5, 0.7, 0.9], [0.1, 0.2, 0.3], trans=1.0)},
        {"type": "geometric", "geometry": {"type": "sphere", "radius": 0.3,
                                           "transform": [{"type": "translate", "offset": [0.2, -1.0, 1.6]}]},
         "material": {"type": "ideal_black"}, "emit_radiance": [10, 9, 8]},
    ]
    return {"scene": {"type": "default", "entities": ents,
                      "env": {"type": "native_sky", "top": [0.3, 0.35, 0.5], "bottom": [0.05, 0.05, 0.05]}},
            "rendering": {"camera": {"type": "thin_lens", "pos": [0, -4.5, 1.2], "dst": [0, 0, -0.4], "up": [0, 0, 1],
                                     "fov": 40},
                          "width": width, "height": height,
                          "renderer": {"type": "pt", "spp": spp, "max_depth": 10, "min_depth": 3},
                          "reporter": {"type": "noout"}}}


def solid_image_scene(tmp: Path, spp=256, width=40, height=30) -> dict:
    """`solid_image` textures: a floor whose ideal-diffuse albedo reads an RGB
    3D image at the world position (scaled into the texture's unit cube), a
    glass sphere whose refraction colour does the same, and a Disney sphere
    whose base colour reads the same 3D image at (u, v, 0)."""
    rng = np.random.default_rng(5)
    grid = rng.uniform(0.05, 0.95, (8, 8, 8, 3)).astype(np.float32)   # (d, h, w, rgb)
    (tmp / "solid.bin").write_bytes(np.int32([8, 8, 8]).tobytes() + grid.tobytes())
    tex3d = {"type": "image3d", "format": "spec", "binary_filename": "${scene-directory}/solid.bin",
             "sample": "nearest", "wrap_u": "repeat", "wrap_v": "repeat", "wrap_w": "repeat",
             "transform": [{"type": "scale", "ratio": 0.25}, {"type": "translate", "offset": [4, 4, 4]}]}
    solid = {"type": "solid_image", "tex3d": tex3d}
    plain = {"type": "solid_image", "tex3d": dict(tex3d, transform=[])}

    def const(v):
        return {"type": "constant", "texel": list(map(float, np.atleast_1d(v)))}
    ents = [
        {"type": "geometric", "geometry": {"type": "quad", "A": [-4, -4, -1], "B": [4, -4, -1], "C": [4, 4, -1],
                                           "D": [-4, 4, -1], "transform": []},
         "material": {"type": "ideal_diffuse", "albedo": solid}},
        {"type": "geometric", "geometry": {"type": "sphere", "radius": 0.6,
                                           "transform": [{"type": "translate", "offset": [-0.8, 0.3, -0.4]}]},
         "material": {"type": "disney", "base_color": plain, "metallic": const(0), "roughness": const(0.5)}},
        {"type": "geometric", "geometry": {"type": "sphere", "radius": 0.5,
                                           "transform": [{"type": "translate", "offset": [0.8, -0.2, -0.5]}]},
         "material": {"type": "glass", "ior": const(1.5), "color_reflection_map": const(0.9),
                      "color_refraction_map": solid}},
        {"type": "geometric", "geometry": {"type": "sphere", "radius": 0.3,
                                           "transform": [{"type": "translate", "offset": [0.2, -1.0, 1.6]}]},
         "material": {"type": "ideal_black"}, "emit_radiance": [10, 9, 8]},
    ]
    return {"scene": {"type": "default", "entities": ents,
                      "env": {"type": "native_sky", "top": [0.3, 0.35, 0.5], "bottom": [0.05, 0.05, 0.05]}},
            "rendering": {"camera": {"type": "thin_lens", "pos": [0, -4.5, 1.2], "dst": [0, 0, -0.4], "up": [0, 0, 1],
                                     "fov": 40},
                          "width": width, "height": height,
                          "renderer": {"type": "pt", "spp": spp, "max_depth": 10, "min_depth": 3},
                          "reporter": {"type": "noout"}}}
