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
