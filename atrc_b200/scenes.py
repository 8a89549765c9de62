"""Seeded synthetic scenes in the Atrc JSON format.

The reference publishes no benchmark scenes (its example assets are not part
of the checkout), so the workloads are generated: a Cornell box, a 2.1M
triangle instanced scene with Disney materials under an importance-sampled
procedural sky, and a participating-media scene.  Every generator writes a
reference-format JSON file plus its assets (``.bm`` meshes in the layout of
src/factory/src/utility/bin_mesh.cpp, ``.pfm`` float environment maps, ``.bin``
density grids in the layout of src/factory/src/utility/texture3d_loader.cpp)
and rounds every float written into JSON to 6 decimals, matching the
reference's std::to_string round trip of JSON numbers.
"""
from __future__ import annotations

import json
import math
import os
from pathlib import Path

import numpy as np

__all__ = ["cornell_box", "instanced_disney", "media_scene", "indoor_room", "write_bm", "write_pfm", "write_grid",
           "icosphere", "heightfield", "cache_dir", "SCENES"]


def r6(x) -> float:
    return float(f"{float(x):.6f}")


def v3(a) -> list:
    return [r6(a[0]), r6(a[1]), r6(a[2])]


def cache_dir() -> Path:
    d = Path(os.environ.get("ATRC_SCENE_CACHE", "/tmp/atrc_scenes"))
    d.mkdir(parents=True, exist_ok=True)
    return d


# ------------------------------------------------------------------ writers
def write_bm(path: Path, pos: np.ndarray, nor: np.ndarray, uv: np.ndarray) -> None:
    """pos, nor: (T, 3, 3) float32; uv: (T, 3, 2)."""
    t = pos.shape[0]
    data = np.concatenate([pos, nor, uv], axis=2).astype(np.float32)  # (T, 3, 8)
    with open(path, "wb") as f:
        f.write(np.uint64(t).tobytes())
        f.write(np.ascontiguousarray(data).tobytes())


def write_pfm(path: Path, rgb: np.ndarray) -> None:
    """rgb: (H, W, 3), row 0 = top (v = 0).  PFM stores the bottom row first."""
    h, w, _ = rgb.shape
    with open(path, "wb") as f:
        f.write(f"PF\n{w} {h}\n-1.0\n".encode())
        f.write(np.ascontiguousarray(rgb[::-1].astype("<f4")).tobytes())


def write_grid(path: Path, grid: np.ndarray) -> None:
    """grid: (D, H, W) float32, z-major (texture3d_loader.cpp:11-37)."""
    d, h, w = grid.shape
    with open(path, "wb") as f:
        f.write(np.array([w, h, d], dtype="<i4").tobytes())
        f.write(np.ascontiguousarray(grid.astype("<f4")).tobytes())


# -------------------------------------------------------------------- noise
def _hash3(ix, iy, iz, seed):
    h = (ix.astype(np.int64) * 73856093) ^ (iy.astype(np.int64) * 19349663) ^ (iz.astype(np.int64) * 83492791) ^ (
        seed * 2654435761)
    h = (h ^ (h >> 13)) * 1274126177
    h = h ^ (h >> 16)
    return (h & 0xFFFFFF).astype(np.float64) / float(0xFFFFFF)


def value_noise3(p: np.ndarray, seed: int) -> np.ndarray:
    """Trilinearly interpolated lattice value noise in [0, 1], smoothstep fade."""
    fl = np.floor(p)
    f = p - fl
    f = f * f * (3 - 2 * f)
    i = fl.astype(np.int64)
    out = 0.0
    for dx in (0, 1):
        for dy in (0, 1):
            for dz in (0, 1):
                w = (f[..., 0] if dx else 1 - f[..., 0]) * (f[..., 1] if dy else 1 - f[..., 1]) * (
                    f[..., 2] if dz else 1 - f[..., 2])
                out = out + w * _hash3(i[..., 0] + dx, i[..., 1] + dy, i[..., 2] + dz, seed)
    return out


def fbm3(p: np.ndarray, seed: int, octaves: int = 5, freq: float = 1.0) -> np.ndarray:
    """Fractional Brownian motion of value noise, in about [-1, 1]."""
    amp, total, norm = 1.0, 0.0, 0.0
    for o in range(octaves):
        total = total + amp * (value_noise3(p * freq * (2 ** o), seed + 17 * o) * 2 - 1)
        norm += amp
        amp *= 0.5
    return total / norm


# ------------------------------------------------------------------- meshes
def _normals_from_faces(v: np.ndarray, f: np.ndarray) -> np.ndarray:
    fn = np.cross(v[f[:, 1]] - v[f[:, 0]], v[f[:, 2]] - v[f[:, 0]])
    vn = np.zeros_like(v)
    for k in range(3):
        np.add.at(vn, f[:, k], fn)
    ln = np.linalg.norm(vn, axis=1, keepdims=True)
    return vn / np.where(ln > 0, ln, 1)


def _icosahedron() -> tuple:
    t = (1 + 5 ** 0.5) / 2
    v = np.array([[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0], [0, -1, t], [0, 1, t], [0, -1, -t], [0, 1, -t],
                  [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]], dtype=np.float64)
    f = np.array([[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11], [1, 5, 9], [5, 11, 4], [11, 10, 2],
                  [10, 7, 6], [7, 1, 8], [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9], [4, 9, 5],
                  [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1]], dtype=np.int64)
    return v / np.linalg.norm(v, axis=1, keepdims=True), f


def _displace(v: np.ndarray, f: np.ndarray, seed: int, amplitude: float) -> tuple:
    disp = 1 + amplitude * fbm3(v * 2.0, seed, 5)
    v = v * disp[:, None]
    n = _normals_from_faces(v, f)
    d = v / np.linalg.norm(v, axis=1, keepdims=True)
    uv = np.stack([0.5 + np.arctan2(d[:, 1], d[:, 0]) / (2 * np.pi), np.arccos(np.clip(d[:, 2], -1, 1)) / np.pi], 1)
    return v.astype(np.float32), n.astype(np.float32), uv.astype(np.float32), f


def geodesic_sphere(freq: int, seed: int, amplitude: float = 0.05) -> tuple:
    """Unit sphere from the icosahedron with every face cut into freq^2
    triangles (class-I geodesic subdivision, 20 freq^2 triangles: 200,000 for
    freq 100), radially displaced by 5-octave fBm."""
    v0, f0 = _icosahedron()
    n = int(freq)
    # barycentric lattice of one face: point (i, j) = A + (B - A) i/n + (C - A) j/n
    ii, jj = np.meshgrid(np.arange(n + 1), np.arange(n + 1), indexing="ij")
    keep = ii + jj <= n
    ii, jj = ii[keep], jj[keep]
    lattice = -np.ones((n + 1, n + 1), np.int64)
    lattice[ii, jj] = np.arange(len(ii))
    up = [(i, j) for i in range(n) for j in range(n - i)]
    down = [(i, j) for i in range(n - 1) for j in range(n - 1 - i)]
    ui, uj = np.array(up).T
    tri = [np.stack([lattice[ui, uj], lattice[ui + 1, uj], lattice[ui, uj + 1]], 1)]
    if down:
        di, dj = np.array(down).T
        tri.append(np.stack([lattice[di + 1, dj], lattice[di + 1, dj + 1], lattice[di, dj + 1]], 1))
    local = np.concatenate(tri)
    pts, faces = [], []
    for k, (a, b, c) in enumerate(f0):
        A, B, C = v0[a], v0[b], v0[c]
        P = A + np.outer(ii / n, B - A) + np.outer(jj / n, C - A)
        pts.append(P / np.linalg.norm(P, axis=1, keepdims=True))
        faces.append(local + k * len(ii))
    pts = np.concatenate(pts)
    faces = np.concatenate(faces)
    # points on shared edges and corners are computed once per face: merge them
    _, first, inv = np.unique(np.round(pts * 1e7).astype(np.int64), axis=0, return_index=True, return_inverse=True)
    return _displace(pts[first], inv.reshape(-1)[faces], seed, amplitude)


def icosphere(level: int, seed: int, amplitude: float = 0.05) -> tuple:
    """Unit icosphere subdivided `level` times, radially displaced by 5-octave fBm."""
    v, f = _icosahedron()
    for _ in range(level):
        e = np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]])
        e.sort(axis=1)
        key = e[:, 0] * (len(v) + 1) + e[:, 1]
        uniq, inv = np.unique(key, return_inverse=True)
        a = uniq // (len(v) + 1)
        b = uniq % (len(v) + 1)
        mid = v[a] + v[b]
        mid /= np.linalg.norm(mid, axis=1, keepdims=True)
        base = len(v)
        v = np.concatenate([v, mid])
        nf = len(f)
        m01, m12, m20 = inv[:nf] + base, inv[nf:2 * nf] + base, inv[2 * nf:] + base
        f = np.concatenate([np.stack([f[:, 0], m01, m20], 1), np.stack([f[:, 1], m12, m01], 1),
                            np.stack([f[:, 2], m20, m12], 1), np.stack([m01, m12, m20], 1)])
    return _displace(v, f, seed, amplitude)


def heightfield(res: int, seed: int, amplitude: float = 0.15) -> tuple:
    """res x res vertices on [-1, 1]^2 (z up), heights from 5-octave fBm."""
    xs = np.linspace(-1, 1, res)
    X, Y = np.meshgrid(xs, xs, indexing="xy")
    P = np.stack([X * 2, Y * 2, np.full_like(X, 0.37)], -1)
    Z = amplitude * fbm3(P, seed, 5)
    v = np.stack([X, Y, Z], -1).reshape(-1, 3)
    i = np.arange(res - 1)
    I, J = np.meshgrid(i, i, indexing="xy")
    a = (J * res + I).ravel()
    b, c, d = a + 1, a + res + 1, a + res
    f = np.concatenate([np.stack([a, b, c], 1), np.stack([a, c, d], 1)])
    n = _normals_from_faces(v, f)
    uv = np.stack([(X.ravel() + 1) / 2, (Y.ravel() + 1) / 2], 1)
    return v.astype(np.float32), n.astype(np.float32), uv.astype(np.float32), f


def _mesh_to_bm(path: Path, mesh) -> int:
    v, n, uv, f = mesh
    write_bm(path, v[f], n[f], uv[f])
    return len(f)


def _box_mesh(half: tuple) -> tuple:
    """12-triangle axis-aligned box centred at the origin, outward faces."""
    hx, hy, hz = half
    c = np.array([[-hx, -hy, -hz], [hx, -hy, -hz], [hx, hy, -hz], [-hx, hy, -hz],
                  [-hx, -hy, hz], [hx, -hy, hz], [hx, hy, hz], [-hx, hy, hz]], dtype=np.float32)
    quads = [(0, 3, 2, 1), (4, 5, 6, 7), (0, 1, 5, 4), (2, 3, 7, 6), (1, 2, 6, 5), (0, 4, 7, 3)]
    pos, nor, uv = [], [], []
    for q in quads:
        a, b, cc, d = (c[k] for k in q)
        nrm = np.cross(b - a, cc - a)
        nrm = nrm / np.linalg.norm(nrm)
        for tri in ((a, b, cc), (a, cc, d)):
            pos.append(np.stack(tri))
            nor.append(np.stack([nrm] * 3))
            uv.append(np.array([[0, 0], [1, 0], [1, 1]], dtype=np.float32))
    return np.array(pos, np.float32), np.array(nor, np.float32), np.array(uv, np.float32)


def _const(v) -> dict:
    return {"type": "constant", "texel": v3(v) if np.ndim(v) else [r6(v)]}


# ----------------------------------------------------------- Cornell (cfg 0)
def cornell_box(out_dir: Path | None = None, seed: int = 1000, width: int = 256, height: int = 256, spp: int = 64,
                renderer: str = "pt", max_depth: int = 8, min_depth: int = 2, subsurface: bool = False) -> Path:
    """Plain pt on a seeded Cornell box: 5 quad walls of [-1,1]^3, two 12-triangle
    boxes rotated by U[0, 30] degrees about y, a 0.5x0.5 quad light at the
    ceiling with radiance (17, 12, 4), Lambertian albedos U[0.1, 0.8]^3 with a
    red and a green wall, pinhole camera with 40 degree FOV, box filter.
    With `subsurface` the two boxes are Disney materials with subsurface
    scattering instead (base colour and bssrdf_A = the box's drawn albedo,
    transmission 0.8, mean free paths of a few hundredths of the box)."""
    out = Path(out_dir) if out_dir else cache_dir() / f"cornell_{seed}{'_sss' if subsurface else ''}"
    out.mkdir(parents=True, exist_ok=True)
    rng = np.random.default_rng(seed)
    alb = lambda: v3(rng.uniform(0.1, 0.8, 3))  # noqa: E731
    walls = [  # (A, B, C, D) with normals facing the box interior, albedo
        ([-1, -1, 1], [1, -1, 1], [1, -1, -1], [-1, -1, -1], alb()),   # floor (normal +y)
        ([-1, 1, -1], [1, 1, -1], [1, 1, 1], [-1, 1, 1], alb()),       # ceiling (normal -y)
        ([-1, -1, -1], [1, -1, -1], [1, 1, -1], [-1, 1, -1], alb()),   # back (normal +z)
        ([-1, -1, 1], [-1, -1, -1], [-1, 1, -1], [-1, 1, 1], [0.63, 0.065, 0.05]),  # left, red (+x)
        ([1, -1, -1], [1, -1, 1], [1, 1, 1], [1, 1, -1], [0.14, 0.45, 0.091]),     # right, green (-x)
    ]
    ents = []
    for a, b, c, d, al in walls:
        ents.append({"type": "geometric",
                     "geometry": {"type": "quad", "A": v3(a), "B": v3(b), "C": v3(c), "D": v3(d), "transform": []},
                     "material": {"type": "ideal_diffuse", "albedo": _const(al)}})
    specs = [((0.3, 0.6, 0.3), (-0.4, -0.4, -0.3)), ((0.3, 0.3, 0.3), (0.4, -0.7, 0.3))]
    for k, (half, pos) in enumerate(specs):
        p, n, uv = _box_mesh(half)
        fn = out / f"box{k}.bm"
        write_bm(fn, p, n, uv)
        deg = r6(rng.uniform(0, 30))
        albedo = rng.uniform(0.1, 0.8, 3)
        if subsurface:
            mat = {"type": "disney", "base_color": _const(albedo), "metallic": _const(0.0),
                   "roughness": _const(0.4), "transmission": _const(0.8), "ior": _const(1.4),
                   "bssrdf_dmfp": _const([0.06, 0.03, 0.02]), "bssrdf_A": _const(albedo)}
        else:
            mat = {"type": "ideal_diffuse", "albedo": _const(albedo)}
        ents.append({"type": "geometric",
                     "geometry": {"type": "triangle_bvh", "filename": "${scene-directory}/" + fn.name,
                                  "transform": [{"type": "translate", "offset": v3(pos)},
                                                {"type": "rotate_y", "deg": deg}]},
                     "material": mat})
    ents.append({"type": "geometric",
                 "geometry": {"type": "quad", "A": [-0.25, 0.999, -0.25], "B": [0.25, 0.999, -0.25],
                              "C": [0.25, 0.999, 0.25], "D": [-0.25, 0.999, 0.25], "transform": []},
                 "material": {"type": "ideal_black"}, "emit_radiance": [17, 12, 4]})
    cfg = {"scene": {"type": "default", "entities": ents, "aggregate": {"type": "bvh"}},
           "rendering": {"camera": {"type": "thin_lens", "pos": [0, 0, 3.8], "dst": [0, 0, 0], "up": [0, 1, 0],
                                    "fov": 40},
                         "width": width, "height": height,
                         "renderer": {"type": renderer, "spp": spp, "max_depth": max_depth, "min_depth": min_depth},
                         "reporter": {"type": "noout"},
                         "film_filter": {"type": "box", "radius": 0.5}}}
    path = out / "scene.json"
    path.write_text(json.dumps(cfg, indent=1))
    return path


# ------------------------------------------------------------------ sky map
def sky_map(width: int = 1024, height: int = 512, sun_dir=(0.3, -0.4, 0.866), sun_radius_deg: float = 0.5,
            sun_peak: float = 5e4) -> np.ndarray:
    """Procedural z-up sky: gradient plus a sun lobe (row 0 = zenith, v = theta / pi)."""
    v = (np.arange(height) + 0.5) / height
    u = (np.arange(width) + 0.5) / width
    theta = v * np.pi
    phi = u * 2 * np.pi
    T, P = np.meshgrid(theta, phi, indexing="ij")
    d = np.stack([np.sin(T) * np.cos(P), np.sin(T) * np.sin(P), np.cos(T)], -1)
    z = d[..., 2]
    top, horizon, ground = np.array([0.25, 0.45, 1.0]), np.array([0.9, 0.85, 0.8]), np.array([0.18, 0.15, 0.12])
    t = np.clip(z, 0, 1)[..., None]
    sky = np.where(z[..., None] >= 0, horizon * (1 - t) + top * t, ground + (horizon - ground) * np.exp(8 * z)[..., None])
    s = np.asarray(sun_dir, np.float64)
    s /= np.linalg.norm(s)
    ang = np.arccos(np.clip(d @ s, -1, 1))
    r = math.radians(sun_radius_deg)
    sun = sun_peak * np.exp(-(ang / r) ** 2 * 2.0)[..., None] * np.array([1.0, 0.92, 0.82])
    return (sky + sun).astype(np.float32)


def _rand_rotation(rng) -> np.ndarray:
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    a, b, c, d = q
    return np.array([[a * a + b * b - c * c - d * d, 2 * (b * c - a * d), 2 * (b * d + a * c)],
                     [2 * (b * c + a * d), a * a - b * b + c * c - d * d, 2 * (c * d - a * b)],
                     [2 * (b * d - a * c), 2 * (c * d + a * b), a * a - b * b - c * c + d * d]])


# --------------------------------------------------- instanced Disney (cfg 1)
def instanced_disney(out_dir: Path | None = None, seed: int = 1001, width: int = 1920, height: int = 1080,
                     spp: int = 256, max_depth: int = 16, renderer: str = "pt_cuda", ico_level: int = 7,
                     hf_res: int = 1024, instances: int = 64) -> Path:
    """64 instances (transform_wrapper + reference) of 4 seeded meshes -- three
    level-7 fBm-displaced icospheres (327,680 triangles each) and a 1024x1024
    heightfield (2,093,058 triangles) -- with uniform random translations in
    [-20, 20]^3, scales in [0.5, 3] and rotations; Disney materials with
    roughness U[0.05, 1], metallic Bernoulli(0.3), base colour U[0.05, 0.95]^3;
    an importance-sampled 1024x512 procedural sky with a 0.5 degree sun of
    peak 5e4."""
    tag = f"inst_{seed}_{ico_level}_{hf_res}_{instances}"
    out = Path(out_dir) if out_dir else cache_dir() / tag
    out.mkdir(parents=True, exist_ok=True)
    rng = np.random.default_rng(seed)
    mesh_files = []
    for k in range(3):
        fn = out / f"ico{k}.bm"
        if not fn.exists():
            _mesh_to_bm(fn, icosphere(ico_level, seed + 11 * k))
        mesh_files.append(fn.name)
    fn = out / "heightfield.bm"
    if not fn.exists():
        _mesh_to_bm(fn, heightfield(hf_res, seed + 97))
    mesh_files.append(fn.name)
    env = out / "sky.pfm"
    if not env.exists():
        write_pfm(env, sky_map())
    meshes = {f"mesh{k}": {"type": "triangle_bvh", "filename": "${scene-directory}/" + m, "transform": []}
              for k, m in enumerate(mesh_files)}
    ents = []
    for i in range(instances):
        m = int(rng.integers(0, 4))
        tr = rng.uniform(-20, 20, 3)
        sc = rng.uniform(0.5, 3)
        R = _rand_rotation(rng)
        mat = {"type": "disney",
               "base_color": _const(rng.uniform(0.05, 0.95, 3)),
               "metallic": _const(1.0 if rng.random() < 0.3 else 0.0),
               "roughness": _const(rng.uniform(0.05, 1.0))}
        ents.append({"type": "geometric",
                     "geometry": {"type": "transform_wrapper",
                                  "internal": {"type": "reference", "name": ["meshes", f"mesh{m}"]},
                                  "transform": [{"type": "translate", "offset": v3(tr)},
                                                {"type": "mat3", "row_major": [r6(x) for x in R.ravel()]},
                                                {"type": "scale", "ratio": r6(sc)}]},
                     "material": mat})
    cfg = {"scene": {"type": "default", "entities": ents, "aggregate": {"type": "bvh"}, "meshes": meshes,
                     "env": {"type": "ibl", "tex": {"type": "hdr", "filename": "${scene-directory}/sky.pfm"}}},
           "rendering": {"camera": {"type": "thin_lens", "pos": [0, -27, 5], "dst": [0, 0, 0], "up": [0, 0, 1],
                                    "fov": 62},
                         "width": width, "height": height,
                         "renderer": {"type": renderer, "spp": spp, "max_depth": max_depth},
                         "reporter": {"type": "noout"}}}
    path = out / "scene.json"
    path.write_text(json.dumps(cfg))
    return path


# ----------------------------------------------------------- media (cfg 2)
def media_scene(out_dir: Path | None = None, seed: int = 1002, width: int = 1024, height: int = 1024, spp: int = 512,
                max_depth: int = 32, renderer: str = "pt_cuda", grid_res: int = 128, sphere_level: int | None = None,
                sphere_freq: int = 100) -> Path:
    """A homogeneous box medium (sigma_a 0.05, sigma_s 0.5, g 0.6) and a 128^3
    fBm density grid scaled to sigma_t in [0, 8] (albedo 0.9, delta tracking)
    enclosing a displaced sphere (a frequency-100 geodesic sphere of 200,000
    triangles by default; `sphere_level` selects a recursively subdivided
    icosphere instead), two quad lights and the procedural sky.
    The medium boxes float 0.02 above the floor: coplanar boundaries would make
    the medium of the segments below them depend on how ties between equal
    hit distances are broken, which the reference leaves to traversal order."""
    sphere_tag = f"l{sphere_level}" if sphere_level is not None else f"f{sphere_freq}"
    out = Path(out_dir) if out_dir else cache_dir() / f"media_{seed}_{grid_res}_{sphere_tag}"
    out.mkdir(parents=True, exist_ok=True)
    rng = np.random.default_rng(seed)
    env = out / "sky.pfm"
    if not env.exists():
        write_pfm(env, sky_map())
    g = out / "density.bin"
    if not g.exists():
        xs = (np.arange(grid_res) + 0.5) / grid_res
        Z, Y, X = np.meshgrid(xs, xs, xs, indexing="ij")
        d = fbm3(np.stack([X, Y, Z], -1) * 4, seed, 5)
        d = (d - d.min()) / (d.max() - d.min()) * 8.0
        write_grid(g, d.astype(np.float32))
    sph = out / f"sphere_{sphere_tag}.bm"
    if not sph.exists():
        mesh = icosphere(sphere_level, seed + 5, 0.05) if sphere_level is not None else \
            geodesic_sphere(sphere_freq, seed + 5, 0.05)
        _mesh_to_bm(sph, mesh)
    unit_box = lambda: {"type": "triangle_bvh", "filename": "${scene-directory}/unitbox.bm"}  # noqa: E731
    p, n, uv = _box_mesh((0.5, 0.5, 0.5))
    write_bm(out / "unitbox.bm", p + 0.5, n, uv)  # [0,1]^3, outward
    ents = [
        {"type": "geometric", "geometry": {"type": "quad", "A": [-6, -6, -1], "B": [6, -6, -1], "C": [6, 6, -1],
                                           "D": [-6, 6, -1], "transform": []},
         "material": {"type": "ideal_diffuse", "albedo": _const([0.6, 0.6, 0.6])}},
        {"type": "geometric", "geometry": {**unit_box(), "transform": [{"type": "translate", "offset": [-2.6, -1, -0.98]},
                                                                        {"type": "scale", "ratio": 2}]},
         "material": {"type": "invisible_surface"},
         "med_in": {"type": "homogeneous", "sigma_a": [0.05], "sigma_s": [0.5], "g": 0.6}},
        {"type": "geometric", "geometry": {**unit_box(), "transform": [{"type": "translate", "offset": [0.4, -1.2, -0.98]},
                                                                        {"type": "scale", "ratio": 2.4}]},
         "material": {"type": "invisible_surface"},
         "med_in": {"type": "heterogeneous",
                    "transform": [{"type": "translate", "offset": [0.4, -1.2, -0.98]}, {"type": "scale", "ratio": 2.4}],
                    "density": {"type": "image3d", "format": "real", "binary_filename": "${scene-directory}/density.bin"},
                    "albedo": {"type": "constant", "texel": [0.9]},
                    "g": {"type": "constant", "texel": [0.0]}}},
        {"type": "geometric", "geometry": {"type": "triangle_bvh", "filename": f"${{scene-directory}}/{sph.name}",
                                           "transform": [{"type": "translate", "offset": [1.6, 0, 0.2]},
                                                         {"type": "scale", "ratio": 0.6}]},
         "material": {"type": "disney", "base_color": _const([0.8, 0.3, 0.2]), "metallic": _const(0.0),
                      "roughness": _const(0.4)}},
        {"type": "geometric", "geometry": {"type": "quad", "A": [-1, -1, 4], "B": [-1, 1, 4], "C": [1, 1, 4],
                                           "D": [1, -1, 4], "transform": [{"type": "translate", "offset": [-3, 0, 0]}]},
         "material": {"type": "ideal_black"}, "emit_radiance": [8, 8, 8]},
        {"type": "geometric", "geometry": {"type": "quad", "A": [-0.5, -0.5, 3], "B": [-0.5, 0.5, 3], "C": [0.5, 0.5, 3],
                                           "D": [0.5, -0.5, 3], "transform": [{"type": "translate", "offset": [3, 1, 0]}]},
         "material": {"type": "ideal_black"}, "emit_radiance": [20, 16, 10]},
    ]
    cfg = {"scene": {"type": "default", "entities": ents, "aggregate": {"type": "bvh"},
                     "env": {"type": "ibl", "tex": {"type": "hdr", "filename": "${scene-directory}/sky.pfm"}}},
           "rendering": {"camera": {"type": "thin_lens", "pos": [0, -9, 3], "dst": [0, 0, 0], "up": [0, 0, 1], "fov": 45},
                         "width": width, "height": height,
                         "renderer": {"type": renderer, "spp": spp, "max_depth": max_depth},
                         "reporter": {"type": "noout"}}}
    path = out / "scene.json"
    path.write_text(json.dumps(cfg))
    return path


# ------------------------------------------------------- indoor room (cfg 3)
def _wall_grid(origin, u_vec, v_vec, nu: int, nv: int, normal, hole=None) -> tuple:
    """nu x nv cells of two triangles spanning origin + [0,1] u_vec + [0,1] v_vec,
    shading normal `normal`; cells whose centre lies in hole = (u0, u1, v0, v1)
    (fractions of the wall) are left out.  Returns (pos, nor, uv) per triangle."""
    o, U, V = (np.asarray(x, np.float64) for x in (origin, u_vec, v_vec))
    iu, iv = np.meshgrid(np.arange(nu), np.arange(nv), indexing="xy")
    iu, iv = iu.ravel(), iv.ravel()
    if hole is not None:
        cu, cv = (iu + 0.5) / nu, (iv + 0.5) / nv
        keep = ~((cu > hole[0]) & (cu < hole[1]) & (cv > hole[2]) & (cv < hole[3]))
        iu, iv = iu[keep], iv[keep]
    u0, u1, v0, v1 = iu / nu, (iu + 1) / nu, iv / nv, (iv + 1) / nv
    p = lambda a, b: o + a[:, None] * U + b[:, None] * V  # noqa: E731
    a, b, c, d = p(u0, v0), p(u1, v0), p(u1, v1), p(u0, v1)
    pos = np.concatenate([np.stack([a, b, c], 1), np.stack([a, c, d], 1)]).astype(np.float32)
    n = len(iu)
    nor = np.broadcast_to(np.asarray(normal, np.float32), (2 * n, 3, 3)).copy()
    uvs = np.stack([np.stack([u0, v0], 1), np.stack([u1, v0], 1), np.stack([u1, v1], 1)], 1)
    uvs2 = np.stack([np.stack([u0, v0], 1), np.stack([u1, v1], 1), np.stack([u0, v1], 1)], 1)
    return pos, nor, np.concatenate([uvs, uvs2]).astype(np.float32)


def indoor_room(out_dir: Path | None = None, seed: int = 1003, width: int = 1280, height: int = 720, spp: int = 64,
                max_depth: int = 16, renderer: str = "pt_cuda", cell: float = 0.1, objects: int = 10,
                object_level: int = 5) -> Path:
    """A closed 20 x 12 x 8 room (x in [-10, 10], y in [-6, 6], z in [0, 8])
    lit only through a 1 x 1 window in the y = -6 wall (x in [-0.5, 0.5],
    z in [4, 5]) by the instanced workload's sky, whose 0.5 degree sun shines
    through the window onto the floor.  The walls are 0.1 m grids (198,200
    triangles) and ten fBm-displaced level-5 icospheres (20,480 triangles each)
    stand on the floor: 403,000 triangles.  Every surface is Disney with
    roughness U[0.02, 0.6], base colour U[0.1, 0.9]^3 and metallic
    Bernoulli(0.2); 1280x720, max depth 16."""
    tag = f"room_{seed}_{cell}_{objects}_{object_level}"
    out = Path(out_dir) if out_dir else cache_dir() / tag
    out.mkdir(parents=True, exist_ok=True)
    rng = np.random.default_rng(seed)
    X0, X1, Y0, Y1, Z0, Z1 = -10.0, 10.0, -6.0, 6.0, 0.0, 8.0
    nx, ny, nz = int(round((X1 - X0) / cell)), int(round((Y1 - Y0) / cell)), int(round((Z1 - Z0) / cell))
    # window: x in [-0.5, 0.5], z in [4, 5] of the y = Y0 wall (fractions of that wall)
    hole = ((-0.5 - X0) / (X1 - X0), (0.5 - X0) / (X1 - X0), (4.0 - Z0) / (Z1 - Z0), (5.0 - Z0) / (Z1 - Z0))
    walls = {  # name: (origin, u, v, nu, nv, inward normal, hole)
        "floor": ((X0, Y0, Z0), (X1 - X0, 0, 0), (0, Y1 - Y0, 0), nx, ny, (0, 0, 1), None),
        "ceiling": ((X0, Y0, Z1), (0, Y1 - Y0, 0), (X1 - X0, 0, 0), ny, nx, (0, 0, -1), None),
        "wall_south": ((X0, Y0, Z0), (X1 - X0, 0, 0), (0, 0, Z1 - Z0), nx, nz, (0, 1, 0), hole),
        "wall_north": ((X0, Y1, Z0), (0, 0, Z1 - Z0), (X1 - X0, 0, 0), nz, nx, (0, -1, 0), None),
        "wall_west": ((X0, Y0, Z0), (0, 0, Z1 - Z0), (0, Y1 - Y0, 0), nz, ny, (1, 0, 0), None),
        "wall_east": ((X1, Y0, Z0), (0, Y1 - Y0, 0), (0, 0, Z1 - Z0), ny, nz, (-1, 0, 0), None),
    }
    if hole is not None and (nx * hole[0]) % 1 or (nz * hole[2]) % 1:
        raise ValueError("the window must align with the wall grid")

    def disney():
        return {"type": "disney", "base_color": _const(rng.uniform(0.1, 0.9, 3)),
                "metallic": _const(1.0 if rng.random() < 0.2 else 0.0),
                "roughness": _const(rng.uniform(0.02, 0.6))}
    ents = []
    for name, (o, u, v, nu, nv, nrm, hl) in walls.items():
        fn = out / f"{name}.bm"
        if not fn.exists():
            write_bm(fn, *_wall_grid(o, u, v, nu, nv, nrm, hl))
        ents.append({"type": "geometric", "geometry": {"type": "triangle_bvh", "filename": "${scene-directory}/" + fn.name,
                                                      "transform": []}, "material": disney()})
    for k in range(objects):
        fn = out / f"object{k}.bm"
        if not fn.exists():
            _mesh_to_bm(fn, icosphere(object_level, seed + 31 * k, amplitude=0.08))
        r = rng.uniform(0.5, 1.2)
        c = (rng.uniform(X0 + 1.5, X1 - 1.5), rng.uniform(Y0 + 1.5, Y1 - 1.5), r * 1.01)
        ents.append({"type": "geometric", "geometry": {"type": "triangle_bvh", "filename": "${scene-directory}/" + fn.name,
                                                      "transform": [{"type": "translate", "offset": v3(c)},
                                                                    {"type": "scale", "ratio": r6(r)}]},
                     "material": disney()})
    env = out / "sky.pfm"
    if not env.exists():
        s = np.array([0.25, -0.8, 0.55])
        write_pfm(env, sky_map(sun_dir=tuple(s / np.linalg.norm(s))))
    cfg = {"scene": {"type": "default", "entities": ents, "aggregate": {"type": "bvh"},
                     "env": {"type": "ibl", "tex": {"type": "hdr", "filename": "${scene-directory}/sky.pfm"}}},
           "rendering": {"camera": {"type": "thin_lens", "pos": [7, 4.5, 2.5], "dst": [-2, -2, 1.5], "up": [0, 0, 1],
                                    "fov": 70},
                         "width": width, "height": height,
                         "renderer": {"type": renderer, "spp": spp, "max_depth": max_depth, "disney_fixed": 1},
                         "reporter": {"type": "noout"}}}
    path = out / "scene.json"
    path.write_text(json.dumps(cfg))
    return path


SCENES = {"cornell": cornell_box, "instanced": instanced_disney, "media": media_scene, "room": indoor_room}
