"""The watertight intersection mode (ATRC_ISECT_WATERTIGHT): Woop, Benthin and
Wald's watertight ray-triangle test (JCGT 2(1), 2013) on the triangles' exact
vertices, beside the reference's Moller-Trumbore
(src/tracer/include/agz/tracer/utility/triangle_aux.h:9-69).

Rays from inside a closed mesh, aimed at points of its shared edges and at its
vertices, must all hit it.  Moller-Trumbore rounds alpha, beta and alpha +
beta per triangle and lets a large share of them through the seams; the
watertight test lets none through.  On the CPU the oracle shows both; on the
GPU the device's watertight traversal is compared bit for bit with the
oracle's, and a watertight render against the oracle's image."""
import json

import numpy as np
import pytest

import oracle
from atrc_b200 import RAY_DTYPE, Config, DeviceScene, Film
from atrc_b200.scenes import _mesh_to_bm, geodesic_sphere
from tests.parity import band_test, classify_closest, global_mean_z, seeded_rays

ORIGIN = np.array([0.013, -0.021, 0.007], np.float32)  # inside the sphere, off-centre


def _closed_mesh_scene(tmp_path, freq=20):
    mesh = geodesic_sphere(freq, 3, amplitude=0.05)
    _mesh_to_bm(tmp_path / "sphere.bm", mesh)
    mat = {"type": "ideal_diffuse", "albedo": {"type": "constant", "texel": [0.5]}}
    cfg = {"scene": {"type": "default", "aggregate": {"type": "bvh"}, "entities": [
        {"type": "geometric", "material": mat,
         "geometry": {"type": "triangle_bvh", "filename": "${scene-directory}/sphere.bm", "transform": []}}]},
        "rendering": {"camera": {"type": "thin_lens", "pos": [0, 0, 0], "dst": [0, 0, 1], "up": [0, 1, 0], "fov": 40},
                      "width": 8, "height": 8, "renderer": {"type": "pt_cuda", "spp": 1}}}
    (tmp_path / "scene.json").write_text(json.dumps(cfg))
    return Config.from_file(tmp_path / "scene.json"), mesh


def _seam_rays(mesh, per_edge=8, seed=0):
    """Rays from ORIGIN through points of every edge (A + s (B - A) in float)
    and through every vertex."""
    v, _, _, f = mesh
    e = np.unique(np.sort(np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]]), 1), axis=0)
    s = np.random.default_rng(seed).uniform(0, 1, (len(e), per_edge)).astype(np.float32)
    a, b = v[e[:, 0]][:, None, :], v[e[:, 1]][:, None, :]
    targets = np.concatenate([(a + s[..., None] * (b - a)).astype(np.float32).reshape(-1, 3), v])
    r = np.zeros(len(targets), RAY_DTYPE)
    r["o"] = ORIGIN
    r["d"] = (targets - ORIGIN).astype(np.float32)
    r["t_min"] = 0
    r["t_max"] = np.inf
    return r


def test_oracle_watertight_closes_mesh_seams(tmp_path):
    cfg, mesh = _closed_mesh_scene(tmp_path)
    desc, _ = cfg.rendering(0)
    ora = oracle.OracleScene(cfg.scene_desc(), desc.eps)
    rays = _seam_rays(mesh)
    for mode in ("closest", "any"):
        wt = ora.trace_rays(rays, mode, watertight=True)
        mt = ora.trace_rays(rays, mode)
        assert (wt["entity"] < 0).sum() == 0, mode
        # the reference's test leaks through the seams it is aimed at
        assert (mt["entity"] < 0).mean() > 0.01, mode


def test_oracle_watertight_agrees_with_mt_off_the_seams(tmp_path):
    cfg, mesh = _closed_mesh_scene(tmp_path)
    desc, _ = cfg.rendering(0)
    ora = oracle.OracleScene(cfg.scene_desc(), desc.eps)
    rays = seeded_rays(50_000, [-1.2] * 3, [1.2] * 3, [0.0, 0.0, -3.0], seed=5)
    wt = ora.trace_rays(rays, "closest", watertight=True)
    mt = ora.trace_rays(rays, "closest")
    same = (wt["entity"] == mt["entity"]) & (wt["prim"] == mt["prim"])
    assert same.mean() > 0.999
    hit = same & (mt["entity"] >= 0)
    assert hit.mean() > 0.3
    rel = np.abs(wt["t"][hit] - mt["t"][hit]) / np.abs(mt["t"][hit])
    # grazing hits make t ill-conditioned; the bulk agrees to float rounding
    assert np.max(rel) < 1e-4 and np.quantile(rel, 0.999) < 1e-5 and np.median(rel) < 1e-6


@pytest.mark.gpu
def test_device_watertight_closes_mesh_seams(tmp_path):
    cfg, mesh = _closed_mesh_scene(tmp_path)
    dev = DeviceScene(cfg)
    rays = _seam_rays(mesh)
    for mode in ("closest", "any"):
        wt = dev.trace_rays(rays, mode, isect=2)
        mt = dev.trace_rays(rays, mode, isect=1)
        assert (wt["entity"] < 0).sum() == 0, mode
        assert (mt["entity"] < 0).mean() > 0.01, mode


@pytest.mark.gpu
def test_device_watertight_bit_exact_with_oracle(tmp_path):
    from atrc_b200.scenes import instanced_disney
    cfg, mesh = _closed_mesh_scene(tmp_path)
    scenes = [(cfg, _seam_rays(mesh))]
    p = instanced_disney(tmp_path / "inst", ico_level=4, hf_res=128, width=64, height=36, spp=4)
    icfg = Config.from_file(p)
    idesc, _ = icfg.rendering(0)
    scenes.append((icfg, seeded_rays(500_000, [-22.0] * 3, [22.0] * 3, list(idesc.camera.pos), seed=19)))
    for cfg_k, rays in scenes:
        desc, _ = cfg_k.rendering(0)
        dev = DeviceScene(cfg_k)
        ora = oracle.OracleScene(cfg_k.scene_desc(), desc.eps)
        g = dev.trace_rays(rays, "closest", isect=2)
        r = ora.trace_rays(rays, "closest", watertight=True)
        c = classify_closest(rays, g, r, ora, watertight=True)
        assert c["error"] == 0, c["errors"]
        assert c["max_ulp_same_prim"] == 0
        assert c["exact"] + c["tie"] + c["ref_fn"] == len(rays)
        ga = dev.trace_rays(rays, "any", isect=2)
        ra = ora.trace_rays(rays, "any", watertight=True)
        assert ((ga["entity"] >= 0) == (ra["entity"] >= 0)).mean() >= 0.9999


@pytest.mark.gpu
def test_watertight_render_within_3_sigma(cornell_path):
    cfg = Config.from_file(cornell_path)
    desc, _ = cfg.rendering(0)
    desc.width, desc.height, desc.spp = 48, 48, 512
    desc.isect_mode = 2
    dev = DeviceScene(cfg)
    ora = oracle.OracleScene(cfg.scene_desc(), desc.eps)
    fg = Film(desc.width, desc.height, value_sq=True)
    fc = Film(desc.width, desc.height, value_sq=True)
    st = dev.render(desc, fg)
    assert st["samples"] == 48 * 48 * 512 and st["watchdog_flags"] == 0
    desc.isect_mode = 0
    ora.render(desc, fc)  # the reference's test: same image in expectation
    r = 0.5 - desc.eps
    frac, allowed, info = band_test(fg, fc, 1 / (4 * r * r))
    assert frac <= allowed, (frac, allowed, info)
    assert global_mean_z(fg, fc) < 4.0
