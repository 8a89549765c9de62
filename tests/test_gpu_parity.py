"""GPU parity against the CPU oracle, through the C ABI.

Ray queries: closest-hit primitive identifiers bit-exact and hit distances
within 2 ulp of the reference's BVH (triangle_bvh.cpp / entity_bvh.cpp with
the Moller-Trumbore test of triangle_aux.h), mismatches classified.
Images: per-pixel mean within a 3-sigma Monte Carlo band of the oracle's
`pt` (failing fraction below the binomial bound)."""
import numpy as np
import pytest

import oracle
from atrc_b200 import Config, DeviceScene, Film
from tests.parity import band_test, classify_closest, global_mean_z, seeded_rays

pytestmark = pytest.mark.gpu


def _scene(path):
    cfg = Config.from_file(path)
    desc, _ = cfg.rendering(0)
    return cfg, desc, DeviceScene(cfg), oracle.OracleScene(cfg.scene_desc(), desc.eps)


@pytest.fixture(scope="module")
def cornell(cornell_path):
    return _scene(cornell_path)


def test_closest_hits_bit_exact_cornell(cornell):
    cfg, desc, dev, ora = cornell
    rays = seeded_rays(400_000, [-1.2] * 3, [1.2] * 3, list(desc.camera.pos), seed=7)
    g = dev.trace_rays(rays, "closest", exact=True)
    r = ora.trace_rays(rays, "closest")
    c = classify_closest(rays, g, r, ora)
    assert c["error"] == 0, c["errors"]
    assert c["max_ulp_same_prim"] == 0
    # ties: two different primitives at the same distance (the box bottoms are
    # coplanar with the floor); the reference keeps the last one it visits
    assert c["exact"] + c["tie"] + c["ref_fn"] == len(rays), c
    assert c["tie"] <= len(rays) * 0.005 and c["exact"] >= len(rays) * 0.99, c
    assert (g["entity"] >= 0).mean() > 0.5


def test_any_hit_matches_cornell(cornell):
    cfg, desc, dev, ora = cornell
    rays = seeded_rays(200_000, [-1.2] * 3, [1.2] * 3, list(desc.camera.pos), seed=8)
    rays["t_max"] = np.random.default_rng(3).uniform(0.05, 3.0, len(rays)).astype(np.float32)
    g = dev.trace_rays(rays, "any", exact=True)
    r = ora.trace_rays(rays, "any")
    agree = (g["entity"] >= 0) == (r["entity"] >= 0)
    assert agree.mean() >= 0.9999
    assert 0.05 < (g["entity"] >= 0).mean() < 0.95


def test_fast_mode_agrees_with_exact(cornell):
    cfg, desc, dev, ora = cornell
    rays = seeded_rays(100_000, [-1.2] * 3, [1.2] * 3, list(desc.camera.pos), seed=9)
    a = dev.trace_rays(rays, "closest", exact=True)
    b = dev.trace_rays(rays, "closest", exact=False)
    same = (a["entity"] == b["entity"]) & (a["prim"] == b["prim"])
    assert same.mean() > 0.999
    hit = same & (a["entity"] >= 0)
    rel = np.abs(a["t"][hit] - b["t"][hit]) / np.maximum(np.abs(a["t"][hit]), 1e-6)
    assert np.mean(rel <= 1e-5) > 0.999 and np.median(rel) < 1e-6


def test_cornell_image_within_3_sigma(cornell_path):
    cfg = Config.from_file(cornell_path)
    desc, _ = cfg.rendering(0)
    desc.width, desc.height, desc.spp = 48, 48, 1024
    dev = DeviceScene(cfg)
    ora = oracle.OracleScene(cfg.scene_desc(), desc.eps)
    fg = Film(desc.width, desc.height, value_sq=True, gbuffer=True)
    fc = Film(desc.width, desc.height, value_sq=True, gbuffer=True)
    stats = dev.render(desc, fg)
    ora.render(desc, fc)
    assert stats["samples"] == desc.width * desc.height * desc.spp
    r = 0.5 - desc.eps
    frac, allowed, info = band_test(fg, fc, 1 / (4 * r * r))
    assert frac <= allowed, (frac, allowed, info)
    assert global_mean_z(fg, fc) < 4.0
    # G-buffer (first-hit albedo / normal) agrees to sampling noise
    wa = fg.weight.reshape(-1, 1)
    ga = fg.albedo.reshape(-1, 3) / wa
    ca = fc.albedo.reshape(-1, 3) / fc.weight.reshape(-1, 1)
    assert np.abs(ga - ca).mean() < 0.02


@pytest.fixture(scope="module")
def instanced(scene_dir):
    from atrc_b200.scenes import instanced_disney
    # same construction as the 1920x1080 workload, smaller meshes
    p = instanced_disney(scene_dir / "inst_small", ico_level=4, hf_res=128, width=64, height=36, spp=256)
    return _scene(p)


def test_closest_hits_bit_exact_instanced(instanced):
    cfg, desc, dev, ora = instanced
    rays = seeded_rays(1_000_000, [-22.0] * 3, [22.0] * 3, list(desc.camera.pos), seed=11)
    g = dev.trace_rays(rays, "closest", exact=True)
    r = ora.trace_rays(rays, "closest")
    c = classify_closest(rays, g, r, ora)
    assert c["error"] == 0, c["errors"]
    assert c["max_ulp_same_prim"] == 0
    assert c["exact"] + c["tie"] + c["ref_fn"] == len(rays)
    assert c["exact"] >= len(rays) * 0.9999, c
    assert 0.02 < (g["entity"] >= 0).mean() < 0.98


def test_axis_aligned_rays_match(instanced):
    # directions with exact zero components (the slab test must not turn
    # 0 * inf into NaN and cull every box)
    from tests.parity import RAY_DTYPE
    cfg, desc, dev, ora = instanced
    rng = np.random.default_rng(21)
    n = 60_000
    rays = np.zeros(n, dtype=RAY_DTYPE)
    rays["o"] = rng.uniform(-20, 20, (n, 3))
    axes = np.concatenate([np.eye(3), -np.eye(3)]).astype(np.float32)
    rays["d"] = axes[rng.integers(0, 6, n)]
    rays["t_min"] = 0
    rays["t_max"] = np.inf
    g = dev.trace_rays(rays, "closest", exact=True)
    r = ora.trace_rays(rays, "closest")
    c = classify_closest(rays, g, r, ora)
    assert c["error"] == 0, c["errors"]
    assert c["exact"] + c["tie"] + c["ref_fn"] == len(rays)
    assert 0.05 < (g["entity"] >= 0).mean() and c["exact"] >= len(rays) * 0.999, c


def test_instanced_disney_ibl_image_within_3_sigma(instanced):
    cfg, desc, dev, ora = instanced
    fg = Film(desc.width, desc.height, value_sq=True)
    fc = Film(desc.width, desc.height, value_sq=True)
    dev.render(desc, fg)
    ora.render(desc, fc)
    r = 0.5 - desc.eps
    frac, allowed, info = band_test(fg, fc, 1 / (4 * r * r))
    assert frac <= allowed, (frac, allowed, info)


def test_media_image_within_3_sigma(scene_dir):
    from atrc_b200.scenes import media_scene
    p = media_scene(scene_dir / "media_small", width=40, height=40, spp=256, grid_res=32, sphere_level=3)
    cfg, desc, dev, ora = _scene(p)
    fg = Film(desc.width, desc.height, value_sq=True)
    fc = Film(desc.width, desc.height, value_sq=True)
    dev.render(desc, fg)
    ora.render(desc, fc)
    r = 0.5 - desc.eps
    frac, allowed, info = band_test(fg, fc, 1 / (4 * r * r))
    assert frac <= allowed, (frac, allowed, info)


@pytest.mark.parametrize("disney_fixed", [0, 1])
def test_feature_scene_within_3_sigma(tmp_path, disney_fixed):
    from tests import kat_scenes as K
    cfg = Config.from_string(K.dumps(K.feature_scene(tmp_path, spp=512)), tmp_path)
    desc, _ = cfg.rendering(0)
    desc.disney_fixed = disney_fixed
    dev = DeviceScene(cfg)
    ora = oracle.OracleScene(cfg.scene_desc(), desc.eps)
    fg = Film(desc.width, desc.height, value_sq=True, gbuffer=True)
    fc = Film(desc.width, desc.height, value_sq=True, gbuffer=True)
    dev.render(desc, fg)
    ora.render(desc, fc)
    r = 0.5 - desc.eps
    frac, allowed, info = band_test(fg, fc, 1 / (4 * r * r))
    assert frac <= allowed, (frac, allowed, info)
    assert global_mean_z(fg, fc) < 4.0
    # first-hit normals (normal map, frames of every shape) agree
    gn = fg.normal.reshape(-1, 3) / fg.weight.reshape(-1, 1)
    cn = fc.normal.reshape(-1, 3) / fc.weight.reshape(-1, 1)
    assert np.mean(np.abs(gn - cn)) < 0.02


def test_materials_scene_within_3_sigma(tmp_path):
    # mirror, glass, anisotropic normal-mapped metal, phong, checker_board
    # and an 8-bit PNG texture against the oracle
    from tests import kat_scenes as K
    cfg = Config.from_string(K.dumps(K.materials_scene(tmp_path, spp=512)), tmp_path)
    desc, _ = cfg.rendering(0)
    dev = DeviceScene(cfg)
    ora = oracle.OracleScene(cfg.scene_desc(), desc.eps)
    fg = Film(desc.width, desc.height, value_sq=True, gbuffer=True)
    fc = Film(desc.width, desc.height, value_sq=True, gbuffer=True)
    dev.render(desc, fg)
    ora.render(desc, fc)
    r = 0.5 - desc.eps
    frac, allowed, info = band_test(fg, fc, 1 / (4 * r * r))
    assert frac <= allowed, (frac, allowed, info)
    assert global_mean_z(fg, fc) < 4.0
    # first-hit albedo (checker, PNG texels, material albedos) agrees
    ga = fg.albedo.reshape(-1, 3) / fg.weight.reshape(-1, 1)
    ca = fc.albedo.reshape(-1, 3) / fc.weight.reshape(-1, 1)
    assert np.abs(ga - ca).mean() < 0.02


def test_subsurface_scene_within_3_sigma(tmp_path):
    # Disney subsurface scattering (normalized diffusion probe, separable
    # exit BSDF) on a sphere and an instanced mesh against the oracle
    from tests import kat_scenes as K
    cfg = Config.from_string(K.dumps(K.subsurface_scene(tmp_path, spp=512)), tmp_path)
    desc, _ = cfg.rendering(0)
    dev = DeviceScene(cfg)
    ora = oracle.OracleScene(cfg.scene_desc(), desc.eps)
    fg = Film(desc.width, desc.height, value_sq=True)
    fc = Film(desc.width, desc.height, value_sq=True)
    stats = dev.render(desc, fg)
    assert stats["watchdog_flags"] == 0
    ora.render(desc, fc)
    r = 0.5 - desc.eps
    frac, allowed, info = band_test(fg, fc, 1 / (4 * r * r))
    assert frac <= allowed, (frac, allowed, info)
    assert global_mean_z(fg, fc) < 4.0


def test_solid_image_scene_within_3_sigma(tmp_path):
    # solid_image read at the world position (ideal diffuse albedo, glass
    # refraction colour) and at (u, v, 0) (Disney base colour)
    from tests import kat_scenes as K
    cfg = Config.from_string(K.dumps(K.solid_image_scene(tmp_path, spp=512)), tmp_path)
    desc, _ = cfg.rendering(0)
    dev = DeviceScene(cfg)
    ora = oracle.OracleScene(cfg.scene_desc(), desc.eps)
    fg = Film(desc.width, desc.height, value_sq=True, gbuffer=True)
    fc = Film(desc.width, desc.height, value_sq=True, gbuffer=True)
    dev.render(desc, fg)
    ora.render(desc, fc)
    r = 0.5 - desc.eps
    frac, allowed, info = band_test(fg, fc, 1 / (4 * r * r))
    assert frac <= allowed, (frac, allowed, info)
    ga = fg.albedo.reshape(-1, 3) / fg.weight.reshape(-1, 1)
    ca = fc.albedo.reshape(-1, 3) / fc.weight.reshape(-1, 1)
    assert np.abs(ga - ca).mean() < 0.02


def test_gaussian_filter_matches(tmp_path):
    from tests import kat_scenes as K
    cfg = Config.from_string(K.dumps(K.feature_scene(tmp_path, spp=128, gaussian=True)), tmp_path)
    desc, _ = cfg.rendering(0)
    dev = DeviceScene(cfg)
    ora = oracle.OracleScene(cfg.scene_desc(), desc.eps)
    fg, fc = Film(desc.width, desc.height, value_sq=True), Film(desc.width, desc.height, value_sq=True)
    dev.render(desc, fg)
    ora.render(desc, fc)
    # the splat footprint: per-tile sampling of the grown bound, per-tile
    # clamps and one-pixel distance steps, as z-scores against the analytic
    # expectation of the weights (the oracle is pinned to it on the CPU)
    from tests.parity import filter_weight_z
    for f in (fg, fc):
        z = filter_weight_z(f.weight, desc.width, desc.height, desc.spp, desc.filter_radius, desc.filter_alpha)
        assert np.mean(np.abs(z)) < 0.9 and np.mean(np.abs(z) > 4) < 0.002, (np.mean(np.abs(z)), np.abs(z).max())
    # conservative per-pixel z (sample count from the filter's peak weight)
    wmax = (1 - np.exp(-2 * 1.5 ** 2)) ** 2
    def st(f):
        w = f.weight.reshape(-1, 1)
        mu = f.value.reshape(-1, 3) / w
        var = np.maximum(f.value_sq.reshape(-1, 3) / w - mu * mu, 0)
        return mu, var, w / wmax
    mg, vg, ng = st(fg)
    mc, vc, nc = st(fc)
    z = np.abs(mg - mc) / np.sqrt(vg / ng + vc / nc + 1e-12)
    assert np.mean(z > 4) < 0.01


def test_closest_hits_bit_exact_1e7_full_workload():
    # the full 3.08M-triangle instanced workload and 10^7 seeded rays
    from atrc_b200.scenes import instanced_disney
    cfg, desc, dev, ora = _scene(instanced_disney())
    rays = seeded_rays(10_000_000, [-22.0] * 3, [22.0] * 3, list(desc.camera.pos), seed=13)
    g = dev.trace_rays(rays, "closest", exact=True)
    r = ora.trace_rays(rays, "closest")
    c = classify_closest(rays, g, r, ora)
    assert c["error"] == 0, c["errors"]
    assert c["max_ulp_same_prim"] == 0
    assert c["exact"] + c["tie"] + c["ref_fn"] == len(rays)
    assert c["exact"] >= len(rays) * 0.9999, c


@pytest.mark.parametrize("case", ["plane", "sphere", "box"])
def test_subsurface_probe_matches_oracle(tmp_path, case):
    # the device's subsurface walk (subsurface_sample) and the oracle's: the
    # fraction of valid samples and the mean weight per channel agree to
    # sampling noise, on a plane, a sphere and an instanced mesh box
    import json
    from tests import kat_scenes as K
    if case == "plane":
        c, o, d = K.subsurface_plane(A=(0.8, 0.5, 0.2)), [0.3, 0.1, 2.0], [0, 0, -1]
    else:
        c = K.subsurface_scene(tmp_path)
        o, d = ([-0.7, -3.0, -0.4], [0, 1, 0]) if case == "sphere" else ([0.8, -3.0, -0.55], [0.01, 1, 0.02])
    cfg = Config.from_string(json.dumps(c), tmp_path)
    desc, _ = cfg.rendering(0)
    dev = DeviceScene(cfg)
    ora = oracle.OracleScene(cfg.scene_desc(), desc.eps)
    n = 200_000
    wg, xg = dev.subsurface_probe(o, d, n, seed=5)
    wo, xo = ora.subsurface(o, d, n, seed=5)
    pg, po = (wg[:, 0] > 0).mean(), (wo[:, 0] > 0).mean()
    assert abs(pg - po) < 5 * np.sqrt(po * (1 - po) * 2 / n) + 1e-6, (pg, po)
    se = np.sqrt(wg.var(0) / n + wo.var(0) / n)
    assert np.all(np.abs(wg.mean(0) - wo.mean(0)) < 5 * se + 1e-6), (wg.mean(0), wo.mean(0), se)
