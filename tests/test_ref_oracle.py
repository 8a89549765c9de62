"""The restated oracle against the reference's own renderer.

oracle/_ref/libatrc_ref.so is Atrc's tracer and factory sources compiled
unchanged against an agz-utils compatibility shim (oracle/ref/); its scene
parsing, BVHs, intersection tests, materials, lights, media and trace_std are
the reference's code.  These tests pin the restated oracle (which the GPU
parity tests use as their checker) to it:

* known answers rendered by the reference itself (white furnace, absorbing
  slab);
* closest hits of seeded rays: the same entity for every ray, and t
  bit-identical except where the reference transforms a ray twice (nested
  transform_wrapper chains, which the device collapses into one instance
  transform) or builds rotation and instance matrices with agz-utils' own
  float matrix code (absent from the checkout; the shim stands in), where t
  agrees to a few ulp;
* images: the per-pixel 3-sigma band and the image-mean z-score, on every
  known-answer scene and small versions of the benchmark scenes.
"""
from __future__ import annotations

import json

import numpy as np
import pytest

import oracle
from atrc_b200 import Config, Film, scenes
from tests import kat_scenes as K
from tests.parity import band_test, global_mean_z, seeded_rays, ulp_diff

pytestmark = pytest.mark.skipif(not oracle.ref_available(),
                                reason="oracle/_ref/libatrc_ref.so not built (oracle/ref/build_ref.py needs the "
                                       "reference checkout)")


def _write(tmp_path, name, cfgd) -> str:
    p = tmp_path / f"{name}.json"
    p.write_text(K.dumps(cfgd))
    return str(p)


def _scene(tmp_path, name: str, spp: int = 256) -> str:
    """Path of a small scene file: the known-answer scenes and reduced
    versions of the benchmark scenes."""
    if name in ("feature", "materials", "subsurface"):
        sub = tmp_path / name
        sub.mkdir(exist_ok=True)
        fn = {"feature": K.feature_scene, "materials": K.materials_scene, "subsurface": K.subsurface_scene}[name]
        return _write(sub, "scene", fn(sub, spp=spp))
    if name == "cornell":
        return str(scenes.cornell_box(tmp_path / "cornell", width=32, height=32, spp=spp))
    if name == "instanced":
        return str(scenes.instanced_disney(tmp_path / "inst", ico_level=4, hf_res=128, width=32, height=18, spp=spp))
    if name == "media":
        return str(scenes.media_scene(tmp_path / "media", width=24, height=24, spp=spp, grid_res=32, sphere_level=3))
    raise KeyError(name)


def _render_both(path: str, spp: int | None = None, seed: int = 3):
    cfg = Config.from_file(path)
    desc, _ = cfg.rendering(0)
    if spp is not None:
        desc.spp = spp
    ref = oracle.RefScene(path)
    fr = Film(desc.width, desc.height, value_sq=True)
    ref.render(fr, spp=desc.spp, seed=seed)
    ora = oracle.OracleScene(cfg.scene_desc(), desc.eps)
    fo = Film(desc.width, desc.height, value_sq=True)
    ora.render(desc, fo)
    return desc, fr, fo


def test_reference_renders_known_answers(tmp_path):
    # white furnace: a convex albedo-1 Lambertian sphere under a uniform sky
    # of radiance 1 reflects all it receives, so every pixel's mean is 1
    p = _write(tmp_path, "furnace", K.furnace(spp=64))
    desc, _ = Config.from_file(p).rendering(0)
    f = Film(desc.width, desc.height, value_sq=True)
    oracle.RefScene(p).render(f, spp=desc.spp, seed=5)
    w = f.weight.sum()
    mean = f.value.reshape(-1, 3).sum(0) / w
    var = f.value_sq.reshape(-1, 3).sum(0) / w - mean ** 2
    se = np.sqrt(np.maximum(var, 1e-12) / (desc.width * desc.height * desc.spp))
    assert np.all(np.abs(mean - 1) < 4 * se + 1e-6), (mean, se)
    # an absorbing slab seen through a narrow camera: exp(-sigma_a d), up to
    # the eps offsets of the segments through it (the same bound as the
    # restated oracle's test)
    cfgd, expect = K.slab(tmp_path, spp=64)
    p = _write(tmp_path, "slab", cfgd)
    desc, _ = Config.from_file(p).rendering(0)
    f = Film(desc.width, desc.height, value_sq=True)
    oracle.RefScene(p).render(f, spp=desc.spp, seed=5)
    img = f.value.reshape(desc.height, desc.width, 3) / f.weight.reshape(desc.height, desc.width, 1)
    assert abs(img[desc.height // 2, desc.width // 2, 0] - expect) < 2e-3 * expect


def _inexact_entities(path: str) -> set[int]:
    """Entities whose t may differ from the reference's by a few ulp: a
    transform_wrapper in the geometry chain (the reference transforms the ray
    once per wrapper, the device once for the collapsed chain), or a rotation
    in a transform (agz-utils builds rotation matrices with its own float
    code, which the checkout does not have)."""
    js = json.loads(open(path).read())
    out = set()
    for i, e in enumerate(js["scene"]["entities"]):
        g = e.get("geometry", {})
        while isinstance(g, dict):
            steps = g.get("transform") or []
            steps = steps if isinstance(steps, list) else [steps]
            if g.get("type") == "transform_wrapper" or \
                    any(str(t.get("type", "")).startswith(("rotate", "mat3")) for t in steps):
                out.add(i)
                break
            g = g.get("internal")
    return out


@pytest.mark.parametrize("name", ["cornell", "feature", "materials", "subsurface", "media", "instanced"])
def test_closest_hits_match_reference(tmp_path, name):
    path = _scene(tmp_path, name, spp=1)
    cfg = Config.from_file(path)
    desc, _ = cfg.rendering(0)
    ref = oracle.RefScene(path)
    ora = oracle.OracleScene(cfg.scene_desc(), desc.eps)
    rays = seeded_rays(100_000, [-22.0] * 3, [22.0] * 3, list(desc.camera.pos), seed=7)
    a, b = ref.trace_rays(rays), ora.trace_rays(rays)
    assert np.array_equal(a["entity"], b["entity"])
    hit = a["entity"] >= 0
    assert hit.sum() > 1000
    u = ulp_diff(a["t"], b["t"])
    if name == "instanced":
        # every entity is a random instance (translate x mat3 x scale)
        uh = u[hit]
        assert np.median(uh) <= 1 and np.quantile(uh, 0.99) <= 128, np.quantile(uh, [0.5, 0.99])
        rel = np.abs(a["t"] - b["t"])[hit] / np.abs(b["t"][hit])
        assert np.quantile(rel, 0.999) < 1e-4
        return
    loose = np.isin(a["entity"], sorted(_inexact_entities(path)))
    assert np.all(u[hit & ~loose] == 0), int(u[hit & ~loose].max())
    if (hit & loose).any():
        assert u[hit & loose].max() <= 4


def test_any_hits_match_reference(tmp_path):
    path = _scene(tmp_path, "feature", spp=1)
    cfg = Config.from_file(path)
    desc, _ = cfg.rendering(0)
    rays = seeded_rays(50_000, [-4.0] * 3, [4.0] * 3, list(desc.camera.pos), seed=11)
    rays["t_max"] = np.random.default_rng(3).uniform(0.5, 6.0, len(rays)).astype(np.float32)
    a = oracle.RefScene(path).trace_rays(rays, mode="any")
    b = oracle.OracleScene(cfg.scene_desc(), desc.eps).trace_rays(rays, mode="any")
    assert np.array_equal(a["entity"] >= 0, b["entity"] >= 0)


@pytest.mark.parametrize("name,spp", [("cornell", 256), ("feature", 256), ("materials", 256), ("subsurface", 256),
                                      ("media", 1024), ("instanced", 128)])
def test_images_match_reference(tmp_path, name, spp):
    desc, fr, fo = _render_both(_scene(tmp_path, name, spp=spp))
    r = 0.5 - desc.eps
    frac, allowed, info = band_test(fr, fo, 1 / (4 * r * r), cluster=3)
    assert frac <= allowed, (frac, allowed, info)
    assert global_mean_z(fr, fo) < 4.0


def test_ao_matches_reference(tmp_path):
    # the reference's ao renderer (render::trace_ao): the parallel-plane known
    # answer and the 3-sigma band against the restated oracle
    cfgd = K.ao_slab(spp=256)
    cfgd["rendering"]["width"] = cfgd["rendering"]["height"] = 32
    p = _write(tmp_path, "ao", cfgd)
    desc, fr, fo = _render_both(p)
    e = desc.eps
    frac = ((0.5 - e) / (1.0 - e)) ** 2
    low, high = np.array([0.1, 0.2, 0.3]), np.array([0.9, 0.8, 0.7])
    want = low + (high - low) * frac
    n = desc.width * desc.height * desc.spp
    sigma = np.abs(high - low) * np.sqrt(frac * (1 - frac) / (n * 5))
    assert np.all(np.abs(fr.image().reshape(-1, 3).mean(0) - want) < 4 * sigma)
    r = 0.5 - desc.eps
    f, allowed, info = band_test(fr, fo, 1 / (4 * r * r), cluster=3)
    assert f <= allowed, (f, allowed, info)


def test_gbuffer_matches_reference(tmp_path):
    # the G-buffer PerPixelRenderer keeps beside the image
    # (perpixel_renderer.cpp:38-44): first-hit albedo and normal and the
    # denoise flag.  Per pixel they are Monte Carlo averages over the pixel's
    # footprint, so the image-wide means are compared
    sub = tmp_path / "feature"
    sub.mkdir()
    p = _write(sub, "scene", K.feature_scene(sub, spp=64))
    cfg = Config.from_file(p)
    desc, _ = cfg.rendering(0)
    fr = Film(desc.width, desc.height, gbuffer=True)
    oracle.RefScene(p).render(fr, spp=desc.spp, seed=3)
    fo = Film(desc.width, desc.height, gbuffer=True)
    oracle.OracleScene(cfg.scene_desc(), desc.eps).render(desc, fo)
    wr, wo = fr.weight.reshape(-1, 1), fo.weight.reshape(-1, 1)
    for k in ("albedo", "normal"):
        a = getattr(fr, k).reshape(-1, 3) / wr
        b = getattr(fo, k).reshape(-1, 3) / wo
        assert np.all(np.abs(a.mean(0) - b.mean(0)) < 1e-3), (k, a.mean(0), b.mean(0))
        assert np.mean(np.abs(a - b).max(1) < 1e-4) > 0.4     # pixels inside one flat surface agree exactly
    np.testing.assert_array_equal(fr.denoise / fr.weight, fo.denoise / fo.weight)


def test_gaussian_filter_matches_reference(tmp_path):
    # the reference's FilmFilterApplier (render_target.h:80) with the Gaussian
    # filter.  The reference scales the filter by a Monte Carlo estimate of
    # 1 / (its integral) (gaussian_filter.cpp:16-38, 64-71); pt_cuda and the oracle
    # leave it unscaled.  The constant cancels in value / weight, so the
    # images agree; the reference's weights, divided by it, follow the same
    # analytic expectation as the oracle's.
    from math import erf, exp, pi, sqrt

    from tests.parity import filter_weight_z
    sub = tmp_path / "gauss"
    sub.mkdir()
    path = _write(sub, "scene", K.feature_scene(sub, spp=128, gaussian=True))
    desc, fr, fo = _render_both(path)
    r, a = desc.filter_radius, desc.filter_alpha
    assert desc.filter_type != 0
    g0 = 1 - exp(-a * r * r)
    norm = float(oracle.RefScene(path).filter_eval([0.0], [0.0])[0]) / (g0 * g0)
    integral = sqrt(pi / a) * erf(r * sqrt(a)) - 2 * r * exp(-a * r * r)
    assert abs(norm * integral ** 2 - 1) < 0.01, norm
    for w in (fr.weight / norm, fo.weight):
        z = filter_weight_z(w, desc.width, desc.height, desc.spp, r, a)
        assert np.mean(np.abs(z)) < 0.9 and np.mean(np.abs(z) > 4) < 0.002, (np.mean(np.abs(z)), np.abs(z).max())
    wmax = g0 * g0

    def st(f, scale):
        w = f.weight.reshape(-1, 1)
        mu = f.value.reshape(-1, 3) / w
        var = np.maximum(f.value_sq.reshape(-1, 3) / w - mu * mu, 0)
        return mu, var, w / (scale * wmax)
    mr, vr, nr = st(fr, norm)
    mo, vo, no = st(fo, 1.0)
    z = np.abs(mr - mo) / np.sqrt(vr / nr + vo / no + 1e-12)
    assert np.mean(z > 4) < 0.01, np.mean(z > 4)
    assert global_mean_z(fr, fo) < 4.0


@pytest.mark.parametrize("name,spp", [("cornell", 256), ("feature", 256), ("subsurface", 256), ("media", 1024)])
def test_nomis_images_match_reference(tmp_path, name, spp):
    # use_mis = 0: the reference's trace_nomis (path_tracing.cpp:227-381),
    # BSDF sampling only, against the oracle's restatement of it
    import json
    from pathlib import Path
    p = Path(_scene(tmp_path, name, spp=spp))
    cfgd = json.loads(p.read_text())
    for entry in cfgd["rendering"] if isinstance(cfgd["rendering"], list) else [cfgd["rendering"]]:
        entry["renderer"]["use_mis"] = 0
    q = p.with_name(p.stem + "_nomis.json")
    q.write_text(json.dumps(cfgd))
    desc, fr, fo = _render_both(str(q))
    assert desc.use_mis == 0
    r = 0.5 - desc.eps
    frac, allowed, info = band_test(fr, fo, 1 / (4 * r * r), cluster=3)
    assert frac <= allowed, (frac, allowed, info)
    assert global_mean_z(fr, fo) < 4.0
