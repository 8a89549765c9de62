"""Known-answer tests of the CPU oracle (analytic results; the reference has
no golden vectors of its own)."""
import math

import numpy as np
import pytest

import oracle
from atrc_b200 import Config, Film
from tests import kat_scenes as K


def _oracle(cfg_dict, scene_dir="."):
    cfg = Config.from_string(K.dumps(cfg_dict), scene_dir)
    desc, _ = cfg.rendering(0)
    return cfg, desc, oracle.OracleScene(cfg.scene_desc(), desc.eps)


def test_white_furnace():
    cfg, desc, ora = _oracle(K.furnace(spp=64))
    f = Film(desc.width, desc.height, value_sq=True)
    ora.render(desc, f)
    img = f.image()
    n = float(f.weight.sum()) * 4 * (0.5 - 3e-4) ** 2
    mu = img.mean()
    var = (f.value_sq.sum() / f.weight.sum() / 3) - mu * mu
    assert abs(mu - 1.0) < 4 * math.sqrt(max(var, 1e-12) / n) + 1e-3, mu


def test_absorbing_slab_transmittance(tmp_path):
    cfgd, expected = K.slab(tmp_path)
    cfg, desc, ora = _oracle(cfgd, tmp_path)
    f = Film(desc.width, desc.height)
    ora.render(desc, f)
    centre = f.image()[4, 4]
    np.testing.assert_allclose(centre, expected, rtol=2e-3)


def test_moller_trumbore_edges_and_vertices():
    cfg, desc, ora = _oracle(K.edge_scene())
    rays, inside = K.edge_rays()
    h = ora.trace_rays(rays)
    assert np.array_equal(h["entity"] >= 0, inside)
    assert np.all(h["t"][inside] == np.float32(2.0))
    # the shared diagonal belongs to the first triangle (ABC is tested first)
    diag = (rays["o"][:, 0] == rays["o"][:, 1]) & inside
    assert np.all(h["prim"][diag] == 0)


def test_env_pdf_normalised(tmp_path):
    from atrc_b200.scenes import sky_map, write_pfm
    write_pfm(tmp_path / "sky.pfm", sky_map(128, 64, sun_peak=500.0, sun_radius_deg=4))
    cfgd = K.furnace()
    cfgd["scene"]["env"] = {"type": "ibl", "tex": {"type": "hdr", "filename": "${scene-directory}/sky.pfm"}}
    cfg, desc, ora = _oracle(cfgd, tmp_path)
    rng = np.random.default_rng(5)
    d = rng.normal(size=(400_000, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    pdf = ora.env_pdf(d.astype(np.float32))
    assert abs(pdf.mean() * 4 * math.pi - 1) < 0.01
    dirs, spdf = ora.env_sample(rng.random((200_000, 3)))
    np.testing.assert_allclose(np.linalg.norm(dirs, axis=1), 1, atol=1e-5)
    # the pdf a sample reports is the pdf of its direction
    # (a direction on a patch border may round into the neighbouring patch)
    assert np.mean(np.isclose(spdf, ora.env_pdf(dirs), rtol=2e-3)) > 0.9999
    # E[1/pdf] over importance samples is the sphere's area
    assert abs(np.mean(1 / spdf) / (4 * math.pi) - 1) < 0.03


def _hemi(n, seed):
    rng = np.random.default_rng(seed)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    d[:, 2] = np.abs(d[:, 2])
    return d.astype(np.float32)


def test_lambert_pdf_and_sampling_consistent():
    cfg, desc, ora = _oracle(K.material_probe({"type": "ideal_diffuse", "albedo": {"type": "constant", "texel": [0.6]}}))
    wo = np.tile(np.float32([0.3, 0.1, 0.95]) / np.linalg.norm([0.3, 0.1, 0.95]), (200_000, 1))
    wi = _hemi(200_000, 1)
    f, pdf = ora.bsdf_eval(0, wi, wo)
    # integral of the pdf over the hemisphere = 1; integral of f cos = albedo
    assert abs(np.mean(pdf) * 2 * math.pi - 1) < 0.01
    assert abs(np.mean(f[:, 0] * wi[:, 2]) * 2 * math.pi - 0.6) < 0.01
    s_wi, s_f, s_pdf, delta = ora.bsdf_sample(0, wo, np.random.default_rng(2).random((200_000, 3)))
    ok = s_pdf > 0
    e_wi, e_pdf = ora.bsdf_eval(0, s_wi[ok], wo[ok])
    np.testing.assert_allclose(s_pdf[ok], e_pdf, rtol=1e-4)
    assert abs(np.mean(1 / s_pdf[ok]) / (2 * math.pi) - 1) < 0.02
    assert not delta.any()


def test_disney_reports_mixture_pdf_but_never_samples_diffuse():
    # disney.cpp:578-589: the diffuse lobe choice is overwritten, so the
    # sampled directions do not follow the reported mixture pdf.
    mat = {"type": "disney", "base_color": {"type": "constant", "texel": [0.9]},
           "metallic": {"type": "constant", "texel": [0.0]}, "roughness": {"type": "constant", "texel": [0.2]}}
    cfg, desc, ora = _oracle(K.material_probe(mat))
    n = 200_000
    wo = np.tile(np.float32([0.0, 0.0, 1.0]), (n, 1))
    wi = _hemi(n, 3)
    _, pdf = ora.bsdf_eval(0, wi, wo)
    assert abs(np.mean(pdf) * 2 * math.pi - 1) < 0.05  # weights sum to 1 without transmission
    s_wi, s_f, s_pdf, _ = ora.bsdf_sample(0, wo, np.random.default_rng(4).random((n, 3)))
    ok = s_pdf > 0
    # under a correct sampler E[1/pdf] would be the hemisphere's area 2 pi;
    # the specular-only sampling makes it far smaller
    ratio = np.mean(1 / s_pdf[ok]) / (2 * math.pi)
    assert ratio < 0.7, ratio
    # the continuation estimate f cos / pdf is biased accordingly
    assert np.mean(s_f[ok, 0] * s_wi[ok, 2] / s_pdf[ok]) > 0


def test_gaussian_splat_follows_the_tiled_reference(tmp_path):
    # render_target.h:355-395: a tile samples its bound grown by the filter
    # radius and splats only into itself; framebuffer.h:49-80 steps the
    # distance by one pixel from the clamped first pixel.  The weights of the
    # film follow that model, and not the model of one film-wide tile.
    from tests.parity import filter_weight_z
    cfg, desc, ora = _oracle(K.feature_scene(tmp_path, spp=64, gaussian=True), tmp_path)
    f = Film(desc.width, desc.height)
    ora.render(desc, f)
    args = (desc.width, desc.height, desc.spp, desc.filter_radius, desc.filter_alpha)
    z = filter_weight_z(f.weight, *args)
    assert np.mean(np.abs(z)) < 0.9 and np.abs(z).max() < 5.5
    z_untiled = filter_weight_z(f.weight, *args, grid=1 << 20)
    assert np.abs(z_untiled).max() > 20


def test_fixed_disney_sampling_follows_its_pdf():
    # with the diffuse lobe sampled, E[1/pdf] over the samples is the area of
    # the hemisphere, and E[f cos / pdf] is the directional albedo (<= 1)
    mat = {"type": "disney", "base_color": {"type": "constant", "texel": [0.9]},
           "metallic": {"type": "constant", "texel": [0.0]}, "roughness": {"type": "constant", "texel": [0.2]}}
    cfg, desc, ora = _oracle(K.material_probe(mat))
    n = 400_000
    wo = np.tile(np.float32([0.0, 0.0, 1.0]), (n, 1))
    s_wi, s_f, s_pdf, _ = ora.bsdf_sample(0, wo, np.random.default_rng(4).random((n, 3)), disney_fixed=True)
    ok = s_pdf > 0
    assert abs(np.mean(np.where(ok, 1 / np.where(ok, s_pdf, 1), 0)) / (2 * math.pi) - 1) < 0.03
    e_f, e_pdf = ora.bsdf_eval(0, s_wi[ok], wo[ok])
    np.testing.assert_allclose(s_pdf[ok], e_pdf, rtol=1e-4)
    # the directional albedo from importance samples matches a uniform-hemisphere estimate
    est = np.sum(s_f[ok, 0] * s_wi[ok, 2] / s_pdf[ok]) / n
    wi = _hemi(n, 9)
    f_u, _ = ora.bsdf_eval(0, wi, wo)
    ref = np.mean(f_u[:, 0] * wi[:, 2]) * 2 * math.pi
    assert abs(est - ref) < 0.02 * ref, (est, ref)
