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


def _const(v):
    return {"type": "constant", "texel": list(np.atleast_1d(v).astype(float))}


def _unit(v):
    v = np.asarray(v, np.float64)
    return (v / np.linalg.norm(v)).astype(np.float32)


def _fresnel_conductor(cos_i, n):
    """Exact Fresnel reflectance of unpolarised light at a conductor of
    complex relative index n (Fresnel equations with Snell's law in C)."""
    cos_i = np.asarray(cos_i, np.complex128)
    sin2_t = (1 - cos_i ** 2) / n ** 2
    cos_t = np.sqrt(1 - sin2_t)
    rs = (cos_i - n * cos_t) / (cos_i + n * cos_t)
    rp = (n * cos_i - cos_t) / (n * cos_i + cos_t)
    return 0.5 * (np.abs(rs) ** 2 + np.abs(rp) ** 2)


def _fresnel_dielectric(cos_i, n):
    sin_t = np.sqrt(np.maximum(0, 1 - cos_i ** 2)) / n
    cos_t = np.sqrt(np.maximum(0, 1 - sin_t ** 2))
    rs = (cos_i - n * cos_t) / (cos_i + n * cos_t)
    rp = (n * cos_i - cos_t) / (n * cos_i + cos_t)
    return 0.5 * (rs ** 2 + rp ** 2)


def test_mirror_reflects_with_the_conductor_fresnel_term():
    # mirror.cpp:62-76 builds ConductorPoint(ior, 1, k): the medium of index
    # `ior` is outside, so the relative complex index is (1 + i k) / ior
    ior, k, col = np.array([1.3, 1.0, 0.8]), np.array([3.9, 2.4, 0.0]), np.array([0.9, 0.8, 0.7])
    mat = {"type": "mirror", "color_map": _const(col), "eta": _const(ior), "k": _const(k)}
    cfg, desc, ora = _oracle(K.material_probe(mat))
    cos_i = np.linspace(0.05, 1.0, 64)
    wo = np.stack([np.sqrt(1 - cos_i ** 2), np.zeros_like(cos_i), cos_i], 1).astype(np.float32)
    wi, f, pdf, delta = ora.bsdf_sample(0, wo, np.full((64, 3), 0.5, np.float32))
    assert delta.all() and np.all(pdf == 1)
    np.testing.assert_allclose(wi, wo * np.float32([-1, -1, 1]), atol=2e-6)
    want = col[None] * np.stack([_fresnel_conductor(cos_i, (1 + 1j * k[c]) / ior[c]) for c in range(3)], 1)
    np.testing.assert_allclose(f * wi[:, 2:3] / pdf[:, None], want, rtol=2e-4, atol=1e-6)
    # delta: eval and pdf are zero for every pair
    ef, ep = ora.bsdf_eval(0, wi, wo)
    assert not ef.any() and not ep.any()


def test_glass_splits_by_the_dielectric_fresnel_term():
    # glass.cpp:34-70: reflect with probability Fr, refract with 1 - Fr;
    # Snell's law; radiance scaled by (eta_i / eta_t)^2 on refraction
    mat = {"type": "glass", "ior": _const(1.5), "color_reflection_map": _const(0.9),
           "color_refraction_map": _const([0.64, 0.81, 1.0])}
    cfg, desc, ora = _oracle(K.material_probe(mat))
    n = 40_000
    for cz in (0.9, 0.4, -0.8, -0.5):
        wo = np.tile(_unit([math.sqrt(1 - cz * cz), 0, cz]), (n, 1))
        u = np.random.default_rng(5).random((n, 3)).astype(np.float32)
        wi, f, pdf, delta = ora.bsdf_sample(0, wo, u)
        assert delta.all()
        inside = cz < 0
        fr = 1.0 if inside and math.sqrt(1 - cz * cz) * 1.5 >= 1 else \
            float(_fresnel_dielectric(abs(cz), 1 / 1.5 if inside else 1.5))
        refl = wi[:, 2] * cz > 0
        assert abs(refl.mean() - fr) < 4 * math.sqrt(fr * (1 - fr) / n) + 1e-6
        np.testing.assert_allclose(pdf[refl], fr, rtol=1e-5)
        np.testing.assert_allclose((f[refl] * np.abs(wi[refl, 2:3]) / pdf[refl, None]), 0.9, rtol=1e-5)
        if fr < 1:
            t = ~refl
            eta = 1 / 1.5 if not inside else 1.5   # eta_i / eta_t along the light path
            sin_o = math.sqrt(1 - cz * cz)
            np.testing.assert_allclose(np.sqrt(1 - wi[t, 2] ** 2), eta * sin_o, rtol=1e-4)
            got = f[t] * np.abs(wi[t, 2:3]) / pdf[t, None]
            np.testing.assert_allclose(got, np.broadcast_to(np.float32(eta * eta) * np.float32([0.8, 0.9, 1.0]),
                                                            got.shape), rtol=1e-5)
    # total internal reflection: always reflected
    wo = np.tile(_unit([0.9, 0, -0.3]), (1000, 1))
    wi, f, pdf, _ = ora.bsdf_sample(0, wo, np.random.default_rng(6).random((1000, 3)).astype(np.float32))
    assert np.all(wi[:, 2] < 0) and np.all(pdf == 1)


@pytest.mark.parametrize("mat", [
    {"type": "metal", "color": _const([0.95, 0.8, 0.5]), "eta": _const([0.2, 0.4, 1.4]), "k": _const([3.9, 2.4, 1.9]),
     "roughness": _const(0.4), "anisotropic": _const(0.5)},
    {"type": "phong", "d": _const([0.5, 0.3, 0.2]), "s": _const([0.4, 0.4, 0.4]), "ns": _const(12)},
], ids=["metal", "phong"])
def test_glossy_sampling_follows_its_pdf(mat):
    # aggregate.h: the sampled f / pdf equal eval / pdf at the sampled
    # direction; the pdf integrates to at most 1 over the hemisphere (the
    # part of a lobe below the horizon is lost); the importance estimate of
    # the directional albedo matches a uniform-hemisphere estimate and is <= 1
    cfg, desc, ora = _oracle(K.material_probe(mat))
    n = 400_000
    wo = np.tile(_unit([0.5, 0.2, 0.8]), (n, 1))
    s_wi, s_f, s_pdf, delta = ora.bsdf_sample(0, wo, np.random.default_rng(8).random((n, 3)).astype(np.float32))
    assert not delta.any()
    ok = s_pdf > 0
    assert ok.mean() > 0.8
    e_f, e_pdf = ora.bsdf_eval(0, s_wi[ok], wo[ok])
    np.testing.assert_allclose(s_pdf[ok], e_pdf, rtol=2e-4)
    np.testing.assert_allclose(s_f[ok], e_f, rtol=2e-4, atol=1e-7)
    wi = _hemi(n, 10)
    f_u, p_u = ora.bsdf_eval(0, wi, wo)
    mass = np.mean(p_u) * 2 * math.pi
    assert 0.85 < mass < 1.01, mass
    est = np.sum(s_f[ok] * s_wi[ok, 2:3] / s_pdf[ok, None], 0) / n
    ref = np.mean(f_u * wi[:, 2:3], 0) * 2 * math.pi
    np.testing.assert_allclose(est, ref, rtol=0.03)
    assert np.all(est <= 1.0)


def test_ao_unblocked_fraction_between_parallel_planes():
    # trace_ao (path_tracing.cpp:383-415): lerp(low, high, unblocked fraction)
    cfg, desc, ora = _oracle(K.ao_slab(h=0.5, dist=1.0, spp=256))
    assert desc.renderer == 1 and desc.ao_sample_count == 5
    f = Film(desc.width, desc.height, gbuffer=True)
    ora.render(desc, f)
    img = f.image().reshape(-1, 3)
    e = desc.eps
    frac = ((0.5 - e) / (1.0 - e)) ** 2
    low, high = np.array([0.1, 0.2, 0.3]), np.array([0.9, 0.8, 0.7])
    want = low + (high - low) * frac
    n = desc.width * desc.height * desc.spp
    sigma = np.abs(high - low) * math.sqrt(frac * (1 - frac) / (n * 5))
    assert np.all(np.abs(img.mean(0) - want) < 5 * sigma + 1e-6), (img.mean(0), want)
    w = f.weight.reshape(-1, 1)
    np.testing.assert_allclose(f.albedo.reshape(-1, 3) / w, np.broadcast_to(high, (64, 3)), rtol=1e-6)
    np.testing.assert_allclose(np.abs(f.normal.reshape(-1, 3) / w)[:, 2], 1.0, rtol=1e-6)


def test_ao_background_on_miss():
    cfg, desc, ora = _oracle(K.ao_slab(spp=4, looking_up=True))
    f = Film(desc.width, desc.height, gbuffer=True)
    ora.render(desc, f)
    np.testing.assert_allclose(f.image().reshape(-1, 3), np.broadcast_to(np.float32([0.05, 0.06, 0.07]), (64, 3)),
                               rtol=1e-6)
    assert not f.albedo.any()


def _nd_cdf(x):
    return 1 - 0.25 * np.exp(-x) - 0.75 * np.exp(-x / 3)


def _nd_inv_cdf(u):
    lo, hi = 0.0, 200.0
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        lo, hi = (mid, hi) if _nd_cdf(mid) < u else (lo, mid)
    return 0.5 * (lo + hi)


@pytest.mark.parametrize("A", [(0.5, 0.5, 0.5), (0.8, 0.5, 0.2)])
def test_subsurface_weight_on_a_plane(A):
    # separable.cpp:107-248 on a flat surface: only the normal-axis probe
    # (probability 1/2) meets the plane, once; its pdf_pi keeps 1/2 of the
    # axis term, so E[w_c] = (1 - Fr(eta, cos 0)) * 2 pi * integral of
    # eval_r,c(r) * (sum over sampled channels whose r_max covers r of
    # pdf_r) / (sum of pdf_r) dr -- for a grey A exactly (1 - Fr) A P(x_max)
    ior, dmfp = 1.3, 0.1
    cfg, desc, ora = _oracle(K.subsurface_plane(A=A, dmfp=(dmfp,) * 3, ior=ior))
    n = 400_000
    w, x = ora.subsurface([0.3, 0.1, 2.0], [0, 0, -1], n, seed=3)
    A = np.array(A, np.float64)
    d = dmfp / (3.5 + 100 * (A - 0.33) ** 4)
    xm = _nd_inv_cdf(0.996)
    fro = 1 - ((ior - 1) / (ior + 1)) ** 2
    r = np.linspace(0, xm * d.max(), 400_001)
    pdf_r = 0.25 * (np.exp(-r[None] / d[:, None]) + np.exp(-r[None] / (3 * d[:, None]))) / d[:, None]
    covered = (r[None] <= xm * d[:, None]) * pdf_r
    ratio = covered.sum(0) / pdf_r.sum(0)
    want = np.array([fro * 2 * np.pi * np.trapezoid(
        A[c] * (np.exp(-r / d[c]) + np.exp(-r / (3 * d[c]))) / (8 * np.pi * d[c]) * ratio, r) for c in range(3)])
    if np.all(A == A[0]):
        np.testing.assert_allclose(want, fro * A * 0.996, rtol=1e-4)
    valid = w[:, 0] > 0
    assert abs(valid.mean() - 0.5 * np.mean([1.0])) < 0.01        # the normal axis only
    se = w.std(0) / math.sqrt(n)
    assert np.all(np.abs(w.mean(0) - want) < 5 * se), (w.mean(0), want, se)
    # exit points on the plane, within r_max of the entry
    dist = np.linalg.norm(x[valid] - np.float32([0.3, 0.1, 0]), axis=1)
    assert np.all(np.abs(x[valid, 2]) < 1e-5) and dist.max() <= xm * d.max() * 1.0001
