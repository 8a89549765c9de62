"""The learned guide on the GPU: the tensor-core network against an FP64
evaluation of the same parameters, the device pdf, training, and the
unbiasedness of guided rendering."""
import math

import numpy as np
import pytest

from atrc_b200 import AtrcError, Config, DeviceScene, Film
from atrc_b200.guide import RECORD_FLOATS, Guide
from tests import guide_ref as R
from tests.parity import band_test, global_mean_z

pytestmark = pytest.mark.gpu


def _unit(rng, n):
    d = rng.normal(size=(n, 3))
    return d / np.linalg.norm(d, axis=1, keepdims=True)


def _random_guide(seed=3):
    g = Guide([-1, -1, -1], [1, 1, 1], log2_table=12, seed=seed, max_select=R.MAX_SELECT)
    info = g.info()
    rng = np.random.default_rng(seed)
    w = np.concatenate([rng.normal(0, 1.5 / math.sqrt(fi), fo * fi)
                        for fo, fi in ((64, 112), (64, 64), (64, 64), (48, 64))]).astype(np.float32)
    t = rng.uniform(-1, 1, info["table_floats"]).astype(np.float32)
    g.set_params(w, t)
    return g, w, t, info


def _queries(rng, n):
    q = np.zeros((n, 10), np.float32)
    q[:, :3] = rng.uniform(-1, 1, (n, 3))
    q[:, 3:6] = _unit(rng, n)
    q[:, 6:9] = _unit(rng, n)
    q[:, 9] = rng.uniform(0, 1, n)
    return q


def test_network_matches_fp64_evaluation():
    g, w, t, info = _random_guide()
    assert info["inputs"] == 112 and info["hidden"] == 64 and info["outputs"] == 48
    rng = np.random.default_rng(11)
    q = _queries(rng, 1000)  # not a multiple of the 128-row tile
    raw = g.eval_raw(q).astype(np.float64)
    emu = R.forward(q, w, t, info, bf16_ops=True)   # BF16 operands, FP64 sums
    ref = R.forward(q, w, t, info)                  # all FP64
    rms = np.sqrt(np.mean(ref ** 2))
    assert rms > 0.1
    # the tensor cores compute exactly the BF16 network up to FP32 summation
    # (and an occasional BF16 tie rounded the other way in a hidden layer)
    err = np.abs(raw - emu)
    assert np.max(err) < 0.02 * rms and np.mean(err) < 1e-3 * rms, (np.max(err) / rms, np.mean(err) / rms)
    # and the FP64 network up to BF16 precision
    assert np.mean(np.abs(raw - ref)) < 0.03 * rms


def test_device_pdf_matches_fp64_evaluation():
    g, w, t, info = _random_guide(5)
    rng = np.random.default_rng(12)
    q = _queries(rng, 4096)
    ref_raw = R.forward(q, w, t, info)
    mu, _, _, c_ref = R.decode(ref_raw)
    # half the directions near a lobe mean, half uniform
    d = _unit(rng, 4096)
    near = mu[np.arange(2048), rng.integers(0, 8, 2048)] + 0.05 * rng.normal(size=(2048, 3))
    d[:2048] = near / np.linalg.norm(near, axis=1, keepdims=True)
    pdf, c = g.pdf(q, d.astype(np.float32))
    ref = R.pdf(ref_raw, d)
    rel = np.abs(pdf - ref) / ref
    assert np.median(rel) < 0.02 and np.quantile(rel, 0.95) < 0.15, (np.median(rel), np.quantile(rel, 0.95))
    # against the same network with BF16 operands (FP64 sums), the device pdf
    # differs only by FP32 summation and the FP32 decode: an order of
    # magnitude tighter
    emu = R.pdf(R.forward(q, w, t, info, bf16_ops=True), d)
    rel16 = np.abs(pdf - emu) / emu
    assert np.median(rel16) < 2e-3 and np.quantile(rel16, 0.95) < 2e-2, (np.median(rel16), np.quantile(rel16, 0.95))
    np.testing.assert_allclose(c, c_ref, atol=0.01)
    assert np.all(c >= 0) and np.all(c <= R.MAX_SELECT + 1e-6)


def test_selection_cap_can_change_between_renders():
    g, _, _, _ = _random_guide(8)
    rng = np.random.default_rng(14)
    q = _queries(rng, 512)
    d = _unit(rng, 512).astype(np.float32)
    _, c9 = g.pdf(q, d)
    g.set_max_select(0.3)
    assert g.info()["max_select"] == pytest.approx(0.3)
    _, c3 = g.pdf(q, d)
    # c = cap * sigmoid(o - 2): the same network, the cap rescales c
    np.testing.assert_allclose(c3, c9 * (0.3 / R.MAX_SELECT), rtol=1e-5, atol=1e-7)
    for bad in (0.0, -0.1, 1.0):
        with pytest.raises(AtrcError):
            g.set_max_select(bad)


def test_mixture_is_a_density():
    g, _, _, _ = _random_guide(7)
    rng = np.random.default_rng(13)
    q = np.repeat(_queries(rng, 4), 200_000, axis=0)
    d = _unit(rng, len(q)).astype(np.float32)
    pdf, _ = g.pdf(q, d)
    # integral over the sphere of every query's mixture is 1
    means = pdf.reshape(4, -1).mean(axis=1) * 4 * math.pi
    np.testing.assert_allclose(means, 1.0, rtol=0.05)


def _vmf_sample(rng, mu, kappa, n):
    u1, u2 = rng.random(n), rng.random(n)
    wz = 1 + np.log(u1 + (1 - u1) * np.exp(-2 * kappa)) / kappa
    v = np.sqrt(np.maximum(0, 1 - wz ** 2))
    phi = 2 * np.pi * u2
    a = np.array([1.0, 0, 0]) if abs(mu[0]) < 0.9 else np.array([0, 1.0, 0])
    x = np.cross(mu, a)
    x /= np.linalg.norm(x)
    y = np.cross(mu, x)
    return (np.cos(phi) * v)[:, None] * x + (np.sin(phi) * v)[:, None] * y + wz[:, None] * mu


def test_training_learns_a_lobe():
    # every record's direction follows one vMF lobe (kappa 30): the optimum
    # of the loss is that lobe chosen with the largest selection probability
    g = Guide([-1, -1, -1], [1, 1, 1], log2_table=12, base_resolution=2, max_resolution=16, batch=1 << 14, seed=9,
              max_select=0.9)
    rng = np.random.default_rng(21)
    n = 1 << 17
    mu = np.array([0.3, -0.5, 0.81])
    mu /= np.linalg.norm(mu)
    rec = np.zeros((n, RECORD_FLOATS), np.float32)
    rec[:, 0:3] = rng.uniform(-0.5, 0.5, (n, 3))
    rec[:, 3:6] = [0, 0, 1]
    rec[:, 6:9] = [0, 0, 1]
    rec[:, 9] = 0.5
    rec[:, 10:13] = _vmf_sample(rng, mu, 30.0, n)
    rec[:, 13] = 1 / (2 * math.pi)    # BSDF pdf of the direction
    rec[:, 17] = 1.0                   # weight
    p_true = 30 / (2 * math.pi) * np.exp(30 * (rec[:, 10:13] @ mu - 1))
    optimum = -np.mean(np.log(0.9 * p_true + 0.1 / (2 * math.pi)))
    q = rec[:512, :10].copy()
    q[:, :3] = rng.uniform(-0.5, 0.5, (512, 3))   # positions not trained on
    at_mu = np.tile(mu, (512, 1)).astype(np.float32)
    before, _ = g.pdf(q, at_mu)
    first = g.train_records(rec, steps=1)
    last = g.train_records(rec, steps=200)
    after, c = g.pdf(q, at_mu)
    assert g.info()["steps"] == 201
    assert first > optimum + 2.0
    assert optimum - 0.3 < last < optimum + 0.5, (first, last, optimum)
    assert np.median(after) > 2.0 > 10 * np.median(before), (np.median(before), np.median(after))
    assert np.median(c) > 0.7


def test_recording_render_keeps_targets(cornell_path):
    cfg = Config.from_file(cornell_path)
    desc, _ = cfg.rendering(0)
    desc.width, desc.height, desc.spp = 64, 64, 4
    dev = DeviceScene(cfg)
    g = Guide.for_scene(dev, log2_table=14, record_capacity=1 << 16)
    st = dev.render_guided(g, desc, Film(64, 64), record=True)
    assert st["samples"] == 64 * 64 * 4
    rec = g.records()
    assert len(rec) > 64 * 64
    wi = rec[:, 10:13]
    np.testing.assert_allclose(np.linalg.norm(wi, axis=1), 1, atol=1e-4)
    tgt = rec[:, 17]
    assert np.all(np.isfinite(tgt)) and np.all(tgt >= 0) and np.mean(tgt > 0) > 0.2
    assert np.all(rec[:, 13] >= 0)
    loss = g.train(steps=4)
    assert np.isfinite(loss)


def test_recording_subsamples_after_a_full_pass(cornell_path):
    # a pass with more guided vertices than record_capacity fills the
    # capacity with its first vertices; training then sets the next pass's
    # recording probability so that it keeps about 0.95 of the capacity,
    # drawn from all of its vertices
    cfg = Config.from_file(cornell_path)
    desc, _ = cfg.rendering(0)
    desc.width, desc.height, desc.spp = 64, 64, 4
    dev = DeviceScene(cfg)
    cap = 1 << 12
    g = Guide.for_scene(dev, log2_table=14, record_capacity=cap, batch=1 << 12)
    dev.render_guided(g, desc, Film(64, 64), record=True)
    assert len(g.records()) == cap                  # saturated: 64 x 64 x 4 samples, several vertices each
    g.train(steps=1)
    desc.first_spp = 4
    dev.render_guided(g, desc, Film(64, 64), record=True)
    rec = g.records()
    assert 0.75 * cap < len(rec) < cap, len(rec)    # about 0.95 cap, not saturated
    # the kept records come from the whole box, not one corner of the film
    pos = rec[:, 0:3]
    assert np.all(pos.max(0) - pos.min(0) > 1.5)
    assert np.mean(rec[:, 17] > 0) > 0.2


def test_guided_render_is_unbiased(cornell_path):
    # guiding changes the sampling, not the expectation: a guided render
    # (after some training) and a plain one agree within 3 sigma per pixel
    cfg = Config.from_file(cornell_path)
    desc, _ = cfg.rendering(0)
    desc.width, desc.height, desc.spp = 48, 48, 512
    dev = DeviceScene(cfg)
    g = Guide.for_scene(dev, log2_table=14, record_capacity=1 << 18, batch=1 << 14)
    train_desc, _ = cfg.rendering(0)
    train_desc.width, train_desc.height, train_desc.spp = 48, 48, 32
    train_desc.seed = 99
    for _ in range(4):
        dev.render_guided(g, train_desc, Film(48, 48), record=True)
        g.train(steps=8)
    plain = Film(48, 48, value_sq=True)
    guided = Film(48, 48, value_sq=True)
    dev.render(desc, plain)
    desc.seed = 1234
    dev.render_guided(g, desc, guided)
    r = 0.5 - desc.eps
    frac, allowed, info = band_test(guided, plain, 1 / (4 * r * r))
    assert frac <= allowed, (frac, allowed, info)
    assert global_mean_z(guided, plain) < 4.0


def _train_records(rng, n):
    rec = np.zeros((n, RECORD_FLOATS), np.float32)
    rec[:, :3] = rng.uniform(-1, 1, (n, 3))
    rec[:, 3:6] = _unit(rng, n)
    rec[:, 6:9] = _unit(rng, n)
    rec[:, 9] = rng.uniform(0, 1, n)
    # half the sampled directions near one lobe, half uniform
    lobe = np.array([0.3, -0.5, 0.81]) / np.linalg.norm([0.3, -0.5, 0.81])
    near = lobe + 0.3 * rng.normal(size=(n, 3))
    wi = np.where(rng.uniform(size=(n, 1)) < 0.5, near, rng.normal(size=(n, 3)))
    rec[:, 10:13] = wi / np.linalg.norm(wi, axis=1, keepdims=True)
    rec[:, 13] = rng.uniform(0.05, 1.0, n)
    rec[:, 17] = rng.uniform(0, 2, n) * (rng.uniform(size=n) > 0.1)
    rec[:, 21] = -1
    return rec


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def test_training_gradients_match_fp64_backward():
    # 300 tiles of 128 records on 148 SMs: CTAs accumulate dW^T in TMEM over
    # two or three tiles before their atomic flush
    g, w, t, info = _random_guide(seed=5)
    g.close()
    g = Guide([-1, -1, -1], [1, 1, 1], log2_table=12, seed=5, record_capacity=1 << 16, max_select=R.MAX_SELECT)
    info = g.info()
    g.set_params(w, t)
    rng = np.random.default_rng(17)
    rec = _train_records(rng, 128 * 300)
    gw, gt, loss = g.gradients(rec)
    rw, rt, rloss = R.backward(rec, w, t, info, bf16_ops=True)
    assert abs(loss - rloss) <= 1e-3 * abs(rloss)
    # the kernel computes exactly the BF16-operand backward up to FP32 sums
    assert _rel(gw, rw) < 5e-3, _rel(gw, rw)
    assert _rel(gt, rt) < 5e-3, _rel(gt, rt)
    cos = float(np.dot(gw, rw) / np.linalg.norm(gw) / np.linalg.norm(rw))
    assert cos > 0.99999, cos
    # per layer, so that a wrong layer cannot hide behind a large one
    offs = np.cumsum([0, 64 * 112, 64 * 64, 64 * 64, 48 * 64])
    for a, b in zip(offs[:-1], offs[1:]):
        assert _rel(gw[a:b], rw[a:b]) < 1e-2, (a, _rel(gw[a:b], rw[a:b]))
    # and against the all-FP64 network to BF16 precision
    fw, ft, _ = R.backward(rec, w, t, info, bf16_ops=False)
    assert _rel(gw, fw) < 0.05 and _rel(gt, ft) < 0.05


def test_adam_steps_match_reference():
    g, w, t, info = _random_guide(seed=6)
    g.close()
    g = Guide([-1, -1, -1], [1, 1, 1], log2_table=12, seed=6, record_capacity=1 << 16, batch=1 << 16,
              max_select=R.MAX_SELECT)
    info = g.info()
    g.set_params(w, t)
    lr = g.desc.learning_rate
    rng = np.random.default_rng(23)
    batches = [_train_records(rng, 128 * 64), _train_records(rng, 128 * 64)]
    p = np.concatenate([w, t]).astype(np.float64)
    m = np.zeros_like(p)
    v = np.zeros_like(p)
    ambiguous = np.zeros(p.shape, bool)
    for step, rec in enumerate(batches, 1):
        gw, gt, _ = g.gradients(rec)          # at the current parameters
        grad = np.concatenate([gw, gt]).astype(np.float64)
        # the gradient is an atomic sum: a second evaluation, in another
        # order, measures each component's rounding
        gw2, gt2, _ = g.gradients(rec)
        noise = np.abs(grad - np.concatenate([gw2, gt2]).astype(np.float64))
        g.train_records(rec, steps=1)         # the same gradient, then one Adam step
        want, m, v = R.adam_step(p, grad, m, v, step, lr)
        pw, pt = g.params()
        got = np.concatenate([pw, pt]).astype(np.float64)
        # train_records sums the gradient once more: a component whose sum is
        # within rounding of zero may take the other sign, and Adam (eps
        # 1e-15) turns that into a full step the other way, now and in every
        # later step through m; everything else moves as the formula says
        # (parameters no record touches have a gradient of exactly zero in
        # every sum, and Adam leaves them where m and v put them)
        touched = (grad != 0) | (noise != 0)
        ambiguous |= touched & (np.abs(grad) <= 8 * noise + 1e-7 * np.sqrt(np.mean(grad ** 2)))
        # From the second step on, m carries the first step's gradient too: a
        # component whose two steps nearly cancel in m is sensitive to the
        # rounding of both sums, which the noise test of one sum does not
        # see.  A wrong formula (moments, bias correction, eps) moves nearly
        # every component; these bounds leave room for the rounding only.
        err = np.abs(got - want)
        ok = err <= 1e-6 + 1e-5 * lr
        assert np.mean(ok[~ambiguous]) > 0.995, (step, np.quantile(err[~ambiguous], [0.5, 0.995]))
        assert np.mean(ok) > 0.99, (step, np.mean(ok), ambiguous.mean())
        moved = np.abs(want - p) > 0
        assert moved.mean() > 0.01
        p = got
