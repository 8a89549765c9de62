"""The guided benchmark's metric on CPU: relMSE against a reference image
(with the reference's own noise taken out) and the time a (time, spp,
relMSE) curve first reaches a target, interpolated log-log."""
import math

import numpy as np

from atrc_b200.guide import rel_mse, time_to


def test_rel_mse_definition():
    rng = np.random.default_rng(5)
    ref = rng.uniform(0.0, 3.0, (4, 6, 3))
    img = ref + rng.normal(0.0, 0.1, ref.shape)
    want = np.mean((img - ref) ** 2 / (ref * ref + 1e-2))
    assert math.isclose(rel_mse(img, ref), want, rel_tol=1e-12)
    # the reference's variance is subtracted pixel by pixel before the ratio
    var = np.full(ref.shape, 1e-3)
    want_v = np.mean(((img - ref) ** 2 - var) / (ref * ref + 1e-2))
    assert math.isclose(rel_mse(img, ref, var), want_v, rel_tol=1e-12)
    assert rel_mse(ref, ref) == 0.0


def test_rel_mse_noise_correction_is_unbiased():
    # E[(I - R)^2] = Var I + Var R for unbiased I, R around the same mean:
    # subtracting Var R leaves Var I, the error against the converged image
    rng = np.random.default_rng(7)
    mu = np.full((256, 256, 3), 2.0)
    s_i, s_r = 0.05, 0.08
    img = mu + rng.normal(0.0, s_i, mu.shape)
    ref = mu + rng.normal(0.0, s_r, mu.shape)
    got = rel_mse(img, ref, np.full(mu.shape, s_r * s_r))
    want = s_i * s_i / (4.0 + 1e-2)
    assert abs(got - want) < 0.1 * want


def test_time_to_power_law_interpolation():
    # relMSE falling as 1/t: log-log interpolation between checkpoints is exact
    curve = [(t, int(10 * t), 1e-2 / t) for t in (0.5, 1.0, 2.0, 4.0)]
    assert math.isclose(time_to(curve, 1e-2 / 3.0), 3.0, rel_tol=1e-12)
    assert math.isclose(time_to(curve, 1e-2 / 1.5), 1.5, rel_tol=1e-12)


def test_time_to_edges():
    curve = [(0.25, 4, 1e-3), (0.5, 8, 5e-4)]
    assert time_to(curve, 2e-3) == 0.25          # reached at the first checkpoint
    assert time_to(curve, 1e-3) == 0.25          # reached exactly
    assert time_to(curve, 1e-4) is None          # never reached
    assert time_to([], 1e-3) is None
    # a checkpoint with zero error stops the interpolation at its own time
    assert time_to([(1.0, 1, 1e-2), (2.0, 2, 0.0)], 1e-3) == 2.0
