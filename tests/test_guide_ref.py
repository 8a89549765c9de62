"""The FP64 training reference of the learned guide (tests/guide_ref.py),
checked against central finite differences of its own loss: the analytic
output gradient of -w log(c g + (1 - c) b), and the backward pass through the
MLP and the hash-grid encoding into the weights and the table.  This pins
the reference that the GPU's tensor-core training kernel is compared with."""
import numpy as np

from tests import guide_ref as R


def _info(log2=10):
    return {"log2_table": log2, "grid_res": [4 + 3 * k for k in range(R.LEVELS)],
            "grid_lo": [-1.0, -1.0, -1.0], "grid_inv_extent": [0.5, 0.5, 0.5]}


def _records(rng, n):
    rec = np.zeros((n, 24))
    rec[:, :3] = rng.uniform(-1, 1, (n, 3))
    for a, b in ((3, 6), (6, 9), (10, 13)):
        d = rng.normal(size=(n, 3))
        rec[:, a:b] = d / np.linalg.norm(d, axis=1, keepdims=True)
    rec[:, 9] = rng.uniform(0, 1, n)
    rec[:, 13] = rng.uniform(0.05, 1.0, n)
    rec[:, 17] = rng.uniform(0, 2, n) * (rng.uniform(size=n) > 0.1)
    return rec


def _params(rng, info):
    w = np.concatenate([rng.normal(0, 1.5 / np.sqrt(fi), fo * fi)
                        for fo, fi in ((64, 112), (64, 64), (64, 64), (48, 64))])
    t = rng.uniform(-1, 1, R.LEVELS * (1 << info["log2_table"]) * 2)
    return w, t


def _loss(rec, w, t, info):
    o = R.forward(rec[:, :10], w, t, info)
    tw = rec[:, 17] / rec[:, 17].sum()
    return R.loss_and_output_grad(o, rec[:, 10:13], rec[:, 13], tw)[0]


def test_output_gradient_matches_finite_differences():
    rng = np.random.default_rng(1)
    n = 16
    o = rng.normal(0, 1, (n, 48))
    o[:, 3:40:5] = rng.uniform(-2, 3, (n, 8))  # log kappa inside the clamp
    rec = _records(rng, n)
    w = rec[:, 17] / rec[:, 17].sum()
    _, d = R.loss_and_output_grad(o, rec[:, 10:13], rec[:, 13], w)
    h = 1e-6
    for j in list(range(41)):
        e = np.zeros_like(o)
        e[:, j] = h
        lp = np.array([R.loss_and_output_grad(o[i:i + 1] + e[i:i + 1], rec[i:i + 1, 10:13], rec[i:i + 1, 13],
                                              w[i:i + 1])[0] for i in range(n)])
        lm = np.array([R.loss_and_output_grad(o[i:i + 1] - e[i:i + 1], rec[i:i + 1, 10:13], rec[i:i + 1, 13],
                                              w[i:i + 1])[0] for i in range(n)])
        fd = (lp - lm) / (2 * h)
        np.testing.assert_allclose(d[:, j], fd, rtol=1e-5, atol=1e-9, err_msg=f"output {j}")
    # unused outputs carry no gradient
    assert np.all(d[:, 41:] == 0)


def test_backward_matches_finite_differences():
    rng = np.random.default_rng(2)
    info = _info()
    rec = _records(rng, 256)
    w, t = _params(rng, info)
    gw, gt, loss = R.backward(rec, w, t, info, bf16_ops=False)
    assert np.isclose(loss, _loss(rec, w, t, info), rtol=1e-12)
    h = 1e-5
    errs = []
    for idx in rng.choice(len(w), 40, replace=False):
        e = np.zeros_like(w)
        e[idx] = h
        fd = (_loss(rec, w + e, t, info) - _loss(rec, w - e, t, info)) / (2 * h)
        errs.append(abs(fd - gw[idx]) / max(abs(fd), 1e-6))
    # a difference straddling a ReLU kink is rare; the bulk agrees to 1e-5
    assert np.median(errs) < 1e-5 and np.mean(np.array(errs) < 1e-3) > 0.9, errs
    touched = np.nonzero(gt)[0]
    assert len(touched) > 100
    errs = []
    for idx in rng.choice(touched, 40, replace=False):
        e = np.zeros_like(t)
        e[idx] = h
        fd = (_loss(rec, w, t + e, info) - _loss(rec, w, t - e, info)) / (2 * h)
        errs.append(abs(fd - gt[idx]) / max(abs(fd), 1e-6))
    assert np.median(errs) < 1e-5 and np.mean(np.array(errs) < 1e-3) > 0.9, errs


def test_adam_reference_first_step_is_signed_learning_rate():
    rng = np.random.default_rng(3)
    g = rng.normal(size=1000)
    g[::7] = 0
    p, m, v = R.adam_step(np.zeros(1000), g, np.zeros(1000), np.zeros(1000), 1, lr=1e-2)
    np.testing.assert_allclose(p, -1e-2 * np.sign(g), rtol=1e-9, atol=1e-12)
