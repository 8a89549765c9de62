"""FP64 NumPy evaluation of the learned guide, from the same parameters the
GPU holds: hash-grid and one-blob encodings, the 112-64-64-64-48 ReLU MLP,
the vMF-mixture decoding and pdf.  ``bf16=True`` rounds the inputs, weights
and hidden activations to BF16 as the tensor-core kernels do, so that the
GPU must match it to FP32 accumulation order."""
from __future__ import annotations

import numpy as np

LEVELS = 16
IN, HID, OUT, LOBES = 112, 64, 48, 8
MAX_SELECT = 0.9      # the selection cap the tests give their guides (AtrcGuideDesc.max_select)
SELECT_OFFSET = -2.0
LOG_KAPPA = (-6.9, 9.2)


def bf16(x: np.ndarray) -> np.ndarray:
    """Round float values to the nearest BF16 (ties to even), as float64."""
    f = np.asarray(x, np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def split_weights(w: np.ndarray):
    o1 = HID * IN
    o2 = o1 + HID * HID
    o3 = o2 + HID * HID
    return (w[:o1].reshape(HID, IN), w[o1:o2].reshape(HID, HID), w[o2:o3].reshape(HID, HID),
            w[o3:o3 + OUT * HID].reshape(OUT, HID))


def hash_slot(res: int, log2: int, x, y, z):
    n = res + 1
    if n ** 3 <= (1 << log2):
        return (x + n * (y + n * z)).astype(np.uint64)
    h = (x.astype(np.uint64) * np.uint64(1)) ^ (y.astype(np.uint64) * np.uint64(2654435761)) ^ \
        (z.astype(np.uint64) * np.uint64(805459861))
    return (h & np.uint64(0xFFFFFFFF)) & np.uint64((1 << log2) - 1)


def encode(queries: np.ndarray, table: np.ndarray, info: dict) -> np.ndarray:
    """queries (n, 10) -> inputs (n, 112)."""
    q = np.asarray(queries, np.float64)
    n = len(q)
    log2 = info["log2_table"]
    lo = np.asarray(info["grid_lo"], np.float64)
    ie = np.asarray(info["grid_inv_extent"], np.float64)
    p01 = np.clip((q[:, :3] - lo) * ie, 0, 1)
    tab = np.asarray(table, np.float64).reshape(LEVELS, 1 << log2, 2)
    x = np.zeros((n, IN))
    for lv in range(LEVELS):
        res = info["grid_res"][lv]
        s = p01 * res
        fl = np.minimum(np.floor(s), res - 1)
        f = s - fl
        i0 = fl.astype(np.int64)
        acc = np.zeros((n, 2))
        for k in range(8):
            d = np.array([k & 1, (k >> 1) & 1, k >> 2])
            slot = hash_slot(res, log2, i0[:, 0] + d[0], i0[:, 1] + d[1], i0[:, 2] + d[2])
            w = np.prod(np.where(d == 1, f, 1 - f), axis=1)
            acc += w[:, None] * tab[lv][slot.astype(np.int64)]
        x[:, 2 * lv:2 * lv + 2] = acc

    def blob(s):
        c = np.clip(s, 0, 1)[:, None] * 16
        return np.maximum(0, 1 - np.abs(c - (np.arange(16) + 0.5)))

    def dirb(d):
        return np.concatenate([blob(0.5 * (np.clip(d[:, 2], -1, 1) + 1)),
                               blob((np.arctan2(d[:, 1], d[:, 0]) + np.pi) / (2 * np.pi))], 1)
    x[:, 32:64] = dirb(q[:, 3:6])
    x[:, 64:96] = dirb(q[:, 6:9])
    x[:, 96] = q[:, 9]
    return x


def forward(queries, weights, table, info, bf16_ops: bool = False) -> np.ndarray:
    x = encode(queries, table, info)
    W = [np.asarray(m, np.float64) for m in split_weights(np.asarray(weights, np.float64))]
    rnd = bf16 if bf16_ops else (lambda a: a)
    h = rnd(x)
    for li, m in enumerate(W):
        z = h @ rnd(m).T
        h = rnd(np.maximum(z, 0)) if li < 3 else z
    return h


def decode(raw: np.ndarray):
    o = np.asarray(raw, np.float64)
    mu = o[:, :40].reshape(-1, LOBES, 5)[:, :, :3]
    mu = mu / np.maximum(np.linalg.norm(mu, axis=2, keepdims=True), 1e-30)
    kappa = np.exp(np.clip(o[:, 3:40:5], *LOG_KAPPA))
    logit = o[:, 4:40:5]
    w = np.exp(logit - logit.max(1, keepdims=True))
    w /= w.sum(1, keepdims=True)
    c = MAX_SELECT / (1 + np.exp(-(o[:, 40] + SELECT_OFFSET)))
    return mu, kappa, w, c


def pdf(raw: np.ndarray, dirs: np.ndarray) -> np.ndarray:
    mu, kappa, w, _ = decode(raw)
    cs = np.einsum("nkj,nj->nk", mu, np.asarray(dirs, np.float64))
    norm = kappa / (2 * np.pi * -np.expm1(-2 * kappa))
    return np.sum(w * norm * np.exp(kappa * (cs - 1)), axis=1)


# ------------------------------------------------------------------ training
# GuideRecord fields (24 floats): pos 0:3, nrm 3:6, wo 6:9, rough 9, wi 10:13,
# pdf_bsdf 13, coef 14:17, target 17, l_arrive 18:21, prev 21, pad 22:24.

def loss_and_output_grad(o: np.ndarray, wi: np.ndarray, pdf_bsdf: np.ndarray, w: np.ndarray):
    """Loss sum_i -w_i log(c_i g_i + (1 - c_i) b_i) of the raw outputs o (n, 48)
    and its gradient with respect to o, in FP64 by the chain rule: g is the
    vMF mixture at wi, b the BSDF pdf, c the selection probability.  Records
    with w <= 0 or q <= 1e-20 contribute nothing; log kappa has no gradient
    where it is clamped."""
    o = np.asarray(o, np.float64)
    n = len(o)
    x = o[:, :40].reshape(n, LOBES, 5)
    m = x[:, :, :3]
    ln = np.linalg.norm(m, axis=2)
    mu = np.where(ln[..., None] > 1e-10, m / np.maximum(ln, 1e-300)[..., None], [0.0, 0.0, 1.0])
    lk = x[:, :, 3]
    kap = np.exp(np.clip(lk, *LOG_KAPPA))
    lg = x[:, :, 4]
    pi = np.exp(lg - lg.max(1, keepdims=True))
    pi /= pi.sum(1, keepdims=True)
    sig = 1 / (1 + np.exp(-(o[:, 40] + SELECT_OFFSET)))
    c = MAX_SELECT * sig
    wi = np.asarray(wi, np.float64)
    cs = np.einsum("nkj,nj->nk", mu, wi)
    v = kap / (2 * np.pi * -np.expm1(-2 * kap)) * np.exp(kap * (cs - 1))
    g = np.sum(pi * v, axis=1)
    b = np.asarray(pdf_bsdf, np.float64)
    q = c * g + (1 - c) * b
    w = np.asarray(w, np.float64)
    ok = (w > 0) & (q > 1e-20)
    loss = float(np.sum(np.where(ok, -w * np.log(np.where(ok, q, 1)), 0)))
    dq = np.where(ok, -w / np.where(ok, q, 1), 0)                # d loss / d q
    d = np.zeros_like(o)
    d[:, 40] = dq * (g - b) * MAX_SELECT * sig * (1 - sig)       # q = c g + (1 - c) b, c = 0.9 sigmoid
    dg = dq * c                                                   # d loss / d g
    dv = dg[:, None] * pi                                         # d loss / d v_k
    d[:, 4:40:5] = dg[:, None] * pi * (v - g[:, None])            # softmax
    # v = N(kappa) exp(kappa (cs - 1)), N = kappa / (2 pi (1 - e^-2kappa)):
    # d v / d log kappa = v (1 - 2 kappa / (e^2kappa - 1) + kappa (cs - 1))
    dlogn = 1 - 2 * kap / np.expm1(2 * kap)
    inside = (lk > LOG_KAPPA[0]) & (lk < LOG_KAPPA[1])
    d[:, 3:40:5] = np.where(inside, dv * v * (dlogn + kap * (cs - 1)), 0)
    # mu = m / |m|: d cs / d m = (wi - cs mu) / |m|
    dm = np.where(ln[..., None] > 1e-10,
                  (dv * v * kap / np.maximum(ln, 1e-300))[..., None] * (wi[:, None, :] - cs[..., None] * mu), 0)
    for j in range(3):
        d[:, j:40:5] = dm[:, :, j]
    return loss, d


def hash_corners(queries: np.ndarray, info: dict, level: int):
    """Table slots (n, 8) and trilinear weights (n, 8) of one level."""
    q = np.asarray(queries, np.float64)
    lo = np.asarray(info["grid_lo"], np.float64)
    ie = np.asarray(info["grid_inv_extent"], np.float64)
    s = np.clip((q[:, :3] - lo) * ie, 0, 1) * info["grid_res"][level]
    fl = np.minimum(np.floor(s), info["grid_res"][level] - 1)
    f = s - fl
    i0 = fl.astype(np.int64)
    slots, ws = [], []
    for k in range(8):
        dd = np.array([k & 1, (k >> 1) & 1, k >> 2])
        slots.append(hash_slot(info["grid_res"][level], info["log2_table"], i0[:, 0] + dd[0], i0[:, 1] + dd[1],
                               i0[:, 2] + dd[2]).astype(np.int64))
        ws.append(np.prod(np.where(dd == 1, f, 1 - f), axis=1))
    return np.stack(slots, 1), np.stack(ws, 1)


def backward(records: np.ndarray, weights: np.ndarray, table: np.ndarray, info: dict, bf16_ops: bool = True):
    """Loss over a batch of records, normalised by the sum of their targets,
    and its gradients with respect to the packed weights and the table.
    With bf16_ops the operands are rounded to BF16 where the tensor-core
    training kernel rounds them: the encoded inputs, the weights, the hidden
    activations and each layer's output gradient; sums stay in FP64."""
    rec = np.asarray(records, np.float64)
    rnd = bf16 if bf16_ops else (lambda a: a)
    x = encode(rec[:, :10], table, info)
    W = [np.asarray(mm, np.float64) for mm in split_weights(np.asarray(weights, np.float64))]
    Wb = [rnd(mm) for mm in W]
    xb = rnd(x)
    z1 = xb @ Wb[0].T
    h1 = rnd(np.maximum(z1, 0))
    z2 = h1 @ Wb[1].T
    h2 = rnd(np.maximum(z2, 0))
    z3 = h2 @ Wb[2].T
    h3 = rnd(np.maximum(z3, 0))
    o = h3 @ Wb[3].T
    t = rec[:, 17]
    w = t / t.sum() if t.sum() > 0 else np.zeros_like(t)
    loss, d4 = loss_and_output_grad(o, rec[:, 10:13], rec[:, 13], w)
    d4 = rnd(d4)
    d3 = rnd((d4 @ Wb[3]) * (z3 > 0))
    d2 = rnd((d3 @ Wb[2]) * (z2 > 0))
    d1 = rnd((d2 @ Wb[1]) * (z1 > 0))
    gw = np.concatenate([(d1.T @ xb).ravel(), (d2.T @ h1).ravel(), (d3.T @ h2).ravel(), (d4.T @ h3).ravel()])
    dx = d1 @ Wb[0][:, :2 * LEVELS]
    log2 = info["log2_table"]
    gt = np.zeros((LEVELS, 1 << log2, 2))
    for lv in range(LEVELS):
        slots, ws = hash_corners(rec[:, :10], info, lv)
        for k in range(8):
            np.add.at(gt[lv], slots[:, k], ws[:, k:k + 1] * dx[:, 2 * lv:2 * lv + 2])
    return gw, gt.ravel(), loss


def adam_step(p, g, m, v, step: int, lr: float, b1: float = 0.9, b2: float = 0.99, eps: float = 1e-15):
    """One Adam update (Kingma and Ba 2015) with bias correction at step
    `step` (1-based); returns the new (p, m, v)."""
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    p = p - lr * (m / (1 - b1 ** step)) / (np.sqrt(v / (1 - b2 ** step)) + eps)
    return p, m, v
