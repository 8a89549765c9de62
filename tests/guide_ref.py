"""FP64 NumPy evaluation of the learned guide, from the same parameters the
GPU holds: hash-grid and one-blob encodings, the 112-64-64-64-48 ReLU MLP,
the vMF-mixture decoding and pdf.  ``bf16=True`` rounds the inputs, weights
and hidden activations to BF16 as the tensor-core kernels do, so that the
GPU must match it to FP32 accumulation order."""
from __future__ import annotations

import numpy as np

LEVELS = 16
IN, HID, OUT, LOBES = 112, 64, 48, 8
MAX_SELECT = 0.9
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
