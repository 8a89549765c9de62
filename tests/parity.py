"""Helpers shared by the parity tests: seeded ray sets, hit comparison with
mismatch classification, and the per-pixel 3-sigma band test."""
from __future__ import annotations

import math

import numpy as np

from atrc_b200 import RAY_DTYPE


def seeded_rays(n: int, lo, hi, cam_pos, seed: int) -> np.ndarray:
    """Half camera-like rays (from cam_pos towards uniform points of the box),
    half rays with origins uniform in the box and uniform directions."""
    rng = np.random.default_rng(seed)
    lo, hi = np.asarray(lo, np.float64), np.asarray(hi, np.float64)
    r = np.zeros(n, dtype=RAY_DTYPE)
    h = n // 2
    tgt = rng.uniform(lo, hi, (h, 3))
    o = np.broadcast_to(np.asarray(cam_pos, np.float64), (h, 3))
    d = tgt - o
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r["o"][:h] = o
    r["d"][:h] = d
    o2 = rng.uniform(lo, hi, (n - h, 3))
    d2 = rng.normal(size=(n - h, 3))
    d2 /= np.linalg.norm(d2, axis=1, keepdims=True)
    r["o"][h:] = o2
    r["d"][h:] = d2
    r["t_min"] = 0
    r["t_max"] = np.inf
    return r


def ulp_diff(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    ai = np.asarray(a, np.float32).view(np.int32).astype(np.int64)
    bi = np.asarray(b, np.float32).view(np.int32).astype(np.int64)
    ai = np.where(ai < 0, -(ai & 0x7FFFFFFF), ai)
    bi = np.where(bi < 0, -(bi & 0x7FFFFFFF), bi)
    return np.abs(ai - bi)


def classify_closest(rays, gpu, ref, oracle_scene, watertight: bool = False):
    """Returns counts: exact (same primitive, t within 2 ulp), tie, ref_fn
    (the reference BVH missed a closer genuine hit, confirmed by the oracle's
    test of that one primitive: Moller-Trumbore, or the watertight test with
    `watertight`), error."""
    same_prim = (gpu["entity"] == ref["entity"]) & (gpu["prim"] == ref["prim"])
    both_miss = (gpu["entity"] < 0) & (ref["entity"] < 0)
    ok_t = ulp_diff(gpu["t"], ref["t"]) <= 2
    exact = both_miss | (same_prim & ok_t)
    out = {"exact": int(exact.sum()), "tie": 0, "ref_fn": 0, "error": 0, "max_ulp_same_prim": 0, "errors": []}
    sp = same_prim & ~both_miss
    if sp.any():
        out["max_ulp_same_prim"] = int(ulp_diff(gpu["t"][sp], ref["t"][sp]).max())
    for i in np.nonzero(~exact)[0]:
        g, r = gpu[i], ref[i]
        if g["entity"] >= 0 and r["entity"] >= 0 and ulp_diff(g["t"], r["t"]) <= 2:
            out["tie"] += 1
            continue
        if g["entity"] >= 0 and (r["entity"] < 0 or g["t"] < r["t"]):
            t = oracle_scene.prim_hit(rays[i], int(g["entity"]), int(g["prim"]), watertight=watertight)
            if t >= 0 and ulp_diff(t, g["t"]) <= 2:
                out["ref_fn"] += 1
                continue
        out["error"] += 1
        if len(out["errors"]) < 10:
            out["errors"].append((int(i), tuple(g.tolist()), tuple(r.tolist())))
    return out


def band_test(gpu_film, ref_film, filter_value: float, sigmas: float = 3.0, cluster: int = 1):
    """Per-pixel, per-channel |mu_g - mu_c| <= k sqrt(s_g^2/N_g + s_c^2/N_c).
    Returns (failing fraction, allowed fraction, details).

    `cluster` = 3 treats the three channels of a pixel as one draw (they
    share every path, so they tend to fail together), which widens the
    binomial margin by sqrt(3).

    With the variances estimated from the samples, the statistic of a pixel
    follows Student's t with the Welch-Satterthwaite degrees of freedom, not
    a normal law: at 64 samples per pixel P(|t| > 3) is about 0.0033 instead
    of 0.0027.  The allowed fraction is therefore the mean of the per-test
    t tail probabilities (0 where both variances are 0, since such a test
    cannot fail) plus the binomial 99.9 % margin."""
    def stats(f):
        w = f.weight.reshape(-1, 1)
        mu = f.value.reshape(-1, 3) / np.where(w > 0, w, 1)
        m2 = f.value_sq.reshape(-1, 3) / np.where(w > 0, w, 1)
        var = np.maximum(m2 - mu * mu, 0)
        n = w / filter_value
        return mu, var, n

    mg, vg, ng = stats(gpu_film)
    mc, vc, nc = stats(ref_film)
    se = np.sqrt(vg / np.maximum(ng, 1) + vc / np.maximum(nc, 1))
    diff = np.abs(mg - mc)
    fail = diff > sigmas * se + 1e-6 * (np.abs(mg) + np.abs(mc))
    tests = fail.size
    from scipy.stats import t as student_t
    a = vg / np.maximum(ng, 1)
    b = vc / np.maximum(nc, 1)
    den = a * a / np.maximum(ng - 1, 1) + b * b / np.maximum(nc - 1, 1)
    dof = np.where(den > 0, (a + b) ** 2 / np.where(den > 0, den, 1), np.inf)
    p_each = np.where(se > 0, 2 * student_t.sf(sigmas, np.broadcast_to(dof, se.shape)), 0.0)
    p = float(p_each.mean())
    allowed = p + 3.1 * math.sqrt(p * (1 - p) * cluster / tests)  # binomial upper 99.9 % bound
    return float(fail.mean()), allowed, {"max_z": float(np.max(diff / np.maximum(se, 1e-12))),
                                         "mean_rel": float(np.mean(np.abs(mg - mc)) / max(np.mean(np.abs(mc)), 1e-12))}


def global_mean_z(gpu_film, ref_film, filter_value: float = 1 / (4 * (0.5 - 3e-4) ** 2)) -> float:
    """z-score (largest over channels) of the difference between the two
    whole-image mean radiances; each sample is one draw of the image-wide
    sample distribution (box filter, one pixel per sample)."""
    def agg(f):
        wsum = float(f.weight.sum())
        mu = f.value.reshape(-1, 3).sum(0) / wsum
        m2 = f.value_sq.reshape(-1, 3).sum(0) / wsum
        return mu, np.maximum(m2 - mu * mu, 0), wsum / filter_value
    mg, vg, ng = agg(gpu_film)
    mc, vc, nc = agg(ref_film)
    se = np.sqrt(vg / ng + vc / nc)
    return float(np.max(np.abs(mg - mc) / np.maximum(se, 1e-30)))


def filter_weight_moments(n: int, radius: float, alpha: float, grid: int = 32, m: int = 4096):
    """1D moments of the Gaussian filter's splat weight along one film axis,
    under the reference's tiled splat (render_target.h:355-395,
    framebuffer.h:36-80): each tile of `grid` pixels samples its bound grown
    by the radius and splats only into itself, stepping the distance by one
    pixel from the tile-clamped first pixel.  Jitter is integrated with the
    midpoint rule over `m` points.  Returns per pixel (sum E[g], sum E[g^2],
    sum E[g]^2) over the sample pixels that reach it; the 2D weight of one
    sample per sample pixel is g(x) g(y), so E[w] = spp m1x m1y and
    Var[w] = spp (s2x s2y - qx qy)."""
    r = np.float32(radius)
    er = math.exp(-alpha * float(r) * float(r))
    m1, s2, q = np.zeros(n), np.zeros(n), np.zeros(n)
    jit = (np.arange(m) + 0.5) / m
    for a0 in range(0, n, grid):
        a1 = min(n, a0 + grid) - 1
        s0 = int(np.floor(np.float32(a0) + np.float32(0.5) - r))
        s1 = int(np.floor(np.float32(a1) + np.float32(0.49999) + r))
        for X in range(s0, s1 + 1):
            sx = (np.float32(X) + jit.astype(np.float32)).astype(np.float32)
            xmin = np.maximum(a0, np.ceil(sx - r - np.float32(0.5)).astype(np.int64))
            xmax = np.minimum(a1, np.floor(sx + r - np.float32(0.5)).astype(np.int64))
            xr = np.abs((xmin + np.float32(0.5)).astype(np.float32) - sx)
            for k in range(int(xmax.max() - xmin.min()) + 1):
                x = xmin + k
                live = (x <= xmax) & (xr <= r)
                g = np.where(live, np.maximum(0.0, np.exp(-alpha * xr.astype(np.float64) ** 2) - er), 0.0)
                for px in np.unique(x[live]):
                    sel = x == px
                    gsel = np.where(sel, g, 0.0)
                    e1 = gsel.sum() / m
                    m1[px] += e1
                    s2[px] += (gsel ** 2).sum() / m
                    q[px] += e1 * e1
                xr = xr + np.float32(1)
    return m1, s2, q


def filter_weight_z(weight: np.ndarray, width: int, height: int, spp: int, radius: float, alpha: float,
                    grid: int = 32) -> np.ndarray:
    """Per-pixel z-scores of a film's Gaussian-filter weights against their
    expectation under the reference's tiled splat."""
    mx, sx, qx = filter_weight_moments(width, radius, alpha, grid)
    my, sy, qy = filter_weight_moments(height, radius, alpha, grid)
    mean = spp * np.outer(my, mx)
    var = spp * (np.outer(sy, sx) - np.outer(qy, qx))
    return (np.asarray(weight).reshape(height, width) - mean) / np.sqrt(np.maximum(var, 1e-300))
