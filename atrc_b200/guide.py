"""Learned path guiding (``atrc_guide_*`` of the C ABI).

    scene = DeviceScene(cfg)
    guide = Guide.for_scene(scene)
    stats = scene.render_guided(guide, desc, film, record=True)   # render + keep records
    guide.train(steps=4)                                          # Adam on the records
    scene.render_guided(guide, desc, film)                        # guided, no recording

The network runs on the tensor cores of the GPU that holds the scene; this
module only moves arrays across the C ABI.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np

from . import _abi as abi
from . import _check, load_library

RECORD_FLOATS = 24   # GuideRecord: pos 3, nrm 3, wo 3, rough, wi 3, pdf_bsdf, coef 3, target, l_arrive 3, prev, pad 2


def _fp(a: np.ndarray):
    return a.ctypes.data_as(abi.c_float_p)


class Guide:
    def __init__(self, lo, hi, device: int = 0, **desc_overrides):
        lib = load_library()
        d = abi.AtrcGuideDesc()
        _check(lib.atrc_guide_default_desc(C.byref(d)))
        for k, v in desc_overrides.items():
            setattr(d, k, v)
        self.desc = d
        lo = np.ascontiguousarray(lo, np.float32)
        hi = np.ascontiguousarray(hi, np.float32)
        h = C.c_void_p()
        _check(lib.atrc_guide_create(device, _fp(lo), _fp(hi), C.byref(d), C.byref(h)))
        self._h = h

    @classmethod
    def for_scene(cls, scene, **desc_overrides) -> "Guide":
        lo = np.zeros(3, np.float32)
        hi = np.zeros(3, np.float32)
        _check(load_library().atrc_cuda_scene_bounds(scene.handle, _fp(lo), _fp(hi)))
        return cls(lo, hi, device=scene.device, **desc_overrides)

    def close(self) -> None:
        if getattr(self, "_h", None):
            try:
                load_library().atrc_guide_destroy(self._h)
            except Exception:  # interpreter shutdown: the library is gone already
                pass
            self._h = None

    def __del__(self):
        self.close()

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    def set_max_select(self, max_select: float) -> None:
        """Cap on the selection probability for the renders that follow."""
        _check(load_library().atrc_guide_set_max_select(self._h, max_select))

    def info(self) -> dict:
        i = abi.AtrcGuideInfo()
        _check(load_library().atrc_guide_info(self._h, C.byref(i)))
        out = {k: getattr(i, k) for k, _ in abi.AtrcGuideInfo._fields_ if not k.startswith("pad")}
        out["grid_lo"] = list(i.grid_lo)
        out["grid_inv_extent"] = list(i.grid_inv_extent)
        out["grid_res"] = list(i.grid_res)
        return out

    def params(self) -> tuple[np.ndarray, np.ndarray]:
        inf = self.info()
        w = np.empty(inf["weights"], np.float32)
        t = np.empty(inf["table_floats"], np.float32)
        _check(load_library().atrc_guide_params(self._h, _fp(w), _fp(t), 0))
        return w, t

    def set_params(self, weights: Optional[np.ndarray] = None, table: Optional[np.ndarray] = None) -> None:
        w = None if weights is None else np.ascontiguousarray(weights, np.float32)
        t = None if table is None else np.ascontiguousarray(table, np.float32)
        _check(load_library().atrc_guide_params(self._h, None if w is None else _fp(w),
                                               None if t is None else _fp(t), 1))

    def eval_raw(self, queries: np.ndarray) -> np.ndarray:
        q = np.ascontiguousarray(queries, np.float32).reshape(-1, 10)
        out = np.empty((len(q), 48), np.float32)
        _check(load_library().atrc_guide_eval(self._h, _fp(q), len(q), _fp(out)))
        return out

    def pdf(self, queries: np.ndarray, dirs: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
        """Mixture pdf of each direction at its query and the selection
        probability, computed on the GPU as the renderer does."""
        q = np.ascontiguousarray(queries, np.float32).reshape(-1, 10)
        d = np.ascontiguousarray(dirs, np.float32).reshape(-1, 3)
        p = np.empty(len(q), np.float32)
        c = np.empty(len(q), np.float32)
        _check(load_library().atrc_guide_pdf(self._h, _fp(q), _fp(d), len(q), _fp(p), _fp(c)))
        return p, c

    def train(self, steps: int = 1) -> float:
        loss = C.c_float()
        _check(load_library().atrc_guide_train(self._h, steps, C.byref(loss)))
        return loss.value

    def train_records(self, records: np.ndarray, steps: int = 1) -> float:
        r = np.ascontiguousarray(records, np.float32).reshape(-1, RECORD_FLOATS)
        loss = C.c_float()
        _check(load_library().atrc_guide_train_records(self._h, _fp(r), len(r), steps, C.byref(loss)))
        return loss.value

    def gradients(self, records: np.ndarray) -> tuple[np.ndarray, np.ndarray, float]:
        """Loss gradients of the weights and the table over `records` at the
        current parameters (atrc_guide_gradients: no Adam step)."""
        r = np.ascontiguousarray(records, np.float32).reshape(-1, RECORD_FLOATS)
        inf = self.info()
        gw = np.empty(inf["weights"], np.float32)
        gt = np.empty(inf["table_floats"], np.float32)
        loss = C.c_float()
        _check(load_library().atrc_guide_gradients(self._h, _fp(r), len(r), _fp(gw), _fp(gt), C.byref(loss)))
        return gw, gt, loss.value

    def records(self) -> np.ndarray:
        n = C.c_size_t()
        lib = load_library()
        _check(lib.atrc_guide_records(self._h, None, 0, C.byref(n)))
        out = np.empty((n.value, RECORD_FLOATS), np.float32)
        if n.value:
            _check(lib.atrc_guide_records(self._h, _fp(out), n.value, C.byref(n)))
        return out


def rel_mse(image, reference, ref_var=None) -> float:
    """Mean over pixels and channels of (I - R)^2 / (R^2 + 1e-2) (torch or
    numpy).  With `ref_var`, the variance of the reference's per-pixel mean,
    the reference's own noise is taken out: E[(I - R)^2] = (E I - mu)^2 +
    Var I + Var R, so subtracting Var R estimates the error against the
    converged image."""
    d = image - reference
    e = d * d
    if ref_var is not None:
        e = e - ref_var
    return float((e / (reference * reference + 1e-2)).mean())


def time_to(curve, target: float) -> Optional[float]:
    """First time a (time, spp, relMSE) curve reaches `target`,
    interpolated log-log between checkpoints."""
    prev = None
    for t, _, e in curve:
        if e <= target:
            if prev is None or prev[1] <= 0 or e <= 0:
                return t
            t0, e0 = prev
            a = (np.log(target) - np.log(e0)) / (np.log(e) - np.log(e0))
            return float(np.exp(np.log(t0) + a * (np.log(t) - np.log(t0))))
        prev = (t, e)
    return None


def render_budget(scene, desc, seconds: float, guide: Optional[Guide] = None, train_fraction: float = 0.25,
                  train_steps: int = 4, spp_per_pass: int = 1, reference=None, checkpoints=(), first_spp: int = 0,
                  ref_var=None, stop_at: Optional[float] = None, warmup: bool = True,
                  select_after: Optional[float] = None):
    """Render passes of `spp_per_pass` samples per pixel into one device film
    until `seconds` of render time have passed.  With a guide, the passes of
    the first `train_fraction` of the budget record training data and run
    `train_steps` Adam steps after each pass; later passes only sample with
    the guide.  The clock runs only inside the render / training calls (the
    calls are synchronous), so the relMSE checkpoints against `reference`
    (a torch CUDA tensor H x W x 3) cost nothing.  With `warmup`, untimed
    passes into a scratch film first do the one-time set-up of the render
    calls the loop makes (graph capture, the guide's per-path buffers); they
    neither record training data that is used nor train, and their samples
    are dropped.  `select_after`, if given, becomes the guide's selection
    cap once training ends.  Returns the film, the (time, spp, relMSE)
    checkpoints and per-phase times."""
    import time

    import torch

    from . import Film
    film = Film(desc.width, desc.height, device=True)
    desc.spp_count = spp_per_pass
    if warmup:
        scratch = Film(desc.width, desc.height, device=True)
        desc.first_spp = first_spp + (1 << 24)
        if guide is None:
            scene.render(desc, scratch)
        else:
            # a recording render's records are replaced by the next one's
            if train_fraction > 0:
                scene.render_guided(guide, desc, scratch, record=True)
            scene.render_guided(guide, desc, scratch, record=False)
        torch.cuda.synchronize()
        del scratch
    elapsed = t_render = t_train = 0.0
    passes = 0
    curve = []
    pending = sorted(checkpoints)
    stopped = False
    raised = False
    while elapsed < seconds and not stopped:
        desc.first_spp = first_spp + passes * spp_per_pass
        training = guide is not None and elapsed < train_fraction * seconds
        if guide is not None and not training and select_after is not None and not raised:
            guide.set_max_select(select_after)
            raised = True
        t0 = time.perf_counter()
        if guide is None:
            scene.render(desc, film)
        else:
            scene.render_guided(guide, desc, film, record=training)
        t1 = time.perf_counter()
        if training:
            guide.train(steps=train_steps)
        t2 = time.perf_counter()
        t_render += t1 - t0
        t_train += t2 - t1
        elapsed += t2 - t0
        passes += 1
        while reference is not None and pending and elapsed >= pending[0]:
            pending.pop(0)
            img = (film.value.view(desc.height, desc.width, 3) /
                   film.weight.view(desc.height, desc.width, 1).clamp_min(1e-30))
            curve.append((elapsed, passes * spp_per_pass, rel_mse(img.float(), reference, ref_var)))
            if stop_at is not None and curve[-1][2] <= stop_at:
                stopped = True
    torch.cuda.synchronize()
    final = None
    if reference is not None:
        img = film.value.view(desc.height, desc.width, 3) / film.weight.view(desc.height, desc.width, 1).clamp_min(1e-30)
        final = rel_mse(img.float(), reference, ref_var)
        curve.append((elapsed, passes * spp_per_pass, final))
    return {"film": film, "seconds": elapsed, "render_s": t_render, "train_s": t_train, "spp": passes * spp_per_pass,
            "curve": curve, "rel_mse": final}
