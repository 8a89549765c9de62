"""atrc_b200 -- B200-native `pt_cuda` renderer for Atrc scenes.

Python plumbing over the C ABI of ``libatrc_cuda.so`` (``include/atrc_cuda.h``):
load an Atrc JSON scene, upload it, trace ray batches and render.  The
compute runs in the library's sm_100a kernels; there is no CPU fallback --
every entry point raises if the native library is missing or no GPU is
present.

    cfg = Config.from_file("scene.json")
    scene = DeviceScene(cfg)              # BVH build + upload
    desc, kind = cfg.rendering(0)         # `pt` / `pt_cuda` settings
    film = Film(desc.width, desc.height)
    stats = scene.render(desc, film)
    rgb = film.image()                    # value / weight, (H, W, 3)
"""
from __future__ import annotations

import ctypes as C
import json
import os
from pathlib import Path
from typing import Callable, Optional

import numpy as np

from . import _abi as abi
from ._abi import AtrcRenderDesc, AtrcRenderStats, AtrcFilm

__all__ = ["AtrcError", "load_library", "library_path", "Config", "DeviceScene", "Film", "RAY_DTYPE", "HIT_DTYPE",
           "ERROR_NAMES"]

ROOT = Path(__file__).resolve().parent
LIB_PATH = Path(os.environ.get("ATRC_LIB", ROOT / "lib" / "libatrc_cuda.so"))

ERROR_NAMES = {0: "ATRC_OK", -1: "ATRC_ERR_INVALID_ARG", -2: "ATRC_ERR_CONFIG", -3: "ATRC_ERR_OUT_OF_MEMORY",
               -4: "ATRC_ERR_CUDA", -5: "ATRC_ERR_CANCELLED", -6: "ATRC_ERR_WATCHDOG", -7: "ATRC_ERR_UNSUPPORTED"}

RAY_DTYPE = np.dtype([("o", "<f4", 3), ("t_min", "<f4"), ("d", "<f4", 3), ("t_max", "<f4")])
HIT_DTYPE = np.dtype([("t", "<f4"), ("entity", "<i4"), ("prim", "<i4"), ("u", "<f4")])


class AtrcError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"{ERROR_NAMES.get(code, code)}: {message}")
        self.code = code


_lib: Optional[C.CDLL] = None


def library_path() -> Path:
    return LIB_PATH


def load_library() -> C.CDLL:
    """Load libatrc_cuda.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m atrc_b200.build`")
    lib = C.CDLL(str(LIB_PATH))
    for name, (res, args) in abi.PROTOTYPES.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    n = len(abi.STRUCT_ORDER)
    sizes = (C.c_uint64 * n)()
    if lib.atrc_abi_struct_sizes(sizes, n) != n:
        raise RuntimeError("ABI mismatch: the library describes a different set of structs")
    for cls, sz in zip(abi.STRUCT_ORDER, sizes):
        if C.sizeof(cls) != sz:
            raise RuntimeError(f"ABI mismatch for {cls.__name__}: python {C.sizeof(cls)} vs library {sz}")
    _lib = lib
    return lib


def _check(rc: int) -> None:
    if rc != 0:
        msg = load_library().atrc_last_error()
        raise AtrcError(rc, msg.decode() if msg else "")


class Config:
    """A parsed Atrc configuration ({"scene": ..., "rendering": ...})."""

    def __init__(self, handle: C.c_void_p, keepalive=None):
        self._h = handle
        self._keep = keepalive

    @classmethod
    def from_file(cls, path: str | os.PathLike) -> "Config":
        lib = load_library()
        h = C.c_void_p()
        _check(lib.atrc_config_load_file(str(path).encode(), C.byref(h)))
        return cls(h)

    @classmethod
    def from_string(cls, text: str | dict, scene_dir: str | os.PathLike = ".") -> "Config":
        lib = load_library()
        if isinstance(text, dict):
            text = json.dumps(text)
        h = C.c_void_p()
        _check(lib.atrc_config_load_string(text.encode(), str(scene_dir).encode(), C.byref(h)))
        return cls(h)

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.atrc_config_destroy(self._h)
            self._h = None

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    def scene_desc(self) -> C.POINTER(abi.AtrcSceneDesc):
        p = C.POINTER(abi.AtrcSceneDesc)()
        _check(load_library().atrc_config_scene(self._h, C.byref(p)))
        p._owner = self  # the description lives in this config's memory
        return p

    def rendering_count(self) -> int:
        n = C.c_int()
        _check(load_library().atrc_config_rendering_count(self._h, C.byref(n)))
        return n.value

    def rendering(self, index: int = 0) -> tuple[AtrcRenderDesc, str]:
        d = AtrcRenderDesc()
        buf = C.create_string_buffer(64)
        _check(load_library().atrc_config_rendering(self._h, index, C.byref(d), buf, 64))
        return d, buf.value.decode()

    def post_processors(self, index: int = 0) -> list:
        lib = load_library()
        need = C.c_size_t()
        _check(lib.atrc_config_post_processors(self._h, index, None, 0, C.byref(need)))
        buf = C.create_string_buffer(need.value)
        _check(lib.atrc_config_post_processors(self._h, index, buf, need.value, None))
        return json.loads(buf.value.decode())


class Film:
    """FP64 film accumulators (host numpy arrays, or device tensors).

    ``device=True`` allocates torch CUDA tensors and passes device pointers
    (the render then never copies the film to the host)."""

    def __init__(self, width: int, height: int, value_sq: bool = False, gbuffer: bool = False,
                 device: bool = False):
        self.width, self.height = width, height
        n = width * height
        self.device = device
        if device:
            import torch
            mk = lambda k: torch.zeros(n * k, dtype=torch.float64, device="cuda")  # noqa: E731
        else:
            mk = lambda k: np.zeros(n * k, dtype=np.float64)  # noqa: E731
        self.value = mk(3)
        self.weight = mk(1)
        self.value_sq = mk(3) if value_sq else None
        self.albedo = mk(3) if gbuffer else None
        self.normal = mk(3) if gbuffer else None
        self.denoise = mk(1) if gbuffer else None
        self._sync()

    def _sync(self) -> None:
        # the library renders on its own stream, which does not wait for
        # torch's: the zero fill must be complete before a render adds to it
        if self.device:
            import torch
            torch.cuda.current_stream().synchronize()

    def _ptr(self, a):
        if a is None:
            return None
        if self.device:
            return C.cast(C.c_void_p(a.data_ptr()), abi.c_double_p)
        return a.ctypes.data_as(abi.c_double_p)

    def as_struct(self) -> AtrcFilm:
        f = AtrcFilm()
        f.value = self._ptr(self.value)
        f.weight = self._ptr(self.weight)
        f.value_sq = self._ptr(self.value_sq)
        f.albedo = self._ptr(self.albedo)
        f.normal = self._ptr(self.normal)
        f.denoise = self._ptr(self.denoise)
        f.on_device = 1 if self.device else 0
        return f

    def clear(self) -> None:
        for a in (self.value, self.weight, self.value_sq, self.albedo, self.normal, self.denoise):
            if a is not None:
                a.fill(0) if not self.device else a.zero_()
        self._sync()

    def _host(self, a):
        return a.cpu().numpy() if self.device else a

    def image(self) -> np.ndarray:
        """value / weight as (H, W, 3) float32 (rows bottom-to-top, as the film)."""
        v = self._host(self.value).reshape(self.height, self.width, 3)
        w = self._host(self.weight).reshape(self.height, self.width, 1)
        r = np.where(w > 0, 1.0 / np.where(w > 0, w, 1), 1.0)
        return (v * r).astype(np.float32)


class DeviceScene:
    """A scene uploaded to the current CUDA device (atrc_cuda_scene_create)."""

    def __init__(self, cfg_or_desc, device: int = 0):
        lib = load_library()
        info = abi.AtrcDeviceInfo()
        _check(lib.atrc_cuda_device_init(device, C.byref(info)))
        self.info = {"name": info.name.decode(), "sm_count": info.sm_count,
                     "cc": (info.cc_major, info.cc_minor), "global_mem_bytes": info.global_mem_bytes}
        desc = cfg_or_desc.scene_desc() if isinstance(cfg_or_desc, Config) else cfg_or_desc
        self._cfg = cfg_or_desc
        h = C.c_void_p()
        _check(lib.atrc_cuda_scene_create(desc, C.byref(h)))
        self._h = h
        self.device = device

    def close(self) -> None:
        if getattr(self, "_h", None) and _lib is not None:
            _lib.atrc_cuda_scene_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    def subsurface_probe(self, o, d, n: int, seed: int = 1):
        """n subsurface walks from the closest hit of ray (o, d)
        (atrc_cuda_subsurface_probe): weights (n, 3), exit points (n, 3)."""
        o = np.ascontiguousarray(o, np.float32)
        d = np.ascontiguousarray(d, np.float32)
        w = np.zeros((n, 3), np.float32)
        x = np.zeros((n, 3), np.float32)
        fp = abi.c_float_p
        _check(load_library().atrc_cuda_subsurface_probe(self._h, o.ctypes.data_as(fp), d.ctypes.data_as(fp), n, seed,
                                                         w.ctypes.data_as(fp), x.ctypes.data_as(fp)))
        return w, x

    def trace_rays(self, rays: np.ndarray, mode: str = "closest", exact: bool = True,
                   isect: Optional[int] = None) -> np.ndarray:
        """rays: RAY_DTYPE array (or (n, 8) float32).  Returns HIT_DTYPE.
        `isect` (an AtrcIsectMode: 0 fast, 1 reference-exact Moller-Trumbore,
        2 watertight) overrides `exact`."""
        r = np.ascontiguousarray(rays)
        if r.dtype != RAY_DTYPE:
            r = np.ascontiguousarray(r, dtype=np.float32).reshape(-1, 8).view(RAY_DTYPE).reshape(-1)
        hits = np.empty(len(r), dtype=HIT_DTYPE)
        m = 0 if mode == "closest" else 1
        _check(load_library().atrc_cuda_trace_rays(
            self._h, r.ctypes.data_as(C.POINTER(abi.AtrcRay)), len(r), hits.ctypes.data_as(C.POINTER(abi.AtrcHit)),
            m, isect if isect is not None else (1 if exact else 0)))
        return hits

    def trace_rays_device(self, d_rays_ptr: int, n: int, d_hits_ptr: int, mode: str = "closest",
                          exact: bool = True) -> None:
        _check(load_library().atrc_cuda_trace_rays_device(self._h, C.c_void_p(d_rays_ptr), n,
                                                         C.c_void_p(d_hits_ptr), 0 if mode == "closest" else 1,
                                                         1 if exact else 0))

    def autotune(self, desc: AtrcRenderDesc, trial_spp: int = 0) -> dict:
        """Search the launch configuration for this scene and view
        (atrc_cuda_autotune); later renders with path_pool 0 and sort_mode -1
        use it."""
        t = abi.AtrcTuning()
        _check(load_library().atrc_cuda_autotune(self._h, C.byref(desc), trial_spp, C.byref(t)))
        return {k: getattr(t, k) for k, _ in abi.AtrcTuning._fields_}

    def tuning(self) -> dict:
        t = abi.AtrcTuning()
        _check(load_library().atrc_cuda_get_tuning(self._h, C.byref(t)))
        return {k: getattr(t, k) for k, _ in abi.AtrcTuning._fields_}

    def set_tuning(self, **kw) -> None:
        t = abi.AtrcTuning()
        _check(load_library().atrc_cuda_get_tuning(self._h, C.byref(t)))
        for k, v in kw.items():
            setattr(t, k, v)
        _check(load_library().atrc_cuda_set_tuning(self._h, C.byref(t)))

    def render_batch(self, descs, films, guide=None) -> tuple[dict, np.ndarray]:
        """Render several views in one wavefront (atrc_cuda_render_batch);
        films must be device films.  Returns the stats and each view's
        completion time in seconds from the start of the call."""
        n = len(descs)
        arr = (AtrcRenderDesc * n)(*descs)
        farr = (AtrcFilm * n)(*[f.as_struct() for f in films])
        secs = (C.c_double * n)()
        st = AtrcRenderStats()
        _check(load_library().atrc_cuda_render_batch(self._h, guide.handle if guide is not None else None, arr, n, farr,
                                                    secs, C.byref(st)))
        return {k: getattr(st, k) for k, _ in AtrcRenderStats._fields_}, np.array(secs[:])

    def render_guided(self, guide, desc: AtrcRenderDesc, film: Film, record: bool = False) -> dict:
        """Render with the learned guide sampling surface vertices
        (atrc_cuda_render_guided); record=True also keeps training records."""
        st = AtrcRenderStats()
        f = film.as_struct()
        _check(load_library().atrc_cuda_render_guided(self._h, guide.handle, C.byref(desc), 1 if record else 0,
                                                     C.byref(f), C.byref(st)))
        return {k: getattr(st, k) for k, _ in AtrcRenderStats._fields_}

    def render(self, desc: AtrcRenderDesc, film: Film, should_stop: Optional[Callable[[], bool]] = None,
               progress: Optional[Callable[[float], None]] = None) -> dict:
        """atrc_cuda_render: `should_stop` is polled between wavefront
        iterations (a true result cancels), `progress` gets percentages."""
        st = AtrcRenderStats()
        f = film.as_struct()
        cb = abi.PROGRESS_FN(lambda pct, user: progress(pct)) if progress else abi.PROGRESS_FN()
        stop = abi.CANCEL_FN(lambda user: 1 if should_stop() else 0) if should_stop else abi.CANCEL_FN()
        _check(load_library().atrc_cuda_render(self._h, C.byref(desc), C.byref(f), stop, cb, None, C.byref(st)))
        return {k: getattr(st, k) for k, _ in AtrcRenderStats._fields_}


# ------------------------------------------------------------ BVH builders

def bvh_build(boxes: np.ndarray, builder: str = "sah", device: int = 0) -> dict:
    """Build a mesh tree over (n, 6) float32 boxes (lo xyz, hi xyz) with the
    host SAH builder or the device PLOC builder; returns the build time, the
    4-wide tree's surface-area cost, its node count, rounds and depth."""
    b = np.ascontiguousarray(boxes, np.float32).reshape(-1, 6)
    info = abi.AtrcBvhBuildInfo()
    kind = {"sah": 0, "ploc": 1}[builder]
    _check(load_library().atrc_bvh_build(kind, device, b.ctypes.data_as(abi.c_float_p), len(b), C.byref(info)))
    return {k: getattr(info, k) for k, _ in abi.AtrcBvhBuildInfo._fields_}


def bvh_cluster_tree(boxes: np.ndarray, device: int = -1) -> dict:
    """PLOC cluster tree over (n, 6) boxes on the host (device < 0) or on a
    GPU: order, left, right, node boxes (internal node n + k), root, rounds."""
    b = np.ascontiguousarray(boxes, np.float32).reshape(-1, 6)
    n = len(b)
    order = np.zeros(n, np.uint32)
    left = np.zeros(max(n - 1, 1), np.int32)
    right = np.zeros(max(n - 1, 1), np.int32)
    nb = np.zeros((max(n - 1, 1), 6), np.float32)
    root, rounds = C.c_int32(), C.c_int32()
    _check(load_library().atrc_bvh_cluster_tree(
        device, b.ctypes.data_as(abi.c_float_p), n, order.ctypes.data_as(C.POINTER(C.c_uint32)),
        left.ctypes.data_as(C.POINTER(C.c_int32)), right.ctypes.data_as(C.POINTER(C.c_int32)),
        nb.ctypes.data_as(abi.c_float_p), C.byref(root), C.byref(rounds)))
    return {"order": order, "left": left[:n - 1], "right": right[:n - 1], "boxes": nb[:n - 1],
            "root": root.value, "rounds": rounds.value}
