"""ctypes binding of the CPU oracle (``oracle/build/liboracle.so``).

TEST INFRASTRUCTURE ONLY: tests/, ``__graft_entry__.smoke()`` and the CPU
baseline of ``bench.py`` use it as the checker / the timed CPU baseline.  The
product package ``atrc_b200`` never imports it.  Parity status: pinned to the
reference's own tracer and factory code, built from its sources against an
agz-utils compatibility shim into ``oracle/_ref/libatrc_ref.so`` (``RefScene``
below; see oracle.h for what the shim leaves unpinned).
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from atrc_b200 import _abi as abi
from atrc_b200 import HIT_DTYPE, RAY_DTYPE

SO = Path(__file__).resolve().parent / "build" / "liboracle.so"
_lib = None


def load() -> C.CDLL:
    global _lib
    if _lib is None:
        if not SO.exists():
            from atrc_b200.build import build_oracle
            build_oracle()
        lib = C.CDLL(str(SO))
        lib.oracle_last_error.restype = C.c_char_p
        lib.oracle_scene_create.argtypes = [C.POINTER(abi.AtrcSceneDesc), C.c_float, C.POINTER(C.c_void_p)]
        lib.oracle_scene_destroy.argtypes = [C.c_void_p]
        lib.oracle_scene_destroy.restype = None
        lib.oracle_trace_rays.argtypes = [C.c_void_p, C.POINTER(abi.AtrcRay), C.c_size_t, C.POINTER(abi.AtrcHit),
                                          C.c_int, C.c_int, C.c_int]
        lib.oracle_prim_hit.argtypes = [C.c_void_p, C.POINTER(abi.AtrcRay), C.c_int, C.c_int, C.c_int,
                                        C.POINTER(C.c_float)]
        lib.oracle_render.argtypes = [C.c_void_p, C.POINTER(abi.AtrcRenderDesc), C.POINTER(abi.AtrcFilm), C.c_int]
        lib.oracle_render_sample.argtypes = [C.c_void_p, C.POINTER(abi.AtrcRenderDesc), C.POINTER(abi.AtrcFilm),
                                             C.c_int, C.c_int]
        lib.oracle_env_pdf.argtypes = [C.c_void_p, abi.c_float_p, C.c_size_t, abi.c_float_p]
        lib.oracle_env_sample.argtypes = [C.c_void_p, abi.c_float_p, C.c_size_t, abi.c_float_p, abi.c_float_p]
        lib.oracle_bsdf_eval.argtypes = [C.c_void_p, C.c_int, abi.c_float_p, abi.c_float_p, C.c_size_t,
                                         abi.c_float_p, abi.c_float_p]
        lib.oracle_bsdf_sample.argtypes = [C.c_void_p, C.c_int, abi.c_float_p, abi.c_float_p, C.c_size_t,
                                           abi.c_float_p, abi.c_float_p, abi.c_float_p, C.POINTER(C.c_int), C.c_int]
        lib.oracle_subsurface.argtypes = [C.c_void_p, abi.c_float_p, abi.c_float_p, C.c_size_t, C.c_uint64,
                                          abi.c_float_p, abi.c_float_p]
        _lib = lib
    return _lib


def _check(rc: int) -> None:
    if rc != 0:
        raise RuntimeError(f"oracle error {rc}: {load().oracle_last_error().decode()}")


def _fp(a: np.ndarray):
    return a.ctypes.data_as(abi.c_float_p)


class OracleScene:
    def __init__(self, scene_desc_ptr, eps: float = 3e-4):
        lib = load()
        h = C.c_void_p()
        _check(lib.oracle_scene_create(scene_desc_ptr, eps, C.byref(h)))
        self._h = h

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.oracle_scene_destroy(self._h)
            self._h = None

    def trace_rays(self, rays: np.ndarray, mode: str = "closest", threads: int = 0,
                   watertight: bool = False) -> np.ndarray:
        """Closest / any hits with the reference's Moller-Trumbore test, or the
        watertight test with `watertight`."""
        r = np.ascontiguousarray(rays, dtype=RAY_DTYPE)
        hits = np.empty(len(r), dtype=HIT_DTYPE)
        _check(load().oracle_trace_rays(self._h, r.ctypes.data_as(C.POINTER(abi.AtrcRay)), len(r),
                                        hits.ctypes.data_as(C.POINTER(abi.AtrcHit)), 0 if mode == "closest" else 1,
                                        2 if watertight else 1, threads))
        return hits

    def prim_hit(self, ray: np.ndarray, entity: int, prim: int, watertight: bool = False) -> float:
        r = np.ascontiguousarray(ray, dtype=RAY_DTYPE).reshape(1)
        t = C.c_float()
        _check(load().oracle_prim_hit(self._h, r.ctypes.data_as(C.POINTER(abi.AtrcRay)), entity, prim,
                                      2 if watertight else 1, C.byref(t)))
        return t.value

    def render(self, desc: abi.AtrcRenderDesc, film, threads: int = 0) -> None:
        f = film.as_struct()
        _check(load().oracle_render(self._h, C.byref(desc), C.byref(f), threads))

    def render_sample(self, desc: abi.AtrcRenderDesc, film, threads: int = 0, tile_stride: int = 1) -> None:
        f = film.as_struct()
        _check(load().oracle_render_sample(self._h, C.byref(desc), C.byref(f), threads, tile_stride))

    def env_pdf(self, dirs: np.ndarray) -> np.ndarray:
        d = np.ascontiguousarray(dirs, dtype=np.float32)
        out = np.empty(len(d), dtype=np.float32)
        _check(load().oracle_env_pdf(self._h, _fp(d), len(d), _fp(out)))
        return out

    def env_sample(self, u3: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
        u = np.ascontiguousarray(u3, dtype=np.float32)
        dirs = np.empty((len(u), 3), dtype=np.float32)
        pdf = np.empty(len(u), dtype=np.float32)
        _check(load().oracle_env_sample(self._h, _fp(u), len(u), _fp(dirs), _fp(pdf)))
        return dirs, pdf

    def bsdf_eval(self, material: int, wi: np.ndarray, wo: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
        wi = np.ascontiguousarray(wi, dtype=np.float32)
        wo = np.ascontiguousarray(wo, dtype=np.float32)
        f = np.empty((len(wi), 3), dtype=np.float32)
        pdf = np.empty(len(wi), dtype=np.float32)
        _check(load().oracle_bsdf_eval(self._h, material, _fp(wi), _fp(wo), len(wi), _fp(f), _fp(pdf)))
        return f, pdf

    def subsurface(self, o, d, n: int, seed: int = 1):
        """n subsurface probes from the closest hit of ray (o, d): weights
        (n, 3) (zero for invalid samples) and exit points (n, 3)."""
        o = np.ascontiguousarray(o, dtype=np.float32)
        d = np.ascontiguousarray(d, dtype=np.float32)
        w = np.empty((n, 3), dtype=np.float32)
        x = np.empty((n, 3), dtype=np.float32)
        _check(load().oracle_subsurface(self._h, _fp(o), _fp(d), n, seed, _fp(w), _fp(x)))
        return w, x

    def bsdf_sample(self, material: int, wo: np.ndarray, u3: np.ndarray, disney_fixed: bool = False):
        wo = np.ascontiguousarray(wo, dtype=np.float32)
        u = np.ascontiguousarray(u3, dtype=np.float32)
        n = len(wo)
        wi = np.empty((n, 3), dtype=np.float32)
        f = np.empty((n, 3), dtype=np.float32)
        pdf = np.empty(n, dtype=np.float32)
        delta = np.empty(n, dtype=np.int32)
        _check(load().oracle_bsdf_sample(self._h, material, _fp(wo), _fp(u), n, _fp(wi), _fp(f), _fp(pdf),
                                         delta.ctypes.data_as(C.POINTER(C.c_int)), int(disney_fixed)))
        return wi, f, pdf, delta


def hardware_threads() -> int:
    return int(load().oracle_hardware_threads())


# ----------------------------------------------------------------------------
# The reference's own renderer: Atrc's tracer and factory sources compiled
# against the agz-utils compatibility shim (oracle/ref/build_ref.py ->
# oracle/_ref/libatrc_ref.so).  Same role as the restatement above -- a
# checker, never the product -- but its scene parsing, BVHs, intersection
# tests, materials, lights, media and trace_std are the reference's code.

REF_SO = Path(__file__).resolve().parent / "_ref" / "libatrc_ref.so"
_ref_lib = None


def ref_available() -> bool:
    return REF_SO.exists()


def load_ref() -> C.CDLL:
    global _ref_lib
    if _ref_lib is None:
        if not REF_SO.exists():
            raise RuntimeError(f"{REF_SO} is missing: build it with `python oracle/ref/build_ref.py` "
                               "where the reference checkout is present")
        lib = C.CDLL(str(REF_SO))
        lib.ref_last_error.restype = C.c_char_p
        lib.ref_scene_create.argtypes = [C.c_char_p, C.c_char_p, C.POINTER(C.c_void_p)]
        lib.ref_scene_destroy.argtypes = [C.c_void_p]
        lib.ref_scene_destroy.restype = None
        lib.ref_entity_count.argtypes = [C.c_void_p]
        lib.ref_trace_rays.argtypes = [C.c_void_p, C.POINTER(abi.AtrcRay), C.c_size_t, C.POINTER(abi.AtrcHit),
                                       C.c_int, C.c_int]
        dp = C.POINTER(C.c_double)
        lib.ref_render.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_uint64, C.c_int,
                                   C.c_int, dp, dp, dp, dp, dp, dp]
        fp = C.POINTER(C.c_float)
        lib.ref_filter_eval.argtypes = [C.c_void_p, C.c_int, fp, fp, C.c_size_t, fp]
        _ref_lib = lib
    return _ref_lib


def _ref_check(rc: int) -> None:
    if rc != 0:
        raise RuntimeError(f"reference renderer: {load_ref().ref_last_error().decode()}")


class RefScene:
    """A scene built by the reference's own factory from its JSON file."""

    def __init__(self, json_path):
        p = Path(json_path)
        h = C.c_void_p()
        _ref_check(load_ref().ref_scene_create(p.read_text().encode(), str(p.parent).encode(), C.byref(h)))
        self._h = h

    def __del__(self):
        if getattr(self, "_h", None) and _ref_lib is not None:
            _ref_lib.ref_scene_destroy(self._h)
            self._h = None

    def entity_count(self) -> int:
        return int(load_ref().ref_entity_count(self._h))

    def trace_rays(self, rays: np.ndarray, mode: str = "closest", threads: int = 0) -> np.ndarray:
        r = np.ascontiguousarray(rays, dtype=RAY_DTYPE)
        hits = np.empty(len(r), dtype=HIT_DTYPE)
        _ref_check(load_ref().ref_trace_rays(self._h, r.ctypes.data_as(C.POINTER(abi.AtrcRay)), len(r),
                                             hits.ctypes.data_as(C.POINTER(abi.AtrcHit)),
                                             0 if mode == "closest" else 1, threads))
        return hits

    def filter_eval(self, x, y, index: int = 0) -> np.ndarray:
        """The reference's film filter of rendering entry `index` at the
        offsets (x, y) from a pixel centre."""
        fp = C.POINTER(C.c_float)
        xa = np.ascontiguousarray(x, np.float32).ravel()
        ya = np.ascontiguousarray(y, np.float32).ravel()
        out = np.empty(len(xa), np.float32)
        _ref_check(load_ref().ref_filter_eval(self._h, index, xa.ctypes.data_as(fp), ya.ctypes.data_as(fp), len(xa),
                                              out.ctypes.data_as(fp)))
        return out

    def render(self, film, index: int = 0, spp: int = 1, first_spp: int = 0, seed: int = 1, threads: int = 0,
               width: int = 0, height: int = 0, tile_stride: int = 1) -> None:
        """Add `spp` samples per pixel of rendering entry `index` (renderer
        pt or ao) into a host Film (value, weight and, where the film has
        them, value_sq and the G-buffer); tile_stride > 1 renders only every
        tile_stride-th task tile."""
        dp = C.POINTER(C.c_double)
        ptr = lambda a: None if a is None else a.ctypes.data_as(dp)  # noqa: E731
        _ref_check(load_ref().ref_render(self._h, index, width, height, first_spp, spp, seed, threads, tile_stride,
                                         ptr(film.value), ptr(film.weight), ptr(film.value_sq),
                                         ptr(film.albedo), ptr(film.normal), ptr(film.denoise)))
