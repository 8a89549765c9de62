"""Build recipe for the in-tree native libraries.

* ``atrc_b200/lib/libatrc_cuda.so`` -- the product: host scene ingestion (g++)
  plus the sm_100a wavefront kernels (nvcc), exporting the C ABI of
  ``include/atrc_cuda.h``.
* ``atrc_b200/bin/atrc_cli`` -- command-line driver (mirrors the reference's
  ``CLI -d scene.json``).
* ``oracle/build/liboracle.so`` -- the CPU oracle (test infrastructure only;
  built by ``build_oracle``).

Host code is compiled without ``-march=native`` and with
``-ffp-contract=off`` so that float expressions round exactly as written; the
reference-exact ray tests depend on it.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent
PKG = ROOT / "atrc_b200"
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "lib" / "libatrc_cuda.so"
CLI = PKG / "bin" / "atrc_cli"
ORACLE_SO = ROOT / "oracle" / "build" / "liboracle.so"

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
CXX = os.environ.get("CXX", "g++")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
HOST_FLAGS = ["-std=c++17", "-O2", "-fPIC", "-ffp-contract=off", "-Wall", "-Wno-unused-function"]
NVCC_FLAGS = ["-std=c++17", "-O3", "-lineinfo", *ARCH, "-Xcompiler", "-fPIC,-ffp-contract=off",
              "--expt-relaxed-constexpr", "-Xptxas", "-O3"]

HOST_SOURCES = ["host/config.cpp", "host/scene_loader.cpp", "host/file_io.cpp", "host/bvh_build.cpp",
                "host/scene_build.cpp", "host/capi_host.cpp"]
CUDA_SOURCES = ["cuda/render.cu", "cuda/guide.cu", "cuda/post.cu", "cuda/bvh_gpu.cu", "cuda/membench.cu"]


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"command failed ({r.returncode}): {' '.join(cmd)}\n{r.stdout}")
    if r.stdout.strip():
        sys.stderr.write(r.stdout)


def _deps(src: Path) -> list[Path]:
    return sorted((CSRC / "host").glob("*.h")) + sorted((CSRC / "cuda").glob("*.h")) + \
        sorted((CSRC / "cuda").glob("*.cuh")) + [ROOT / "include" / "atrc_cuda.h", src]


def _stale(obj: Path, src: Path) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return any(d.stat().st_mtime > t for d in _deps(src))


def _compile(src_rel: str, verbose_ptxas: bool) -> Path:
    src = CSRC / src_rel
    obj = BUILD / (src_rel.replace("/", "_") + ".o")
    if not _stale(obj, src):
        return obj
    obj.parent.mkdir(parents=True, exist_ok=True)
    if src.suffix == ".cu":
        cmd = [NVCC, *NVCC_FLAGS, "-c", str(src), "-o", str(obj)]
        if verbose_ptxas:
            cmd[1:1] = ["-Xptxas", "-v"]
    else:
        cmd = [CXX, *HOST_FLAGS, "-c", str(src), "-o", str(obj)]
    _run(cmd)
    return obj


def build_library(verbose_ptxas: bool = False) -> Path:
    """Compile and link libatrc_cuda.so (sm_100a)."""
    BUILD.mkdir(parents=True, exist_ok=True)
    with cf.ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose_ptxas), HOST_SOURCES + CUDA_SOURCES))
    LIB.parent.mkdir(parents=True, exist_ok=True)
    if not LIB.exists() or any(o.stat().st_mtime > LIB.stat().st_mtime for o in objs):
        tmp = LIB.with_suffix(".so.tmp")
        _run([NVCC, *ARCH, "-shared", "-o", str(tmp), *map(str, objs), "-lpthread", "-lz"])
        os.replace(tmp, LIB)
    return LIB


def build_cli() -> Path:
    """Link the command-line driver against libatrc_cuda.so."""
    src = CSRC / "cli" / "main.cpp"
    if not src.exists():
        return CLI
    lib = build_library()
    CLI.parent.mkdir(parents=True, exist_ok=True)
    if not CLI.exists() or max(src.stat().st_mtime, lib.stat().st_mtime) > CLI.stat().st_mtime:
        _run([CXX, *HOST_FLAGS, str(src), "-o", str(CLI), f"-L{lib.parent}", "-latrc_cuda",
              "-Wl,-rpath,$ORIGIN/../lib", "-lpthread"])
    return CLI


def build_oracle() -> Path:
    """Compile the CPU oracle (test infrastructure)."""
    src = ROOT / "oracle" / "pt_oracle.cpp"
    ORACLE_SO.parent.mkdir(parents=True, exist_ok=True)
    deps = [src, ROOT / "oracle" / "oracle.h", ROOT / "include" / "atrc_cuda.h"]
    if not ORACLE_SO.exists() or any(d.stat().st_mtime > ORACLE_SO.stat().st_mtime for d in deps):
        tmp = ORACLE_SO.with_suffix(".so.tmp")
        _run([CXX, "-std=c++17", "-O2", "-fPIC", "-ffp-contract=off", "-shared", str(src), "-o", str(tmp),
              "-lpthread"])
        os.replace(tmp, ORACLE_SO)
    return ORACLE_SO


def clean() -> None:
    shutil.rmtree(BUILD, ignore_errors=True)


if __name__ == "__main__":
    print(build_library(verbose_ptxas="-v" in sys.argv))
    print(build_oracle())
    print(build_cli())
