"""Build the reference's own `pt` renderer as a second oracle (test
infrastructure): Atrc's tracer and factory sources, compiled unchanged from
where they lie in the reference checkout, against this directory's
agz-utils compatibility shim (agz-utils/), plus the C entry points of
ref_api.cpp, into oracle/_ref/libatrc_ref.so.

    python oracle/ref/build_ref.py [--reference DIR] [-j N] [--keep-going]

Every tracer and factory source is compiled except the optional Embree and
OIDN back ends (and the files in EXCLUDE); the creators that would make the
objects left out link to stubs in ref_stubs.cpp that throw.  The library travels with the
repository like the other built files; the reference checkout is needed only
to build it.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
OUT = ROOT / "oracle" / "_ref"
SO = OUT / "libatrc_ref.so"

# translation units of the reference (paths inside the checkout): every
# tracer and factory source but the optional Embree and OIDN back ends and
# those listed in EXCLUDE (they need parts of agz-utils the pt path does not)
EXCLUDE_WORDS = ("embree", "oidn")
EXCLUDE = {
    # the paper material reads a table shipped as a large blob the checkout
    # does not have (paper_rho_dt.txt, listed in .MISSING_LARGE_BLOBS)
    "src/tracer/src/core/material/paper.cpp",
}


def reference_sources(ref: Path) -> list[str]:
    out = []
    for sub in ("src/tracer/src", "src/factory/src"):
        for f in sorted((ref / sub).rglob("*.cpp")):
            rel = str(f.relative_to(ref))
            if any(w in rel for w in EXCLUDE_WORDS) or rel in EXCLUDE:
                continue
            out.append(rel)
    return out


OURS = ["ref_api.cpp", "ref_stubs.cpp", "_shim_io.cpp"]

CXX = os.environ.get("CXX", "g++")
# the reference's default CMake build type is Release (CMakeLists.txt:21-22),
# which for g++ means -O3 -DNDEBUG; no -march, so x86-64 code without FMA
FLAGS = ["-std=c++20", "-O3", "-DNDEBUG", "-fPIC", "-ffp-contract=off", "-w", "-DSPDLOG_HEADER_ONLY"]


def includes(ref: Path) -> list[str]:
    return [f"-I{HERE}", f"-I{ref / 'src/tracer/include'}", f"-I{ref / 'src/factory/include'}",
            f"-I{ref / 'lib/misc'}", f"-I{ref / 'lib/spdlog/include'}", f"-I{ROOT / 'include'}"]


def compile_one(src: Path, obj: Path, inc: list[str], newest_dep: float) -> tuple[Path, str]:
    obj.parent.mkdir(parents=True, exist_ok=True)
    if obj.exists() and obj.stat().st_mtime > max(src.stat().st_mtime, newest_dep):
        return obj, ""
    r = subprocess.run([CXX, *FLAGS, *inc, "-c", str(src), "-o", str(obj)], capture_output=True, text=True)
    return obj, (r.stdout + r.stderr) if r.returncode else ""


def build(ref: Path, jobs: int, keep_going: bool) -> Path:
    inc = includes(ref)
    srcs = [(ref / s, OUT / "obj" / (s.replace("/", "_") + ".o")) for s in reference_sources(ref)]
    srcs += [(HERE / s, OUT / "obj" / ("ours_" + s + ".o")) for s in OURS]
    # objects are rebuilt when the shim, the C ABI header or the flags change
    (OUT / "obj").mkdir(parents=True, exist_ok=True)
    stamp = OUT / "obj" / "flags.txt"
    flags = " ".join([CXX, *FLAGS, *inc])
    if not stamp.exists() or stamp.read_text() != flags:
        stamp.write_text(flags)
    deps = [stamp, ROOT / "include" / "atrc_cuda.h", *HERE.glob("agz-utils/**/*.h")]
    newest = max(p.stat().st_mtime for p in deps)
    errors = []
    objs = []
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        for obj, err in ex.map(lambda a: compile_one(a[0], a[1], inc, newest), srcs):
            objs.append(obj)
            if err:
                errors.append((obj.name, err))
    if errors:
        for name, err in errors:
            sys.stderr.write(f"==== {name}\n{err[:6000]}\n")
        if not keep_going:
            raise SystemExit(f"{len(errors)} translation units failed")
    r = subprocess.run([CXX, "-shared", "-o", str(SO), *map(str, objs), "-Wl,--no-undefined", "-lpthread", "-lz"],
                       capture_output=True, text=True)
    if r.returncode:
        raise SystemExit(r.stdout + r.stderr)
    return SO


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default="/root/reference")
    ap.add_argument("-j", type=int, default=os.cpu_count() or 4)
    ap.add_argument("--keep-going", action="store_true")
    ap.add_argument("--if-present", action="store_true",
                    help="exit 0 without building when the reference checkout is absent")
    a = ap.parse_args()
    if a.if_present and not (Path(a.reference) / "src" / "tracer").is_dir():
        print("reference checkout absent: oracle/_ref not built")
        raise SystemExit(0)
    print(build(Path(a.reference), a.j, a.keep_going))
