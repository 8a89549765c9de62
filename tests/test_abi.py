"""The C-ABI library loads, exports every declared entry point and agrees
with its bindings on struct layouts (no GPU calls), and on a machine without
a GPU its device path fails with an error instead of falling back."""
import ctypes as C
import re
from pathlib import Path

import pytest
import torch

import atrc_b200
from atrc_b200 import _abi as abi

ROOT = Path(__file__).resolve().parent.parent


def declared_functions():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = h.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*[A-Za-z_][\w\s\*]*?\b(atrc_\w+)\s*\(", text, flags=re.M):
            names.add(m.group(1))
    return names


def test_header_declares_entry_points():
    names = declared_functions()
    for required in ["atrc_cuda_scene_create", "atrc_cuda_render", "atrc_cuda_trace_rays", "atrc_config_load_file",
                     "atrc_last_error", "atrc_film_resolve", "atrc_cuda_device_init"]:
        assert required in names


def test_library_exports_every_declared_symbol():
    lib = atrc_b200.load_library()
    missing = [n for n in sorted(declared_functions()) if not hasattr(lib, n)]
    assert not missing, missing


def test_struct_layouts_match():
    lib = atrc_b200.load_library()
    n = len(abi.STRUCT_ORDER)
    sizes = (C.c_uint64 * n)()
    assert lib.atrc_abi_struct_sizes(sizes, n) == n == 17
    for cls, size in zip(abi.STRUCT_ORDER, sizes):
        assert C.sizeof(cls) == size, cls.__name__
    assert C.sizeof(abi.AtrcRay) == 32 and C.sizeof(abi.AtrcHit) == 16


def test_abi_version():
    assert atrc_b200.load_library().atrc_abi_version() == 2


def test_errors_are_reported_without_a_gpu():
    lib = atrc_b200.load_library()
    h = C.c_void_p()
    rc = lib.atrc_config_load_string(b"{not json", b".", C.byref(h))
    assert rc == -2
    assert b"JSON" in lib.atrc_last_error()
    rc = lib.atrc_cuda_scene_create(None, C.byref(h))
    assert rc == -1
    assert b"null" in lib.atrc_last_error()


@pytest.mark.skipif(torch.cuda.is_available(), reason="checks the behaviour on a machine without a GPU")
def test_device_path_fails_loudly_without_a_gpu(tmp_path):
    """No CPU fallback: creating a device scene without a GPU is an error."""
    from atrc_b200 import Config, DeviceScene, scenes
    cfg = Config.from_file(scenes.cornell_box(tmp_path / "c", width=16, height=16, spp=1))
    with pytest.raises(atrc_b200.AtrcError, match="ATRC_ERR_CUDA"):
        DeviceScene(cfg)
