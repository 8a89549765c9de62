"""The output path on the device: film resolve, the reference's `gamma` and
`aces` post processors, the 8-bit encoding of `save_to_img` /
`save_gbuffer_to_png`, the whole post-processor chain and the CLI driver."""
import ctypes as C
import json
import struct
import subprocess
import zlib
from pathlib import Path

import numpy as np
import pytest
import torch

from atrc_b200 import Config, DeviceScene, Film, load_library

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parent.parent


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def read_png(path: Path) -> np.ndarray:
    """8-bit RGB PNG (as the library writes it) -> (H, W, 3) uint8, rows top first."""
    data = path.read_bytes()
    assert data[:8] == b"\x89PNG\r\n\x1a\n"
    pos, idat = 8, b""
    w = h = 0
    while pos < len(data):
        n, = struct.unpack(">I", data[pos:pos + 4])
        kind = data[pos + 4:pos + 8]
        body = data[pos + 8:pos + 8 + n]
        if kind == b"IHDR":
            w, h = struct.unpack(">II", body[:8])
        elif kind == b"IDAT":
            idat += body
        pos += 12 + n
    raw = np.frombuffer(zlib.decompress(idat), np.uint8).reshape(h, 1 + 3 * w)
    assert np.all(raw[:, 0] == 0)
    return raw[:, 1:].reshape(h, w, 3)


def aces(x):
    x = x.astype(np.float32)
    return np.clip((x * (np.float32(2.51) * x + np.float32(0.03))) / (x * (np.float32(2.43) * x + np.float32(0.59))
                                                                   + np.float32(0.14)), 0, 1)


def encode(img, gamma):
    v = np.clip(np.power(img.astype(np.float32), np.float32(gamma)), 0, 1)
    v = np.where(np.isnan(v), 0, v)
    return (v * np.float32(255)).astype(np.uint8)[::-1]


@pytest.fixture(scope="module")
def rendered(cornell_path):
    cfg = Config.from_file(cornell_path)
    desc, _ = cfg.rendering(0)
    desc.width, desc.height, desc.spp = 48, 40, 16
    dev = DeviceScene(cfg)
    film = Film(48, 40, gbuffer=True, device=True)
    dev.render(desc, film)
    return film


def test_resolve_and_post_steps_match_the_reference_formulas(rendered):
    lib = load_library()
    f = rendered
    W, H = f.width, f.height
    rgb = torch.empty(H * W * 3, dtype=torch.float32, device="cuda")
    alb = torch.empty_like(rgb)
    nrm = torch.empty_like(rgb)
    st = f.as_struct()
    assert lib.atrc_cuda_film_resolve(C.byref(st), W, H, _ptr(rgb), _ptr(alb), _ptr(nrm)) == 0
    w = f.weight.cpu().numpy()
    ref = (f.value.cpu().numpy().reshape(-1, 3) / w[:, None]).astype(np.float32)
    np.testing.assert_array_equal(rgb.cpu().numpy().reshape(-1, 3), ref)
    np.testing.assert_array_equal(alb.cpu().numpy().reshape(-1, 3),
                                  (f.albedo.cpu().numpy().reshape(-1, 3) / w[:, None]).astype(np.float32))
    # aces then gamma, in place
    assert lib.atrc_cuda_post_apply(_ptr(rgb), W, H, 1, C.c_float(1.7)) == 0
    exp = aces(ref * np.float32(1.7))
    np.testing.assert_allclose(rgb.cpu().numpy().reshape(-1, 3), exp, rtol=1e-6, atol=1e-7)
    assert lib.atrc_cuda_post_apply(_ptr(rgb), W, H, 0, C.c_float(1 / 2.2)) == 0
    exp = np.power(exp, np.float32(1 / 2.2))
    np.testing.assert_allclose(rgb.cpu().numpy().reshape(-1, 3), exp, rtol=2e-6, atol=1e-7)
    # 8-bit encoding: flipped, clamp(c^g) * 255
    out = torch.empty(H * W * 3, dtype=torch.uint8, device="cuda")
    assert lib.atrc_cuda_encode_ldr(_ptr(rgb), W, H, C.c_float(1.0), _ptr(out)) == 0
    got = out.cpu().numpy().reshape(H, W, 3).astype(int)
    want = encode(exp.reshape(H, W, 3), 1.0).astype(int)
    assert np.max(np.abs(got - want)) <= 1 and np.mean(got != want) < 1e-3
    assert lib.atrc_cuda_post_apply(_ptr(rgb), W, H, 0, C.c_float(-1)) == -1


def test_post_processor_chain(rendered, tmp_path):
    f = rendered
    W, H = f.width, f.height
    chain = [{"type": "aces", "exposure": 2.0},
             {"type": "save_to_img", "filename": "${scene-directory}/out/a.png", "inv_gamma": 2.2},
             {"type": "gamma", "gamma": 0.5},
             {"type": "save_to_img", "filename": "${scene-directory}/out/b.hdr"},
             {"type": "save_gbuffer_to_png", "albedo": "${scene-directory}/out/alb.png",
              "normal": "${scene-directory}/out/nor.png"},
             {"type": "resize", "size": [10, 10]}]
    log = C.create_string_buffer(4096)
    st = f.as_struct()
    rc = load_library().atrc_cuda_post_process(C.byref(st), W, H, json.dumps(chain).encode(), str(tmp_path).encode(),
                                              log, 4096)
    assert rc == 0, load_library().atrc_last_error()
    text = log.value.decode()
    assert "skipped resize" in text and text.count("saved") == 4
    w = f.weight.cpu().numpy()[:, None]
    img = (f.value.cpu().numpy().reshape(-1, 3) / w).astype(np.float32)
    a = aces(img * np.float32(2.0))
    got = read_png(tmp_path / "out" / "a.png").astype(int)
    want = encode(a.reshape(H, W, 3), 1 / 2.2).astype(int)
    assert np.max(np.abs(got - want)) <= 1 and np.mean(got != want) < 1e-3
    assert (tmp_path / "out" / "b.hdr").read_bytes().startswith(b"#?RADIANCE")
    nor = read_png(tmp_path / "out" / "nor.png").astype(int)
    n = (f.normal.cpu().numpy().reshape(-1, 3) / w).astype(np.float32)
    want_n = encode(((n + 1) * np.float32(0.5)).reshape(H, W, 3), 1.0).astype(int)
    assert np.max(np.abs(nor - want_n)) <= 1


def test_cli_renders_and_post_processes(tmp_path, cornell_path):
    cfg = json.loads(Path(cornell_path).read_text())
    src = Path(cornell_path).parent
    cfg["rendering"]["width"] = cfg["rendering"]["height"] = 32
    cfg["rendering"]["renderer"]["spp"] = 4
    cfg["rendering"]["renderer"]["type"] = "pt"   # rendered by pt_cuda through --renderer
    cfg["rendering"]["post_processors"] = [{"type": "save_to_img", "filename": "${scene-directory}/cli.png"}]
    scene = src / "cli_scene.json"
    scene.write_text(json.dumps(cfg))
    out = subprocess.run([str(ROOT / "atrc_b200" / "bin" / "atrc_cli"), "-d", str(scene), "--renderer", "pt_cuda"],
                         capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
    img = read_png(src / "cli.png")
    assert img.shape == (32, 32, 3) and img.max() > 0
