"""The image writers of the output path (atrc_save_image: png / hdr / pfm, as
the `save_to_img` post processor) read back through the scene loader's image
readers, on CPU.  Films are rows bottom-first; the files hold the top row
first, so a file read back as a texture is the film flipped vertically."""
import ctypes as C

import numpy as np
import pytest

from atrc_b200 import AtrcError, Config, load_library
from tests.test_config import QUAD, base


def _save(path, rgb, gamma=1.0):
    lib = load_library()
    lib.atrc_save_image.argtypes = [C.c_char_p, C.c_char_p, C.c_void_p, C.c_int, C.c_int, C.c_float]
    h, w, _ = rgb.shape
    a = np.ascontiguousarray(rgb, np.float32)
    return lib.atrc_save_image(str(path).encode(), None, a.ctypes.data, w, h, gamma)


def _read_back(tmp_path, fn, kind):
    c = base([QUAD], env={"type": "ibl", "tex": {"type": kind, "filename": "${scene-directory}/" + fn}})
    cfg = Config.from_string(c, tmp_path)
    s = cfg.scene_desc().contents
    t = s.textures2d[s.env.tex]
    return np.ctypeslib.as_array(t.data, shape=(t.height * t.width * 3,)).reshape(t.height, t.width, 3).copy()


def _film(h, w, seed):
    rng = np.random.default_rng(seed)
    rgb = rng.lognormal(0.0, 2.0, (h, w, 3)).astype(np.float32)
    rgb[:, w // 3: w // 3 + min(w, 150)] = rgb[:, w // 3: w // 3 + 1]   # long runs for the RLE encoder
    rgb[0, 0] = 0.0
    return rgb


def test_pfm_round_trip_is_exact(tmp_path):
    rgb = _film(4, 9, 1)
    assert _save(tmp_path / "f.pfm", rgb) == 0
    np.testing.assert_array_equal(_read_back(tmp_path, "f.pfm", "hdr"), rgb[::-1])


@pytest.mark.parametrize("w", [5, 400])
def test_hdr_round_trip_within_rgbe_precision(tmp_path, w):
    # w = 5 is written flat, w = 400 run-length encoded (runs longer than
    # 127 bytes and literals longer than 128 included)
    rgb = _film(6, w, 2)
    assert _save(tmp_path / "f.hdr", rgb) == 0
    got = _read_back(tmp_path, "f.hdr", "hdr")
    want = rgb[::-1]
    m = want.max(axis=2, keepdims=True)
    # RGBE keeps 8 bits below the largest channel's exponent and truncates
    assert np.all(got <= want) and np.all(want - got <= m / 128 + 1e-30)
    raw = (tmp_path / "f.hdr").read_bytes()
    body = raw[raw.index(b"+X %d\n" % w) + len(b"+X %d\n" % w):]
    if w >= 8:
        assert body[:4] == bytes([2, 2, w >> 8, w & 255]) and len(body) < 6 * w * 4
    else:
        assert len(body) == 6 * w * 4


def test_png_round_trip(tmp_path):
    rgb = _film(5, 7, 3) / 8.0
    gamma = 1 / 2.2
    assert _save(tmp_path / "f.png", rgb, gamma) == 0
    got = _read_back(tmp_path, "f.png", "image")
    want = np.floor(np.clip(rgb[::-1].astype(np.float64) ** gamma, 0, 1) * 255) / 255
    assert np.abs(got - want).max() <= 1 / 255 + 1e-6


def test_unknown_extension_is_an_error(tmp_path):
    assert _save(tmp_path / "f.bmp", np.ones((2, 2, 3), np.float32)) != 0
    with pytest.raises(AtrcError):
        from atrc_b200 import _check
        _check(_save(tmp_path / "g.bmp", np.ones((2, 2, 3), np.float32)))
