"""The `ao` renderer (trace_ao, path_tracing.cpp:383-415) on the device:
an analytic known answer, and a 3-sigma image band against the oracle's
`ao` on the Cornell box."""
import json
import math

import numpy as np
import pytest

import oracle
from atrc_b200 import Config, DeviceScene, Film
from tests import kat_scenes as K
from tests.parity import band_test, global_mean_z

pytestmark = pytest.mark.gpu


def test_ao_unblocked_fraction_between_parallel_planes():
    cfg = Config.from_string(K.dumps(K.ao_slab(h=0.5, dist=1.0, spp=1024)), ".")
    desc, _ = cfg.rendering(0)
    f = Film(desc.width, desc.height, gbuffer=True)
    stats = DeviceScene(cfg).render(desc, f)
    assert stats["samples"] == desc.width * desc.height * desc.spp
    assert stats["rays_shadow"] == stats["samples"] * desc.ao_sample_count
    img = f.image().reshape(-1, 3)
    e = desc.eps
    frac = ((0.5 - e) / (1.0 - e)) ** 2
    low, high = np.array([0.1, 0.2, 0.3]), np.array([0.9, 0.8, 0.7])
    want = low + (high - low) * frac
    sigma = np.abs(high - low) * math.sqrt(frac * (1 - frac) / (desc.width * desc.height * desc.spp * 5))
    assert np.all(np.abs(img.mean(0) - want) < 5 * sigma + 1e-6), (img.mean(0), want)
    w = f.weight.reshape(-1, 1)
    np.testing.assert_allclose(f.albedo.reshape(-1, 3) / w, np.broadcast_to(high, (64, 3)), rtol=1e-6)


def test_ao_background_on_miss():
    cfg = Config.from_string(K.dumps(K.ao_slab(spp=4, looking_up=True)), ".")
    desc, _ = cfg.rendering(0)
    f = Film(desc.width, desc.height, gbuffer=True)
    DeviceScene(cfg).render(desc, f)
    np.testing.assert_allclose(f.image().reshape(-1, 3), np.broadcast_to(np.float32([0.05, 0.06, 0.07]), (64, 3)),
                               rtol=1e-6)
    assert not f.albedo.any()


def test_ao_cornell_within_3_sigma(cornell_path, tmp_path):
    cfgd = json.loads(open(cornell_path).read())
    cfgd["rendering"]["renderer"] = {"type": "ao", "spp": 512, "ao_sample_count": 4, "max_occlusion_distance": 0.3,
                                     "low_color": [0.05, 0.1, 0.2], "high_color": [1.0, 0.9, 0.8],
                                     "background_color": [0.3, 0.3, 0.3]}
    cfgd["rendering"]["width"] = cfgd["rendering"]["height"] = 48
    from pathlib import Path
    cfg = Config.from_string(json.dumps(cfgd), str(Path(cornell_path).parent))
    desc, _ = cfg.rendering(0)
    dev = DeviceScene(cfg)
    ora = oracle.OracleScene(cfg.scene_desc(), desc.eps)
    fg = Film(desc.width, desc.height, value_sq=True, gbuffer=True)
    fc = Film(desc.width, desc.height, value_sq=True, gbuffer=True)
    dev.render(desc, fg)
    ora.render(desc, fc)
    r = 0.5 - desc.eps
    frac, allowed, info = band_test(fg, fc, 1 / (4 * r * r))
    assert frac <= allowed, (frac, allowed, info)
    assert global_mean_z(fg, fc) < 4.0
    gn = fg.normal.reshape(-1, 3) / fg.weight.reshape(-1, 1)
    cn = fc.normal.reshape(-1, 3) / fc.weight.reshape(-1, 1)
    assert np.mean(np.abs(gn - cn)) < 0.02
