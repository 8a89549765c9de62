"""The device path against the reference's own renderer (oracle/_ref) on the
benchmark scenes at their stated geometry and settings, through the C ABI.

* the seeded Cornell box at its full size (256 x 256, 64 spp,
  max depth 8), every pixel in the 3-sigma band.
* the instanced Disney + IBL scene, 3.08M unique triangles in 64
  instances, at its full 1920 x 1080 film and depth 16 with 16 spp (the
  reference's CPU time at 256 spp would be minutes), the band over 8 x 8
  pixel blocks; closest hits of 10^6 seeded rays.
* the media scene (128^3 fBm grid, 200,000-triangle sphere, two
  area lights and the sky) at its 512 spp and depth 32 on a 48 x 48 film.
* the indoor room at its full 1280 x 720 film with 16 spp, the
  band over 8 x 8 pixel blocks.

The reference renders through its own factory, BVHs, materials, lights,
media and trace_std (`tests/test_ref_oracle.py` pins the restated oracle to
the same library on small scenes).
"""
import numpy as np
import pytest

import oracle
from atrc_b200 import Config, DeviceScene, Film, scenes
from tests.parity import band_test, global_mean_z, seeded_rays, ulp_diff

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not oracle.ref_available(), reason="oracle/_ref/libatrc_ref.so not built")]

BOX = 1 / (4 * (0.5 - 3e-4) ** 2)  # box filter weight of one sample


def _device_and_reference(path, spp=None, seed=41):
    cfg = Config.from_file(path)
    desc, _ = cfg.rendering(0)
    if spp is not None:
        desc.spp = spp
    # the reference samples Disney with its own sampler (disney.cpp:578-589),
    # whatever a pt_cuda key asks for
    desc.disney_fixed = 0
    fg = Film(desc.width, desc.height, value_sq=True)
    st = DeviceScene(cfg).render(desc, fg)
    assert st["samples"] == desc.width * desc.height * desc.spp and st["watchdog_flags"] == 0
    fr = Film(desc.width, desc.height, value_sq=True)
    oracle.RefScene(path).render(fr, spp=desc.spp, seed=seed)
    return desc, fg, fr


class _Blocks:
    """A film's sums over b x b pixel blocks (value, weight and value_sq are
    sums over samples, so block sums estimate block means): at 16 spp a
    pixel's few samples from a heavy-tailed distribution (sun and sky hits)
    do not follow the t law the band test assumes; 8 x 8 blocks of 1,024
    samples do."""

    def __init__(self, f, w, h, b):
        H, W = h // b, w // b
        def agg(a, c):
            return a.reshape(h, w, c)[:H * b, :W * b].reshape(H, b, W, b, c).sum((1, 3)).reshape(-1)
        self.value, self.weight, self.value_sq = agg(f.value, 3), agg(f.weight, 1), agg(f.value_sq, 3)


def _assert_band(fg, fr, desc=None, block=1):
    if block > 1:
        fg, fr = _Blocks(fg, desc.width, desc.height, block), _Blocks(fr, desc.width, desc.height, block)
    frac, allowed, info = band_test(fg, fr, BOX, cluster=3)
    assert frac <= allowed, (frac, allowed, info)
    assert global_mean_z(fg, fr) < 4.0


def test_cornell_full_size_matches_reference(scene_dir):
    desc, fg, fr = _device_and_reference(scenes.cornell_box(scene_dir / "ref_cornell_256"))
    assert (desc.width, desc.height, desc.spp, desc.max_depth) == (256, 256, 64, 8)
    _assert_band(fg, fr)


@pytest.fixture(scope="module")
def instanced_full(scene_dir):
    return scenes.instanced_disney(scene_dir / "ref_inst_full")


def test_instanced_full_film_matches_reference(instanced_full):
    desc, fg, fr = _device_and_reference(instanced_full, spp=16)
    assert (desc.width, desc.height, desc.max_depth) == (1920, 1080, 16)
    _assert_band(fg, fr, desc, block=8)


def test_instanced_closest_hits_match_reference(instanced_full):
    cfg = Config.from_file(instanced_full)
    desc, _ = cfg.rendering(0)
    sd = cfg.scene_desc().contents
    assert sum(int(sd.meshes[i].triangle_count) for i in range(sd.mesh_count)) == 3_076_098
    rays = seeded_rays(1_000_000, [-22.0] * 3, [22.0] * 3, list(desc.camera.pos), seed=23)
    g = DeviceScene(cfg).trace_rays(rays, "closest", exact=True)
    r = oracle.RefScene(instanced_full).trace_rays(rays, "closest")
    assert (g["entity"] == r["entity"]).mean() >= 0.9999
    hit = (g["entity"] == r["entity"]) & (g["entity"] >= 0)
    assert hit.sum() > 100_000
    # instance matrices come from agz-utils' float matrix code in the
    # reference (restated by the shim): t agrees to matrix rounding
    u = ulp_diff(g["t"][hit], r["t"][hit])
    assert np.median(u) <= 1 and np.quantile(u, 0.99) <= 128, np.quantile(u, [0.5, 0.99])


def test_media_matches_reference(scene_dir):
    path = scenes.media_scene(scene_dir / "ref_media_128", width=48, height=48, spp=512)
    desc, fg, fr = _device_and_reference(path)
    assert (desc.spp, desc.max_depth) == (512, 32)
    _assert_band(fg, fr)


def test_room_full_film_matches_reference(scene_dir):
    desc, fg, fr = _device_and_reference(scenes.indoor_room(scene_dir / "ref_room_720p"), spp=16)
    assert (desc.width, desc.height, desc.max_depth) == (1280, 720, 16)
    _assert_band(fg, fr, desc, block=8)
