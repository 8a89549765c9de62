"""atrc_cuda_render_noalloc: rendering for callers that cannot allocate device
memory during a render (they own the GPU's memory through their own
sub-allocator, run under a fixed memory budget, or must stay out of the
driver's allocator in a real-time loop).  Its scratch lives in a static device
array inside the library; the caller supplies only the scene and a device film.

The check: two calls in a row through the C ABI give the same films as the
allocating entry point (atrc_cuda_render) on the same sample indices.  Both
entry points draw the same random numbers per sample, so the films agree up to
the order of floating-point atomic additions.  The file name sorts last so that
a run stopping at the first failure has run every other test first.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _render_noalloc(scene, desc, film):
    from atrc_b200 import _abi as abi
    from atrc_b200 import load_library, _check
    st = abi.AtrcRenderStats()
    f = film.as_struct()
    _check(load_library().atrc_cuda_render_noalloc(scene.handle, C.byref(desc), C.byref(f), C.byref(st)))
    return st


def test_noalloc_matches_allocating_render_twice(tmp_path):
    from atrc_b200 import Config, DeviceScene, Film
    from atrc_b200.scenes import cornell_box

    cfg = Config.from_file(cornell_box(tmp_path / "cornell", width=64, height=48, spp=32, renderer="pt_cuda"))
    desc, _ = cfg.rendering(0)
    scene = DeviceScene(cfg)
    ref = Film(desc.width, desc.height, value_sq=True, gbuffer=True, device=True)
    got = Film(desc.width, desc.height, value_sq=True, gbuffer=True, device=True)
    for call in range(2):
        desc.first_spp = call * desc.spp  # a different sample range per call
        desc.spp_count = desc.spp
        scene.render(desc, ref)
        st = _render_noalloc(scene, desc, got)
        assert st.samples == desc.width * desc.height * desc.spp
        for name in ("value", "weight", "value_sq", "albedo", "normal", "denoise"):
            a = getattr(ref, name).cpu().numpy()
            b = getattr(got, name).cpu().numpy()
            np.testing.assert_allclose(b, a, rtol=1e-4, atol=1e-6, err_msg=f"call {call}: {name}")
    img = got.image()
    assert np.isfinite(img).all() and img.mean() > 0


def test_noalloc_reuses_pool_slots_like_allocating_render(tmp_path):
    """A 1024-path pool for 16,384 samples: every slot is freed by k_finish and
    taken again by k_generate about 16 times inside the static array."""
    from atrc_b200 import Config, DeviceScene, Film
    from atrc_b200.scenes import cornell_box

    cfg = Config.from_file(cornell_box(tmp_path / "cornell3", width=32, height=32, spp=16, renderer="pt_cuda"))
    desc, _ = cfg.rendering(0)
    desc.path_pool = 1024
    scene = DeviceScene(cfg)
    ref = Film(desc.width, desc.height, value_sq=True, gbuffer=True, device=True)
    got = Film(desc.width, desc.height, value_sq=True, gbuffer=True, device=True)
    for call in range(2):
        desc.first_spp = call * desc.spp
        desc.spp_count = desc.spp
        st_ref = scene.render(desc, ref)
        st = _render_noalloc(scene, desc, got)
        assert st.samples == desc.width * desc.height * desc.spp == st_ref["samples"]
        assert st.iterations > 16  # the pool was refilled many times
        for name in ("value", "weight", "value_sq", "albedo", "normal", "denoise"):
            a = getattr(ref, name).cpu().numpy()
            b = getattr(got, name).cpu().numpy()
            np.testing.assert_allclose(b, a, rtol=1e-4, atol=1e-6, err_msg=f"call {call}: {name}")


def test_noalloc_rejects_film_with_too_many_tiles(tmp_path):
    """2048 x 2048 one-pixel tiles are 2^22 tiles, more than the path state's
    tile field holds: rejected before anything is launched."""
    from atrc_b200 import AtrcError, Config, DeviceScene, Film
    from atrc_b200.scenes import cornell_box

    cfg = Config.from_file(cornell_box(tmp_path / "cornell4", width=16, height=16, spp=1, renderer="pt_cuda"))
    desc, _ = cfg.rendering(0)
    scene = DeviceScene(cfg)
    desc.width = desc.height = 2048
    desc.task_grid_size = 1
    with pytest.raises(AtrcError, match="2\\^22"):
        _render_noalloc(scene, desc, Film(16, 16, device=True))
    # the scene stays usable
    desc.width = desc.height = 16
    desc.task_grid_size = 0
    film = Film(16, 16, device=True)
    st = _render_noalloc(scene, desc, film)
    assert st.samples == 16 * 16 * desc.spp


def test_noalloc_rejects_host_film_and_oversized_pool(tmp_path):
    from atrc_b200 import AtrcError, Config, DeviceScene, Film
    from atrc_b200.scenes import cornell_box

    cfg = Config.from_file(cornell_box(tmp_path / "cornell2", width=16, height=16, spp=4, renderer="pt_cuda"))
    desc, _ = cfg.rendering(0)
    scene = DeviceScene(cfg)
    with pytest.raises(AtrcError, match="device pointers"):
        _render_noalloc(scene, desc, Film(16, 16))
    desc.path_pool = 1 << 24
    with pytest.raises(AtrcError, match="exceeds the maximum"):
        _render_noalloc(scene, desc, Film(16, 16, device=True))
