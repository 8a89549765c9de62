"""Known answers and API behaviour of the CUDA path (through the C ABI)."""
import ctypes as C
import math
import threading

import numpy as np
import pytest

from atrc_b200 import AtrcError, Config, DeviceScene, Film
from tests import kat_scenes as K

pytestmark = pytest.mark.gpu


def _dev(cfg_dict, scene_dir="."):
    cfg = Config.from_string(K.dumps(cfg_dict), scene_dir)
    desc, _ = cfg.rendering(0)
    return cfg, desc, DeviceScene(cfg)


def test_white_furnace_gpu():
    cfg, desc, dev = _dev(K.furnace(spp=256, renderer="pt_cuda"))
    f = Film(desc.width, desc.height, value_sq=True)
    dev.render(desc, f)
    mu = f.image().mean()
    n = float(f.weight.sum()) * 4 * (0.5 - 3e-4) ** 2
    var = f.value_sq.sum() / f.weight.sum() / 3 - mu * mu
    assert abs(mu - 1.0) < 4 * math.sqrt(max(var, 1e-12) / n) + 1e-3, mu


def test_absorbing_slab_gpu(tmp_path):
    cfgd, expected = K.slab(tmp_path, renderer="pt_cuda")
    cfg, desc, dev = _dev(cfgd, tmp_path)
    f = Film(desc.width, desc.height)
    dev.render(desc, f)
    np.testing.assert_allclose(f.image()[4, 4], expected, rtol=2e-3)


def test_moller_trumbore_edges_gpu():
    import oracle
    cfg, desc, dev = _dev(K.edge_scene())
    rays, inside = K.edge_rays()
    for exact in (True, False):
        h = dev.trace_rays(rays, exact=exact)
        assert np.array_equal(h["entity"] >= 0, inside)
        assert np.all(h["t"][inside] == np.float32(2.0))
    ref = oracle.OracleScene(cfg.scene_desc()).trace_rays(rays)
    assert np.array_equal(dev.trace_rays(rays, exact=True)["t"], ref["t"])


def test_sample_split_is_exact(cornell_path):
    # sample indices [0, 8) at once == [0, 4) + [4, 8): the multi-GPU sharding
    cfg = Config.from_file(cornell_path)
    desc, _ = cfg.rendering(0)
    desc.width, desc.height = 40, 32
    dev = DeviceScene(cfg)
    whole, split = Film(40, 32, value_sq=True), Film(40, 32, value_sq=True)
    desc.first_spp, desc.spp_count = 0, 8
    dev.render(desc, whole)
    for first in (0, 4):
        desc.first_spp, desc.spp_count = first, 4
        dev.render(desc, split)
    for name in ("value", "weight", "value_sq"):
        np.testing.assert_allclose(getattr(split, name), getattr(whole, name), rtol=1e-9, atol=1e-12)


def test_device_film_equals_host_film(cornell_path):
    cfg = Config.from_file(cornell_path)
    desc, _ = cfg.rendering(0)
    desc.width, desc.height, desc.spp = 32, 24, 8
    dev = DeviceScene(cfg)
    a, b = Film(32, 24), Film(32, 24, device=True)
    dev.render(desc, a)
    dev.render(desc, b)
    np.testing.assert_allclose(b.value.cpu().numpy(), a.value, rtol=1e-9, atol=1e-12)


def test_cancel_returns_partial_film(cornell_path):
    cfg = Config.from_file(cornell_path)
    desc, _ = cfg.rendering(0)
    desc.width, desc.height, desc.spp = 256, 256, 4096
    desc.path_pool = 1 << 16
    dev = DeviceScene(cfg)
    f = Film(256, 256)
    flag = [False]
    seen = []

    def progress(p):
        seen.append(p)
        if len(seen) == 3:
            flag[0] = True
    with pytest.raises(AtrcError, match="CANCELLED"):
        dev.render(desc, f, should_stop=lambda: flag[0], progress=progress)
    done = f.weight.sum() * 4 * (0.5 - 3e-4) ** 2
    assert 0 < done < 256 * 256 * 4096


def test_invalid_arguments_are_rejected(cornell_path):
    cfg = Config.from_file(cornell_path)
    desc, _ = cfg.rendering(0)
    dev = DeviceScene(cfg)
    bad = Film(desc.width, desc.height)
    desc.spp = 0
    with pytest.raises(AtrcError, match="INVALID_ARG"):
        dev.render(desc, bad)
    desc.spp = 4
    desc.filter_radius = 0.0001
    with pytest.raises(AtrcError, match="filter"):
        dev.render(desc, bad)
    from atrc_b200 import _abi as abi
    from atrc_b200 import load_library
    rays = np.zeros(4, dtype=abi.AtrcRay)
    hits = np.zeros(4, dtype=abi.AtrcHit)
    rc = load_library().atrc_cuda_trace_rays(dev.handle, rays.ctypes.data_as(C.POINTER(abi.AtrcRay)), 4,
                                             hits.ctypes.data_as(C.POINTER(abi.AtrcHit)), 7, 1)
    assert rc == -1


def test_empty_scene_and_threads(tmp_path):
    cfgd = K.furnace(renderer="pt_cuda", spp=4)
    cfgd["scene"]["entities"] = []
    cfg, desc, dev = _dev(cfgd)
    f = Film(desc.width, desc.height)
    dev.render(desc, f)
    np.testing.assert_allclose(f.image(), 1.0, rtol=1e-6)  # only the uniform sky
    # two scenes rendered from two host threads at once
    cfg2, desc2, dev2 = _dev(K.furnace(renderer="pt_cuda", spp=16))
    out = {}

    def run(k, d, s):
        ff = Film(d.width, d.height)
        s.render(d, ff)
        out[k] = ff.image().mean()
    ts = [threading.Thread(target=run, args=(k, desc2, dev2 if k else dev)) for k in range(2)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    assert abs(out[0] - 1) < 1e-5 and abs(out[1] - 1) < 0.05


@pytest.mark.parametrize("scene", ["cornell", "media", "phong", "materials"])
def test_shade_queue_sort_changes_nothing(scene, cornell_path, scene_dir, tmp_path):
    # sorting hit records by material key only reorders the shade queue: every
    # path keeps its own random stream, so the films agree up to the order in
    # which the FP32 shadow-ray results of several lights add into one path.
    # "phong": three materials, one of the last type (type-sort key 8 with
    # fewer materials than types); "materials": every surface type but two
    from atrc_b200 import scenes
    if scene in ("phong", "materials"):
        d = K.materials_scene(tmp_path)
        if scene == "phong":
            d["scene"]["entities"] = [d["scene"]["entities"][k] for k in (0, 5, 6)]
        cfg = Config.from_string(K.dumps(d), str(tmp_path))
    else:
        cfg = Config.from_file(cornell_path if scene == "cornell" else scenes.media_scene(scene_dir))
    desc, _ = cfg.rendering(0)
    desc.width, desc.height, desc.spp = 64, 48, 8
    dev = DeviceScene(cfg)
    films = []
    for mode in (0, 1, 2):
        desc.sort_mode = mode
        f = Film(desc.width, desc.height, value_sq=True)
        dev.render(desc, f)
        films.append(f)
    for f in films[1:]:
        np.testing.assert_allclose(f.value, films[0].value, rtol=2e-6, atol=1e-9)
        np.testing.assert_allclose(f.weight, films[0].weight, rtol=1e-12)
    desc.sort_mode = 5
    with pytest.raises(AtrcError, match="sort_mode"):
        dev.render(desc, Film(desc.width, desc.height))


def test_render_stats_are_filled(cornell_path):
    # per-kernel device times come from events recorded inside the captured
    # bounce-loop graph
    cfg = Config.from_file(cornell_path)
    desc, _ = cfg.rendering(0)
    desc.width, desc.height, desc.spp = 64, 64, 16
    dev = DeviceScene(cfg)
    st = dev.render(desc, Film(64, 64))
    assert st["samples"] == 64 * 64 * 16
    assert st["extend_seconds"] > 0 and st["shade_seconds"] > 0 and st["shadow_seconds"] > 0
    assert st["extend_seconds"] + st["shade_seconds"] + st["shadow_seconds"] <= st["kernel_seconds"] * 1.01
    assert st["rays_closest"] >= st["samples"] and st["kernel_launches"] > 6


def test_autotune_picks_a_valid_configuration(cornell_path):
    cfg = Config.from_file(cornell_path)
    desc, _ = cfg.rendering(0)
    desc.width, desc.height, desc.spp = 128, 96, 8
    dev = DeviceScene(cfg)
    ref = Film(128, 96)
    desc.sort_mode, desc.path_pool = 0, 1 << 16
    dev.render(desc, ref)
    t = dev.autotune(desc, trial_spp=2)
    assert t["trials"] >= 4 and t["sort_mode"] in (0, 1, 2)
    assert t["path_pool"] >= 1024 and t["ms_per_msample"] > 0
    assert t["ms_per_msample"] <= t["default_ms_per_msample"] * 1.0001
    assert dev.tuning() == t
    # renders that leave the choice to the library use it; the image does
    # not depend on the launch configuration (one light: bit-exact paths)
    desc.sort_mode, desc.path_pool = -1, 0
    f = Film(128, 96)
    dev.render(desc, f)
    np.testing.assert_allclose(f.value, ref.value, rtol=1e-9, atol=1e-12)
    with pytest.raises(AtrcError, match="out of range"):
        dev.set_tuning(gen_threads=100)
    dev.set_tuning(sort_mode=2, path_pool=4096)
    assert dev.tuning()["sort_mode"] == 2 and dev.tuning()["path_pool"] == 4096


@pytest.mark.parametrize("sort_mode", [0, 2])
def test_extend_fetch_matches_one_ray_per_thread(scene_dir, sort_mode):
    # k_extend_fetch (persistent warps refilling finished lanes) finds the
    # same closest hits as k_extend: the same paths, traversal work and film
    from atrc_b200.scenes import instanced_disney
    p = instanced_disney(scene_dir / "inst_small", ico_level=4, hf_res=128, width=64, height=36, spp=64)
    cfg = Config.from_file(p)
    desc, _ = cfg.rendering(0)
    desc.sort_mode, desc.count_traversal = sort_mode, 1
    dev = DeviceScene(cfg)
    out = []
    for fetch in (0, 1):
        dev.set_tuning(extend_fetch=fetch, path_pool=1 << 14)
        f = Film(desc.width, desc.height)
        st = dev.render(desc, f)
        assert st["watchdog_flags"] == 0
        out.append((f, st))
    (fa, sa), (fb, sb) = out
    for k in ("samples", "rays_closest", "rays_shadow"):
        assert sa[k] == sb[k], k
    # the work differs a little: a lane visits its parked leaf when its whole
    # warp holds leaves, and which rays share a warp differs between kernels
    for k in ("nodes_closest", "tris_closest", "ents_closest"):
        assert abs(sa[k] - sb[k]) <= 0.01 * sa[k], k
    # (shadow contributions are FP32 atomics, whose order may differ)
    np.testing.assert_allclose(fb.value, fa.value, rtol=2e-6, atol=1e-9)
    np.testing.assert_array_equal(fb.weight, fa.weight)


@pytest.mark.parametrize("scene", ["instanced", "media", "subsurface"])
@pytest.mark.parametrize("sort_mode", [0, 2])
def test_queue_order_changes_nothing(scene, sort_mode, scene_dir, tmp_path):
    # the extend queue in slot order (continuations marked per slot, queued
    # by the slot scan) or in shade order (continuations appended by k_shade
    # and k_subsurface) holds the same paths: same samples, rays and film,
    # with a pool small enough that slots are reused many times
    from atrc_b200 import scenes
    if scene == "instanced":
        cfg = Config.from_file(scenes.instanced_disney(scene_dir / "inst_small", ico_level=4, hf_res=128,
                                                       width=64, height=36, spp=64))
    elif scene == "media":
        cfg = Config.from_file(scenes.media_scene(scene_dir))
    else:
        cfg = Config.from_string(K.dumps(K.subsurface_scene(tmp_path)), str(tmp_path))
    desc, _ = cfg.rendering(0)
    desc.width, desc.height, desc.spp = 64, 36, 32
    desc.sort_mode = sort_mode
    dev = DeviceScene(cfg)
    out = []
    for q in (0, 1):
        dev.set_tuning(queue_order=q, path_pool=1 << 13)
        assert dev.tuning()["queue_order"] == q
        f = Film(desc.width, desc.height)
        st = dev.render(desc, f)
        assert st["watchdog_flags"] == 0
        out.append((f, st))
    (fa, sa), (fb, sb) = out
    assert sa["samples"] == sb["samples"] == desc.width * desc.height * desc.spp
    for k in ("rays_closest", "rays_shadow"):
        assert sa[k] == sb[k], k
    np.testing.assert_allclose(fb.value, fa.value, rtol=2e-6, atol=1e-9)
    np.testing.assert_array_equal(fb.weight, fa.weight)


@pytest.mark.parametrize("scene", ["instanced", "media"])
def test_shadow_fetch_matches_one_ray_per_thread(scene, scene_dir):
    # k_shadow_fetch (persistent warps refilling finished lanes from the
    # shadow queue) decides the same occlusions as k_shadow: same rays,
    # traversal work and film
    from atrc_b200 import scenes
    if scene == "instanced":
        p = scenes.instanced_disney(scene_dir / "inst_small", ico_level=4, hf_res=128, width=64, height=36, spp=64)
    else:
        p = scenes.media_scene(scene_dir)
    cfg = Config.from_file(p)
    desc, _ = cfg.rendering(0)
    desc.width, desc.height, desc.spp = 64, 36, 32
    desc.count_traversal = 1
    dev = DeviceScene(cfg)
    out = []
    for fetch in (0, 1):
        dev.set_tuning(shadow_fetch=fetch, path_pool=1 << 14)
        assert dev.tuning()["shadow_fetch"] == fetch
        f = Film(desc.width, desc.height)
        st = dev.render(desc, f)
        assert st["watchdog_flags"] == 0
        out.append((f, st))
    (fa, sa), (fb, sb) = out
    for k in ("samples", "rays_closest", "rays_shadow"):
        assert sa[k] == sb[k], k
    assert sa["rays_shadow"] > 0
    # which rays share a warp differs, and with it leaf postponement's visits
    for k in ("nodes_shadow", "tris_shadow", "ents_shadow"):
        assert abs(sa[k] - sb[k]) <= 0.01 * sa[k], k
    np.testing.assert_allclose(fb.value, fa.value, rtol=2e-6, atol=1e-9)
    np.testing.assert_array_equal(fb.weight, fa.weight)


@pytest.mark.parametrize("scene", ["cornell", "media", "instanced"])
def test_shadow_queue_sort_changes_nothing(scene, cornell_path, scene_dir):
    # the shadow-queue sort (AtrcTuning.shadow_sort) only changes the order in
    # which any-hit rays are traced: the films agree up to the order in which
    # the FP32 shadow-ray results of several lights add into one path
    from atrc_b200 import scenes
    if scene == "cornell":
        cfg = Config.from_file(cornell_path)
    elif scene == "media":
        cfg = Config.from_file(scenes.media_scene(scene_dir / "media_shsort", grid_res=32, sphere_level=3))
    else:
        cfg = Config.from_file(scenes.instanced_disney(scene_dir / "inst_shsort", ico_level=4, hf_res=128))
    desc, _ = cfg.rendering(0)
    desc.width, desc.height, desc.spp = 64, 48, 8
    desc.path_pool = 1 << 14  # slots are reused: the queue is sorted in every iteration
    dev = DeviceScene(cfg)
    films = []
    for on in (0, 1):
        dev.set_tuning(shadow_sort=on)
        assert dev.tuning()["shadow_sort"] == on
        f = Film(desc.width, desc.height, value_sq=True)
        st = dev.render(desc, f)
        assert st["watchdog_flags"] == 0 and st["rays_shadow"] > 0
        films.append(f)
    np.testing.assert_allclose(films[1].value, films[0].value, rtol=2e-6, atol=1e-9)
    np.testing.assert_allclose(films[1].weight, films[0].weight, rtol=1e-12)
