"""Batched multi-view rendering (atrc_cuda_render_batch): several views in one
wavefront equal the same views rendered one by one."""
import numpy as np
import pytest

from atrc_b200 import AtrcError, Config, DeviceScene, Film

pytestmark = pytest.mark.gpu


def _views(cfg, specs):
    out = []
    for (w, h, spp, shift, seed) in specs:
        d, _ = cfg.rendering(0)
        d.width, d.height, d.spp, d.seed = w, h, spp, seed
        d.camera.pos[0] += shift
        out.append(d)
    return out


def test_batch_equals_views_rendered_one_by_one(cornell_path):
    cfg = Config.from_file(cornell_path)
    dev = DeviceScene(cfg)
    specs = [(64, 48, 8, 0.0, 1), (32, 32, 32, 0.3, 2), (96, 80, 3, -0.2, 3), (8, 8, 64, 0.1, 4)]
    views = _views(cfg, specs)
    for d in views:
        d.sort_mode, d.path_pool = 0, 1 << 14
    batch = [Film(d.width, d.height, value_sq=True, device=True) for d in views]
    st, secs = dev.render_batch(views, batch)
    assert st["samples"] == sum(w * h * spp for w, h, spp, _, _ in specs)
    assert np.all(secs > 0) and np.all(secs <= st["seconds"] + 1e-6)
    for d, fb in zip(views, batch):
        one = Film(d.width, d.height, value_sq=True, device=True)
        dev.render(d, one)
        # one light: every path is the same in both runs; only the order of
        # the FP64 film atomics differs
        np.testing.assert_allclose(fb.value.cpu().numpy(), one.value.cpu().numpy(), rtol=1e-9, atol=1e-12)
        np.testing.assert_allclose(fb.weight.cpu().numpy(), one.weight.cpu().numpy(), rtol=1e-12)


def test_batch_rejects_mixed_settings(cornell_path):
    cfg = Config.from_file(cornell_path)
    dev = DeviceScene(cfg)
    views = _views(cfg, [(16, 16, 2, 0.0, 1), (16, 16, 2, 0.0, 2)])
    films = [Film(16, 16, device=True) for _ in views]
    views[1].max_depth += 1
    with pytest.raises(AtrcError, match="share"):
        dev.render_batch(views, films)
    views[1].max_depth -= 1
    with pytest.raises(AtrcError, match="device"):
        dev.render_batch(views, [Film(16, 16), films[1]])


def test_guided_batch(cornell_path):
    from atrc_b200.guide import Guide
    cfg = Config.from_file(cornell_path)
    dev = DeviceScene(cfg)
    g = Guide.for_scene(dev, log2_table=14, record_capacity=1 << 16, batch=1 << 14)
    train, _ = cfg.rendering(0)
    train.width, train.height, train.spp = 32, 32, 8
    dev.render_guided(g, train, Film(32, 32), record=True)
    g.train(steps=4)
    views = _views(cfg, [(48, 48, 16, 0.0, 5), (24, 24, 64, 0.2, 6)])
    films = [Film(d.width, d.height, device=True) for d in views]
    st, secs = dev.render_batch(views, films, guide=g)
    assert st["samples"] == 48 * 48 * 16 + 24 * 24 * 64
    for d, f in zip(views, films):
        img = f.image()
        assert np.all(np.isfinite(img)) and img.mean() > 0


def test_device_loop_long_paths_small_pool(scene_dir):
    # depth-32 paths through media with a 1024-path pool: many refills of the
    # pool inside one graph launch; the loop bound must not cut the render
    # short, and the batch must equal the single-view render of the same view
    from atrc_b200.scenes import media_scene
    cfg = Config.from_file(media_scene(scene_dir / "media_loop", width=24, height=24, spp=64, grid_res=32,
                                       sphere_level=3))
    dev = DeviceScene(cfg)
    d, _ = cfg.rendering(0)
    d.sort_mode, d.path_pool = 0, 1024
    fb = Film(d.width, d.height, device=True)
    st, secs = dev.render_batch([d], [fb])
    assert st["samples"] == 24 * 24 * 64 and st["watchdog_flags"] == 0
    # 36,864 samples through 1,024 slots: the pool is refilled about 36 times
    assert secs[0] > 0 and st["iterations"] > 40
    one = Film(d.width, d.height, device=True)
    dev.render(d, one)
    np.testing.assert_allclose(fb.weight.cpu().numpy(), one.weight.cpu().numpy(), rtol=1e-12)
    np.testing.assert_allclose(fb.value.cpu().numpy(), one.value.cpu().numpy(), rtol=1e-6, atol=1e-9)
