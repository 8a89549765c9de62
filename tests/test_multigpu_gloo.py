"""The sample-split multi-GPU path on CPU: two gloo ranks render disjoint
sample ranges (with the oracle standing in for the GPU kernels) and reduce
their films to rank 0 after every step, as the benchmark's timed loop does;
the result equals rendering every range in one process, each sample counted
once."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from atrc_b200.multigpu import first_spp

STEPS = 2


def test_sample_ranges_are_disjoint():
    seen = set()
    for step in range(3):
        for rank in range(4):
            a = first_spp(step, rank, 4, 8)
            r = set(range(a, a + 8))
            assert not (r & seen)
            seen |= r
    assert seen == set(range(3 * 4 * 8))
    with pytest.raises(ValueError):
        first_spp(0, 2, 2, 8)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, scene_path, out_dir):
    import torch
    import torch.distributed as dist

    import oracle
    from atrc_b200 import Config, Film
    from atrc_b200.multigpu import reduce_film
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    cfg = Config.from_file(scene_path)
    desc, _ = cfg.rendering(0)
    ora = oracle.OracleScene(cfg.scene_desc(), desc.eps)
    tf = type("F", (), {})()
    tf.value = torch.zeros(desc.width * desc.height * 3, dtype=torch.float64)
    tf.weight = torch.zeros(desc.width * desc.height, dtype=torch.float64)
    desc.spp_count = 2
    for step in range(STEPS):
        film = Film(desc.width, desc.height)
        film.value[:] = tf.value.numpy().reshape(film.value.shape)
        film.weight[:] = tf.weight.numpy().reshape(film.weight.shape)
        desc.first_spp = first_spp(step, rank, world, 2)
        ora.render(desc, film, threads=1)
        tf.value.copy_(torch.from_numpy(film.value.reshape(-1)))
        tf.weight.copy_(torch.from_numpy(film.weight.reshape(-1)))
        reduce_film(tf, dist, 0)
        if rank != 0:
            assert not tf.value.any() and not tf.weight.any()
    if rank == 0:
        np.save(os.path.join(out_dir, "value.npy"), tf.value.numpy())
        np.save(os.path.join(out_dir, "weight.npy"), tf.weight.numpy())
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_gloo_film_reduce(tmp_path):
    import oracle
    from atrc_b200 import Config, Film
    from atrc_b200.scenes import cornell_box
    scene = cornell_box(tmp_path / "c", width=24, height=16, spp=4)
    mp.start_processes(_worker, args=(2, _free_port(), str(scene), str(tmp_path)), nprocs=2, start_method="spawn")
    value = np.load(tmp_path / "value.npy")
    weight = np.load(tmp_path / "weight.npy")
    cfg = Config.from_file(scene)
    desc, _ = cfg.rendering(0)
    ora = oracle.OracleScene(cfg.scene_desc(), desc.eps)
    ref = Film(desc.width, desc.height)
    desc.spp_count = 2
    for step in range(STEPS):
        for rank in range(2):
            desc.first_spp = first_spp(step, rank, 2, 2)
            ora.render(desc, ref, threads=1)
    np.testing.assert_allclose(value.reshape(ref.value.shape), ref.value, rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(weight.reshape(ref.weight.shape), ref.weight, rtol=1e-12)
    assert weight.sum() > 0
