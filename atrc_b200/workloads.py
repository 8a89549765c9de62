"""Fixed workloads for profiling the kernels under ncu (each runs its scene
through the public API and exits; the renders are the same ones the bench
times).

    python -m atrc_b200.workloads instanced [--spp 2] [--warmup 3] [--steps 1]
        the 1920x1080 instanced Disney + IBL scene: scene build, autotune,
        warm-up steps, then `steps` steps of `spp` samples per pixel; each
        timed step is wrapped in an NVTX range named "step"
    python -m atrc_b200.workloads guided-room [--train-passes 3] [--passes 3]
        the 1280x720 indoor room: autotune, plain passes, guided passes that
        record and train, then guided passes that only sample (1 spp each)
    python -m atrc_b200.workloads subsurface [--spp 4] [--warmup 2] [--steps 1]
        the Cornell box at 1024x1024 with its two boxes made of Disney
        materials with subsurface scattering (the k_subsurface walk)
    python -m atrc_b200.workloads ploc
        the instanced scene with every mesh tree built by the device PLOC
        builder (bvh_gpu.cu), then one 1-spp render
    python -m atrc_b200.workloads rays [--count 10000000]
        closest-hit queries of seeded rays against the instanced scene
        through atrc_cuda_trace_rays (k_trace_rays)
"""
from __future__ import annotations

import argparse


def instanced(spp: int, warmup: int, steps: int) -> None:
    import torch

    from . import Config, DeviceScene, Film, scenes
    cfg = Config.from_file(scenes.instanced_disney())
    desc, _ = cfg.rendering(0)
    scene = DeviceScene(cfg)
    scene.autotune(desc, trial_spp=2)
    film = Film(desc.width, desc.height, device=True)
    desc.spp_count = spp
    for k in range(warmup + steps):
        desc.first_spp = k * spp
        if k >= warmup:
            torch.cuda.nvtx.range_push("step")
        stats = scene.render(desc, film)
        if k >= warmup:
            torch.cuda.synchronize()
            torch.cuda.nvtx.range_pop()
            print(f"step {k - warmup}: closest rays {stats['rays_closest']}, shadow rays {stats['rays_shadow']}")


def subsurface(spp: int, warmup: int, steps: int) -> None:
    import torch

    from . import Config, DeviceScene, Film, scenes
    cfg = Config.from_file(scenes.cornell_box(width=1024, height=1024, renderer="pt_cuda", subsurface=True))
    desc, _ = cfg.rendering(0)
    scene = DeviceScene(cfg)
    film = Film(desc.width, desc.height, device=True)
    desc.spp_count = spp
    for k in range(warmup + steps):
        desc.first_spp = k * spp
        stats = scene.render(desc, film)
        torch.cuda.synchronize()
        if k >= warmup:
            print(f"step {k - warmup}: closest rays {stats['rays_closest']}, shadow rays {stats['rays_shadow']}")


def ploc() -> None:
    import json
    from pathlib import Path

    from . import Config, DeviceScene, Film, scenes
    path = Path(scenes.instanced_disney())
    d = json.loads(path.read_text())
    d["scene"]["bvh_builder"] = "ploc"
    cfg = Config.from_string(json.dumps(d), str(path.parent))
    desc, _ = cfg.rendering(0)
    scene = DeviceScene(cfg)
    desc.spp_count = 1
    stats = scene.render(desc, Film(desc.width, desc.height, device=True))
    print(f"closest rays {stats['rays_closest']}")


def rays(count: int) -> None:
    import numpy as np

    from . import RAY_DTYPE, Config, DeviceScene, scenes
    cfg = Config.from_file(scenes.instanced_disney())
    desc, _ = cfg.rendering(0)
    scene = DeviceScene(cfg)
    rng = np.random.default_rng(7)
    r = np.zeros(count, RAY_DTYPE)
    r["o"] = np.broadcast_to(np.asarray(desc.camera.pos, np.float32), (count, 3))
    tgt = rng.uniform(-20, 20, (count, 3))
    dd = tgt - r["o"]
    r["d"] = dd / np.linalg.norm(dd, axis=1, keepdims=True)
    r["t_max"] = np.inf
    for _ in range(2):
        h = scene.trace_rays(r, "closest")
    print(f"hits {(h['entity'] >= 0).mean():.3f}")


def guided_room(train_passes: int, passes: int) -> None:
    import torch

    from . import Config, DeviceScene, Film, scenes
    from .guide import Guide
    cfg = Config.from_file(scenes.indoor_room())
    desc, _ = cfg.rendering(0)
    scene = DeviceScene(cfg)
    scene.autotune(desc, trial_spp=1)
    film = Film(desc.width, desc.height, device=True)
    desc.spp_count = 1
    for k in range(3):
        desc.first_spp = k
        scene.render(desc, film)
    guide = Guide.for_scene(scene)
    # the last recording pass (with its Adam steps) and the last guided pass
    # run inside NVTX ranges "train_pass" and "guided_pass" for profilers
    for k in range(train_passes):
        desc.first_spp = 3 + k
        last = k == train_passes - 1
        if last:
            torch.cuda.nvtx.range_push("train_pass")
        scene.render_guided(guide, desc, film, record=True)
        guide.train(steps=4)
        if last:
            torch.cuda.synchronize()
            torch.cuda.nvtx.range_pop()
    for k in range(passes):
        desc.first_spp = 3 + train_passes + k
        last = k == passes - 1
        if last:
            torch.cuda.nvtx.range_push("guided_pass")
        scene.render_guided(guide, desc, film, record=False)
        if last:
            torch.cuda.synchronize()
            torch.cuda.nvtx.range_pop()
    guide.close()


def main() -> None:
    p = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    sub = p.add_subparsers(dest="workload", required=True)
    a = sub.add_parser("instanced")
    a.add_argument("--spp", type=int, default=2)
    a.add_argument("--warmup", type=int, default=3)
    a.add_argument("--steps", type=int, default=1)
    b = sub.add_parser("guided-room")
    b.add_argument("--train-passes", type=int, default=3)
    b.add_argument("--passes", type=int, default=3)
    sub.add_parser("ploc")
    e = sub.add_parser("rays")
    e.add_argument("--count", type=int, default=10_000_000)
    c = sub.add_parser("subsurface")
    c.add_argument("--spp", type=int, default=4)
    c.add_argument("--warmup", type=int, default=2)
    c.add_argument("--steps", type=int, default=1)
    args = p.parse_args()
    if args.workload == "instanced":
        instanced(args.spp, args.warmup, args.steps)
    elif args.workload == "subsurface":
        subsurface(args.spp, args.warmup, args.steps)
    elif args.workload == "ploc":
        ploc()
    elif args.workload == "rays":
        rays(args.count)
    else:
        guided_room(args.train_passes, args.passes)


if __name__ == "__main__":
    main()
