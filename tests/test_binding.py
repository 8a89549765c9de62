"""The reference-side pt_cuda plugin (atrc_b200/csrc/plugin/pt_cuda_renderer.hpp)
compiled against stand-ins of Atrc's interfaces (tests/binding/reference_stubs.h).

* CPU: every entry of a two-entry "rendering" array, created through the
  creating context the way Atrc's CLI creates it, composes to JSON that loads
  to the same AtrcRenderDesc as the whole scene file's entry.  The groups are
  handed over as factory::config_to_json prints them (every value a string,
  floats with six decimals, src/factory/src/utility/config_cvt.cpp:10-48).
* GPU: with the reference's Renderer member layout (renderer.h:17-24), a
  render_async that raises doing_rendering_ runs to the end, and stop_async
  (which raises stop_rendering_) stops the next one early with the samples
  taken so far.
"""
import json
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
BINDING = ROOT / "tests" / "binding"


def _build(tmp_path: Path) -> Path:
    from atrc_b200 import build
    lib = build.build_library()
    exe = tmp_path / "binding_test"
    subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", f"-I{BINDING}", f"-I{ROOT / 'atrc_b200/csrc/plugin'}",
                    f"-I{ROOT / 'include'}", str(BINDING / "binding_test.cpp"), "-o", str(exe),
                    f"-L{lib.parent}", "-latrc_cuda", f"-Wl,-rpath,{lib.parent}", "-lpthread"],
                   check=True, capture_output=True, text=True)
    return exe


def _as_config_values(node):
    """A JSON node as config_to_json prints it: scalars become the strings
    ConfigValue holds (config_cvt.cpp:40-48)."""
    if isinstance(node, dict):
        return {k: _as_config_values(v) for k, v in node.items()}
    if isinstance(node, list):
        return [_as_config_values(v) for v in node]
    if isinstance(node, bool):
        return "1" if node else "0"
    if isinstance(node, int):
        return str(node)
    if isinstance(node, float):
        return "%f" % float(np.float32(node))
    return node


def _write_plan(tmp_path: Path, scene_file: Path) -> Path:
    root = json.loads(scene_file.read_text())
    rendering = root["rendering"] if isinstance(root["rendering"], list) else [root["rendering"]]
    (tmp_path / "scene_group.json").write_text(json.dumps(_as_config_values(root["scene"])))
    lines = [f"scene_dir {scene_file.parent}", f"scene {tmp_path / 'scene_group.json'}"]
    for i, r in enumerate(rendering):
        cam = tmp_path / f"camera{i}.json"
        cam.write_text(json.dumps(_as_config_values(r["camera"])))
        ren = tmp_path / f"renderer{i}.json"
        ren.write_text(json.dumps(_as_config_values(r["renderer"])))
        if "film_filter" in r:
            ff = tmp_path / f"filter{i}.json"
            ff.write_text(json.dumps(_as_config_values(r["film_filter"])))
            ftype, fpath = r["film_filter"]["type"], str(ff)
        else:
            ftype, fpath = "-", "-"
        eps = "%f" % float(np.float32(r.get("eps", 3e-4)))
        lines.append(f"entry {r['width']} {r['height']} {eps} {r['camera']['type']} {cam} {ftype} {fpath} {ren}")
    plan = tmp_path / "plan.txt"
    plan.write_text("\n".join(lines) + "\n")
    return plan


def _two_entry_scene(tmp_path: Path) -> Path:
    from atrc_b200.scenes import cornell_box
    path = cornell_box(tmp_path / "cornell", width=40, height=30, spp=8, renderer="pt_cuda")
    root = json.loads(path.read_text())
    first = root["rendering"]
    second = json.loads(json.dumps(first))
    second["width"], second["height"] = 24, 36
    second["camera"]["pos"] = [0.25, -0.1, 3.5]
    second["camera"]["fov"] = 33.5
    second["film_filter"] = {"type": "gaussian", "radius": 1.5, "alpha": 2.5}
    second["renderer"] = {"type": "pt_cuda", "spp": 3, "min_depth": 3, "max_depth": 11, "cont_prob": 0.75,
                          "specular_depth": 7, "use_mis": 0, "task_grid_size": 16}
    second["eps"] = 0.0005
    del first["film_filter"]
    root["rendering"] = [first, second]
    path.write_text(json.dumps(root, indent=1))
    return path


def test_binding_compose_matches_whole_config(tmp_path):
    from atrc_b200 import Config
    exe = _build(tmp_path)
    scene = _two_entry_scene(tmp_path)
    plan = _write_plan(tmp_path, scene)
    r = subprocess.run([str(exe), "compose", str(plan)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    got = [json.loads(line) for line in r.stdout.splitlines()]
    cfg = Config.from_file(scene)
    assert cfg.rendering_count() == len(got) == 2
    for i, g in enumerate(got):
        want, kind = cfg.rendering(i)
        assert g["type"] == kind == "pt_cuda"
        for k in ("width", "height", "spp", "min_depth", "max_depth", "specular_depth", "use_mis", "filter_type",
                  "task_grid_size"):
            assert g[k] == getattr(want, k), (i, k)
        for k in ("cont_prob", "filter_radius", "filter_alpha", "eps"):
            assert g[k] == pytest.approx(float(getattr(want, k)), rel=0, abs=0), (i, k)
        for k in ("fov", "lens_radius", "focal_distance"):
            assert g[k] == pytest.approx(float(getattr(want.camera, k)), rel=0, abs=0), (i, k)
        assert g["pos"] == [pytest.approx(float(x), rel=0, abs=0) for x in want.camera.pos]
    # the two entries differ, so neither was read from the other
    assert got[0]["spp"] != got[1]["spp"] and got[0]["filter_type"] != got[1]["filter_type"]


def test_binding_refuses_use_mis_zero(tmp_path):
    # the second entry asks for use_mis = 0 (the reference's trace_nomis):
    # render() throws before building a device scene, with a message that
    # names the key; the first entry does not fail for that reason
    exe = _build(tmp_path)
    scene = _two_entry_scene(tmp_path)
    plan = _write_plan(tmp_path, scene)
    r = subprocess.run([str(exe), "refuse", str(plan)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    got = [json.loads(line) for line in r.stdout.splitlines()]
    assert [g["entry"] for g in got] == [0, 1]
    assert "use_mis = 0" in got[1]["error"] and "trace_nomis" in got[1]["error"]
    assert "use_mis" not in got[0]["error"]


@pytest.mark.gpu
def test_binding_async_cancel_uses_stop_rendering_only(tmp_path):
    from atrc_b200.scenes import cornell_box
    exe = _build(tmp_path)
    scene = cornell_box(tmp_path / "cornell", width=256, height=256, spp=2048, renderer="pt_cuda")
    root = json.loads(scene.read_text())
    root["rendering"]["renderer"]["path_pool"] = 1 << 16  # many windows, many progress reports
    scene.write_text(json.dumps(root, indent=1))
    plan = _write_plan(tmp_path, scene)
    r = subprocess.run([str(exe), "async", str(plan)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    out = json.loads(r.stdout.splitlines()[0])
    # The box filter has radius r = 0.5 - eps and value 1 / (4 r^2); a sample
    # adds it to its pixel when it lies within r of the centre on both axes
    # (probability (2r)^2), so E[weight] = 1 per sample and the total of N
    # samples is N within a few standard deviations of the Bernoulli draws.
    rad = 0.5 - 3e-4
    n = 256 * 256 * 2048
    p_in = (2 * rad) ** 2
    sd = np.sqrt(n * p_in * (1 - p_in)) / (4 * rad * rad)
    full = float(n)
    # doing_rendering_ was raised for the whole render and did not cancel it
    assert out["doing_seen"] == 1 and out["full_status"] == 0
    assert abs(out["full_weight"] - full) < 6 * sd, (out["full_weight"] - full, sd)
    assert out["image_rows"] == 256
    # stop_async raised stop_rendering_: cancelled, with a partial film
    assert out["stop_status"] == -5  # ATRC_ERR_CANCELLED
    assert 0 < out["stop_weight"] < full
    assert out["stop_progress"] >= 2 and out["doing_after"] == 0
