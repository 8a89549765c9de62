"""Scene ingestion: the factory mirror of the reference's creators (CPU only)."""
import ctypes as C
import json

import numpy as np
import pytest

from atrc_b200 import AtrcError, Config


def base(entities, rendering=None, **scene):
    r = {"camera": {"type": "thin_lens", "pos": [0, 0, 5], "dst": [0, 0, 0], "up": [0, 1, 0], "fov": 40},
         "width": 32, "height": 16, "renderer": {"type": "pt", "spp": 4}, "reporter": {"type": "noout"}}
    if rendering:
        r.update(rendering)
    return {"scene": {"type": "default", "entities": entities, **scene}, "rendering": r}


QUAD = {"type": "geometric",
        "geometry": {"type": "quad", "A": [-1, -1, 0], "B": [1, -1, 0], "C": [1, 1, 0], "D": [-1, 1, 0],
                     "transform": []},
        "material": {"type": "ideal_diffuse", "albedo": {"type": "constant", "texel": [0.5]}}}


def test_pt_defaults_match_reference_creator():
    # renderer_creators.cpp:127-146
    cfg = Config.from_string(base([QUAD]))
    d, kind = cfg.rendering(0)
    assert kind == "pt"
    assert (d.spp, d.min_depth, d.max_depth, d.specular_depth, d.use_mis) == (4, 5, 10, 20, 1)
    assert d.cont_prob == pytest.approx(0.9)
    assert d.eps == pytest.approx(3e-4)
    assert d.filter_type == 0 and d.filter_radius == pytest.approx(0.5)
    assert d.camera.fov == pytest.approx(np.deg2rad(40), rel=1e-6)
    assert d.camera.focal_distance == 1 and d.camera.lens_radius == 0


def test_pt_cuda_accepts_pt_keys():
    cfg = Config.from_string(base([QUAD], {"renderer": {"type": "pt_cuda", "spp": 8, "min_depth": 2,
                                                        "max_depth": 7, "cont_prob": 0.5}}))
    d, kind = cfg.rendering(0)
    assert kind == "pt_cuda" and (d.spp, d.min_depth, d.max_depth) == (8, 2, 7)
    assert d.cont_prob == pytest.approx(0.5)


def test_floats_round_trip_through_six_decimals():
    # config_cvt.cpp:43: std::to_string then std::stof
    q = json.loads(json.dumps(QUAD))
    q["geometry"]["A"] = [-1.23456789, -1, 0]
    cfg = Config.from_string(base([q]))
    g = cfg.scene_desc().contents.geometries[0]
    assert g.p[0][0] == np.float32(-1.234568)


def test_entity_skip_suffix_and_void_medium():
    skipped = dict(QUAD, type="geometric//")
    cfg = Config.from_string(base([QUAD, skipped]))
    s = cfg.scene_desc().contents
    assert s.entity_count == 1
    assert s.medium_count >= 1 and s.media[0].type == 0  # the void medium
    e = s.entities[0]
    assert e.medium_in == 0 and e.medium_out == 0 and e.power == -1


def test_transform_list_applies_last_first():
    q = json.loads(json.dumps(QUAD))
    q["geometry"]["transform"] = [{"type": "translate", "offset": [1, 2, 3]}, {"type": "scale", "ratio": 2}]
    cfg = Config.from_string(base([q]))
    m = np.array(cfg.scene_desc().contents.geometries[0].transform.m).reshape(3, 4)
    p = m[:, :3] @ np.array([1.0, 1.0, 1.0]) + m[:, 3]
    assert np.allclose(p, [3, 4, 5])  # scale first, then translate
    inv = np.array(cfg.scene_desc().contents.geometries[0].transform.inv).reshape(3, 4)
    assert np.allclose(inv[:, :3] @ p + inv[:, 3], [1, 1, 1])


def test_rotate_and_mat3():
    q = json.loads(json.dumps(QUAD))
    q["geometry"]["transform"] = [{"type": "rotate_z", "deg": 90}]
    c1 = Config.from_string(base([q]))
    m = np.array(c1.scene_desc().contents.geometries[0].transform.m).reshape(3, 4)
    assert np.allclose(m[:, :3] @ [1, 0, 0], [0, 1, 0], atol=1e-6)
    q["geometry"]["transform"] = {"type": "mat3", "row_major": [0, -1, 0, 1, 0, 0, 0, 0, 1]}
    c2 = Config.from_string(base([q]))
    m2 = np.array(c2.scene_desc().contents.geometries[0].transform.m).reshape(3, 4)
    assert np.allclose(m2, m, atol=1e-6)


def test_reference_creator_shares_geometry(tmp_path):
    from atrc_b200.scenes import _box_mesh, write_bm
    p, n, uv = _box_mesh((1, 1, 1))
    write_bm(tmp_path / "b.bm", p, n, uv)
    ents = []
    for k in range(3):
        ents.append({"type": "geometric",
                     "geometry": {"type": "transform_wrapper",
                                  "internal": {"type": "reference", "name": ["lib", "box"]},
                                  "transform": [{"type": "translate", "offset": [3 * k, 0, 0]}]},
                     "material": {"type": "ideal_diffuse", "albedo": {"type": "constant", "texel": [0.5]}}})
    cfg = Config.from_string(base(ents, lib={"box": {"type": "triangle_bvh", "filename": "${scene-directory}/b.bm",
                                                     "transform": []}}), tmp_path)
    s = cfg.scene_desc().contents
    assert s.entity_count == 3 and s.geometry_count == 1 and s.mesh_count == 1
    assert s.meshes[0].triangle_count == 12
    assert all(s.entities[i].geometry == 0 and s.entities[i].has_instance for i in range(3))
    assert s.entities[2].instance.m[3] == pytest.approx(6.0)


def test_bm_mesh_layout(tmp_path):
    from atrc_b200.scenes import write_bm
    pos = np.arange(18, dtype=np.float32).reshape(2, 3, 3)
    nor = np.ones((2, 3, 3), np.float32)
    uv = np.zeros((2, 3, 2), np.float32)
    write_bm(tmp_path / "m.bm", pos, nor, uv)
    q = {"type": "geometric", "geometry": {"type": "triangle_bvh", "filename": "${scene-directory}/m.bm",
                                           "transform": []},
         "material": {"type": "ideal_black"}}
    cfg = Config.from_string(base([q]), tmp_path)
    s = cfg.scene_desc().contents
    m = s.meshes[0]
    v = np.ctypeslib.as_array(m.vertices, shape=(int(m.triangle_count) * 24,))
    assert np.array_equal(v.reshape(2, 3, 8)[..., :3], pos)


def test_disney_defaults():
    q = json.loads(json.dumps(QUAD))
    q["material"] = {"type": "disney", "base_color": {"type": "constant", "texel": [0.2, 0.4, 0.6]},
                     "metallic": {"type": "constant", "texel": [0.0]},
                     "roughness": {"type": "constant", "texel": [0.3]}}
    cfg = Config.from_string(base([q]))
    s = cfg.scene_desc().contents
    m = s.materials[0]
    assert m.type == 2
    tex = lambda k: s.textures2d[m.tex[k]].texel[0]  # noqa: E731
    # material_creators.cpp:56-113 defaults
    assert tex(3) == 0 and tex(5) == pytest.approx(1.5) and tex(6) == 1 and tex(7) == 0
    assert tex(12) == 1 and m.tex[4] == m.tex[2]  # transmission_roughness defaults to roughness


def test_unknown_types_fail_loudly():
    q = json.loads(json.dumps(QUAD))
    q["material"] = {"type": "paper", "color": {"type": "constant", "texel": [0.5]}}
    with pytest.raises(AtrcError, match="not supported"):
        Config.from_string(base([q]))
    q["material"] = {"type": "glass", "ior": {"type": "constant", "texel": [1.5]}}
    with pytest.raises(AtrcError, match="empty color reflection/refraction map"):
        Config.from_string(base([q]))
    q["material"] = {"type": "no_such_thing"}
    with pytest.raises(AtrcError):
        Config.from_string(base([q]))
    with pytest.raises(AtrcError, match="missing field"):
        Config.from_string({"scene": {"type": "default"}})


def test_rendering_array_and_filters():
    c = base([QUAD])
    r0 = c["rendering"]
    r1 = dict(r0, film_filter={"type": "gaussian", "radius": 1.5, "alpha": 2}, eps=1e-3,
              camera={"type": "pinhole", "pos": [0, 0, 5], "dst": [0, 0, 0], "up": [0, 1, 0], "width": 2,
                      "dist": 1})
    c["rendering"] = [r0, r1]
    cfg = Config.from_string(c)
    assert cfg.rendering_count() == 2
    d1, _ = cfg.rendering(1)
    assert d1.filter_type == 1 and d1.filter_radius == pytest.approx(1.5) and d1.eps == pytest.approx(1e-3)
    # pinhole: fov = 2 atan(height / (2 dist)) with height = width / aspect
    assert d1.camera.fov == pytest.approx(2 * np.arctan((2 / 2.0) / 2), rel=1e-6)


def test_env_and_media(tmp_path):
    from atrc_b200.scenes import write_pfm, write_grid
    write_pfm(tmp_path / "e.pfm", np.ones((8, 16, 3), np.float32))
    write_grid(tmp_path / "g.bin", np.arange(8, dtype=np.float32).reshape(2, 2, 2))
    q = json.loads(json.dumps(QUAD))
    q["med_in"] = {"type": "heterogeneous", "transform": [],
                   "density": {"type": "image3d", "format": "real", "binary_filename": "${scene-directory}/g.bin"},
                   "albedo": {"type": "constant", "texel": [0.9]}, "g": {"type": "constant", "texel": [0.1]}}
    q["med_out"] = {"type": "homogeneous", "sigma_a": [0.1], "sigma_s": [0.2, 0.3, 0.4], "g": 0.5}
    c = base([q], env={"type": "ibl", "tex": {"type": "hdr", "filename": "${scene-directory}/e.pfm"}})
    cfg = Config.from_string(c, tmp_path)
    s = cfg.scene_desc().contents
    assert s.env.type == 1 and s.textures2d[s.env.tex].width == 16 and s.textures2d[s.env.tex].height == 8
    e = s.entities[0]
    assert s.media[e.medium_in].type == 2 and s.media[e.medium_out].type == 1
    t3 = s.textures3d[s.media[e.medium_in].density]
    assert (t3.width, t3.height, t3.depth, t3.channels) == (2, 2, 2, 1) and t3.max_real == 7
    assert list(s.media[e.medium_out].sigma_s) == pytest.approx([0.2, 0.3, 0.4])


def test_post_processors_round_trip():
    c = base([QUAD], {"post_processors": [{"type": "save_to_img", "filename": "out.png", "inv_gamma": 2.2}]})
    pp = Config.from_string(c).post_processors(0)
    assert pp[0]["type"] == "save_to_img" and float(pp[0]["inv_gamma"]) == pytest.approx(2.2)


def test_mirror_glass_metal_phong_and_checker_board():
    c = lambda *v: {"type": "constant", "texel": list(v)}  # noqa: E731
    mats = [("mirror", {"color_map": c(0.9), "eta": c(1.5), "k": c(2.0)}, 4, 3),
            ("glass", {"ior": c(1.45), "color_map": c(0.8)}, 5, 3),
            ("metal", {"color": c(0.9, 0.6, 0.3), "eta": c(0.2), "k": c(3.0), "roughness": c(0.3),
                       "anisotropic": c(0.0)}, 6, 5),
            ("phong", {"d": c(0.5), "s": c(0.4), "ns": c(30)}, 7, 3)]
    for name, params, code, slots in mats:
        q = json.loads(json.dumps(QUAD))
        q["material"] = {"type": name, **params}
        cfg = Config.from_string(base([q]))  # keep the config alive while reading its tables
        s = cfg.scene_desc().contents
        m = s.materials[0]
        assert m.type == code and all(m.tex[k] >= 0 for k in range(slots))
    # glass: one color_map serves reflection and refraction
    q = json.loads(json.dumps(QUAD))
    q["material"] = {"type": "glass", "ior": c(1.45), "color_map": c(0.8)}
    cfg = Config.from_string(base([q]))
    s = cfg.scene_desc().contents
    assert s.materials[0].tex[0] == s.materials[0].tex[1]
    # checker_board (texture2d_creators.cpp:29-48)
    q = json.loads(json.dumps(QUAD))
    q["material"] = {"type": "ideal_diffuse",
                     "albedo": {"type": "checker_board", "grid_count": 4, "color1": [1, 0, 0], "color2": [0, 0, 1]}}
    cfg = Config.from_string(base([q]))
    s = cfg.scene_desc().contents
    t = s.textures2d[s.materials[0].tex[0]]
    assert t.type == 2 and t.grid_count == 4 and list(t.texel) == [1, 0, 0] and list(t.texel2) == [0, 0, 1]
    q["material"]["albedo"]["grid_count"] = 0
    with pytest.raises(AtrcError, match="grid_count"):
        Config.from_string(base([q]))


def test_png_and_ppm_textures(tmp_path):
    # 8-bit images load as byte / 255, row 0 = top (PNG filters undone)
    import zlib
    import struct
    rng = np.random.default_rng(3)
    img = rng.integers(0, 256, (5, 7, 3), dtype=np.uint8)

    def chunk(kind, body):
        return struct.pack(">I", len(body)) + kind + body + struct.pack(">I", zlib.crc32(kind + body))
    rows = b""
    for y in range(5):  # rows with the Sub, Up, Paeth and None filters
        ft = y % 5
        r = img[y].astype(int).ravel()
        prev = img[y - 1].astype(int).ravel() if y else np.zeros_like(r)
        left = np.concatenate([[0, 0, 0], r[:-3]])
        upleft = np.concatenate([[0, 0, 0], prev[:-3]])
        if ft == 1:
            f = r - left
        elif ft == 2:
            f = r - prev
        elif ft == 3:
            f = r - (left + prev) // 2
        elif ft == 4:
            p = left + prev - upleft
            pa, pb, pc = abs(p - left), abs(p - prev), abs(p - upleft)
            pred = np.where((pa <= pb) & (pa <= pc), left, np.where(pb <= pc, prev, upleft))
            f = r - pred
        else:
            f = r
        rows += bytes([ft]) + bytes((f % 256).astype(np.uint8))
    png = b"\x89PNG\r\n\x1a\n" + chunk(b"IHDR", struct.pack(">IIBBBBB", 7, 5, 8, 2, 0, 0, 0)) + \
        chunk(b"IDAT", zlib.compress(rows)) + chunk(b"IEND", b"")
    (tmp_path / "t.png").write_bytes(png)
    (tmp_path / "t.ppm").write_bytes(b"P6\n7 5\n255\n" + img.tobytes())
    for fn in ("t.png", "t.ppm"):
        q = json.loads(json.dumps(QUAD))
        q["material"] = {"type": "ideal_diffuse", "albedo": {"type": "image", "filename": "${scene-directory}/" + fn}}
        cfg = Config.from_string(base([q]), tmp_path)
        s = cfg.scene_desc().contents
        t = s.textures2d[s.materials[0].tex[0]]
        assert (t.width, t.height) == (7, 5)
        got = np.ctypeslib.as_array(t.data, shape=(5 * 7 * 3,)).reshape(5, 7, 3)
        np.testing.assert_array_equal(got, img.astype(np.float32) / np.float32(255))


def test_ao_renderer_keys_and_bvh_builder():
    # AORendererCreator (renderer_creators.cpp:19-38) defaults and keys
    d, kind = Config.from_string(base([QUAD], {"renderer": {"type": "ao", "spp": 3}})).rendering(0)
    assert kind == "ao" and d.renderer == 1 and d.spp == 3
    assert (d.ao_sample_count, d.ao_max_distance) == (5, 1.0)
    assert list(d.ao_low) == [0, 0, 0] and list(d.ao_high) == [1, 1, 1] and list(d.ao_background) == [0, 0, 0]
    d, _ = Config.from_string(base([QUAD], {"renderer": {"type": "ao", "spp": 1, "ao_sample_count": 9,
                                                         "max_occlusion_distance": 2.5, "low_color": [0.25],
                                                         "high_color": [1, 0.5, 0.25]}})).rendering(0)
    assert d.ao_sample_count == 9 and d.ao_max_distance == pytest.approx(2.5)
    assert list(d.ao_low) == [0.25] * 3 and list(d.ao_high) == [1, 0.5, 0.25]
    with pytest.raises(AtrcError, match="ao_sample_count"):
        Config.from_string(base([QUAD], {"renderer": {"type": "ao", "spp": 1, "ao_sample_count": 0}}))
    with pytest.raises(AtrcError, match="not supported"):
        Config.from_string(base([QUAD], {"renderer": {"type": "bdpt", "spp": 1}}))
    # pt_cuda scene key: builder of the device scene's mesh trees
    assert Config.from_string(base([QUAD])).scene_desc().contents.bvh_builder == 0
    for name, v in (("sah", 0), ("ploc", 1), ("auto", 2)):
        assert Config.from_string(base([QUAD], bvh_builder=name)).scene_desc().contents.bvh_builder == v
    with pytest.raises(AtrcError, match="bvh_builder"):
        Config.from_string(base([QUAD], bvh_builder="lbvh"))


def _mesh_vertices(tmp_path, name):
    q = {"type": "geometric", "geometry": {"type": "triangle_bvh", "filename": "${scene-directory}/" + name,
                                           "transform": []},
         "material": {"type": "ideal_black"}}
    cfg = Config.from_string(base([q]), tmp_path)
    m = cfg.scene_desc().contents.meshes[0]
    return np.ctypeslib.as_array(m.vertices, shape=(int(m.triangle_count) * 24,)).reshape(-1, 3, 8).copy()


def test_obj_and_stl_meshes(tmp_path):
    # OBJ: positions / uvs / normals, negative indices, polygon fans
    (tmp_path / "m.obj").write_text("v 0 0 0\nv 1 0 0\nv 1 1 0\nv 0 1 0\nvt 0 0\nvt 1 0\nvt 1 1\nvt 0 1\n"
                                    "vn 0 0 1\nf 1/1/1 2/2/1 3/3/1 4/4/1\nf -4 -2 -1\n")
    v = _mesh_vertices(tmp_path, "m.obj")
    assert v.shape == (3, 3, 8)
    np.testing.assert_array_equal(v[1, :, :3], [[0, 0, 0], [1, 1, 0], [0, 1, 0]])
    np.testing.assert_array_equal(v[1, :, 6:], [[0, 0], [1, 1], [0, 1]])
    np.testing.assert_array_equal(v[2, :, 3:6], np.tile([0, 0, 1], (3, 1)))     # winding normal
    # binary STL (its header starts with "solid", as some exporters write)
    tris = np.array([[[0, 0, 0], [1, 0, 0], [0, 1, 0]], [[0, 0, 1], [0, 1, 1], [1, 0, 1]]], np.float32)
    body = b"".join(np.float32([0, 0, 0]).tobytes() + t.tobytes() + b"\0\0" for t in tris)
    (tmp_path / "b.stl").write_bytes(b"solid exported".ljust(80, b" ") + np.uint32(2).tobytes() + body)
    v = _mesh_vertices(tmp_path, "b.stl")
    np.testing.assert_array_equal(v[..., :3], tris)
    np.testing.assert_allclose(v[0, :, 3:6], np.tile([0, 0, 1], (3, 1)))
    np.testing.assert_allclose(v[1, :, 3:6], np.tile([0, 0, -1], (3, 1)))
    assert not v[..., 6:].any()
    # ASCII STL with its own facet normals
    (tmp_path / "a.stl").write_text("solid t\n facet normal 0 0 2\n  outer loop\n   vertex 0 0 0\n   vertex 2 0 0\n"
                                    "   vertex 0 2 0\n  endloop\n endfacet\nendsolid t\n")
    v = _mesh_vertices(tmp_path, "a.stl")
    np.testing.assert_array_equal(v[0, :, :3], [[0, 0, 0], [2, 0, 0], [0, 2, 0]])
    np.testing.assert_allclose(v[0, :, 3:6], np.tile([0, 0, 1], (3, 1)))
    (tmp_path / "bad.stl").write_text("solid t\n facet normal 0 0 1\n outer loop\n vertex 0 0 0\n endfacet\n")
    with pytest.raises(AtrcError, match="three vertices"):
        _mesh_vertices(tmp_path, "bad.stl")


def test_solid_image_texture():
    # SolidImageCreator (texture2d_creators.cpp:148-163): a 3D texture behind
    # the 2D interface, without the 2D common parameters
    q = json.loads(json.dumps(QUAD))
    q["material"]["albedo"] = {"type": "solid_image", "transform": [{"type": "scale", "ratio": 3}],
                               "tex3d": {"type": "constant", "texel": [0.2, 0.4, 0.6]}}
    cfg = Config.from_string(base([q]))
    s = cfg.scene_desc().contents
    t = [s.textures2d[i] for i in range(s.texture2d_count) if s.textures2d[i].type == 3]
    assert len(t) == 1 and 0 <= t[0].tex3d < s.texture3d_count
    assert list(t[0].uv_transform) == [1, 0, 0, 0, 1, 0] and t[0].wrap_u == 0 and t[0].inv_gamma == 1
    assert list(s.textures3d[t[0].tex3d].texel) == pytest.approx([0.2, 0.4, 0.6])


def _rgbe_decode(px):
    m, e = px[..., :3].astype(np.float64), px[..., 3].astype(np.int64)
    return np.where(e[..., None] > 0, m * np.ldexp(1.0, e - 136)[..., None], 0.0).astype(np.float32)


def _rgbe_rle_scanline(row):
    """New-style RLE scanline: per channel a run of the first five values
    (all equal) then the rest as one literal."""
    w = len(row)
    out = bytes([2, 2, w >> 8, w & 255])
    for c in range(4):
        ch = row[:, c]
        out += bytes([128 + 5, ch[0]]) + bytes([w - 5]) + bytes(ch[5:])
    return out


def test_radiance_hdr_flat_and_rle(tmp_path):
    # .hdr textures: RGBE texels decode to m * 2^(e - 136), e = 0 is black;
    # "-Y h +X w" puts the first scanline on top
    rng = np.random.default_rng(11)
    h, w = 3, 12
    px = rng.integers(0, 256, (h, w, 4), dtype=np.uint8)
    px[:, :5] = px[:, :1]            # the run the encoder below writes
    px[0, 7, 3] = 0                  # one black texel
    head = b"#?RADIANCE\nFORMAT=32-bit_rle_rgbe\n\n-Y %d +X %d\n"
    (tmp_path / "rle.hdr").write_bytes(head % (h, w) + b"".join(_rgbe_rle_scanline(px[y]) for y in range(h)))
    flat = rng.integers(0, 256, (2, 4, 4), dtype=np.uint8)
    (tmp_path / "flat.hdr").write_bytes(head % (2, 4) + flat.tobytes())
    for fn, want in (("rle.hdr", _rgbe_decode(px)), ("flat.hdr", _rgbe_decode(flat))):
        c = base([QUAD], env={"type": "ibl", "tex": {"type": "hdr", "filename": "${scene-directory}/" + fn}})
        cfg = Config.from_string(c, tmp_path)  # owns the texel arrays
        s = cfg.scene_desc().contents
        t = s.textures2d[s.env.tex]
        assert (t.height, t.width) == want.shape[:2]
        got = np.ctypeslib.as_array(t.data, shape=(want.size,)).reshape(want.shape)
        np.testing.assert_array_equal(got, want)
    # malformed files are configuration errors, not garbage texels
    good = (tmp_path / "rle.hdr").read_bytes()
    bad = {"trunc.hdr": (good[:-3], "truncated HDR"),
           "run.hdr": (good.replace(bytes([128 + 5]), bytes([128 + 40]), 1), "bad HDR run length"),
           "size.hdr": (head % (0, 4), "bad HDR size")}
    for fn, (data, msg) in bad.items():
        (tmp_path / fn).write_bytes(data)
        c = base([QUAD], env={"type": "ibl", "tex": {"type": "hdr", "filename": "${scene-directory}/" + fn}})
        with pytest.raises(AtrcError, match=msg):
            Config.from_string(c, tmp_path).scene_desc()


def test_scene_description_keeps_its_config_alive(tmp_path):
    # the description points into the config's memory: holding only the
    # description (or its contents) must keep the config alive
    import gc
    from atrc_b200.scenes import write_pfm
    img = np.arange(8 * 16 * 3, dtype=np.float32).reshape(8, 16, 3)
    write_pfm(tmp_path / "e.pfm", img)
    c = base([QUAD], env={"type": "ibl", "tex": {"type": "hdr", "filename": "${scene-directory}/e.pfm"}})
    s = Config.from_string(c, tmp_path).scene_desc().contents
    gc.collect()
    t = s.textures2d[s.env.tex]
    got = np.ctypeslib.as_array(t.data, shape=(img.size,)).reshape(img.shape)
    np.testing.assert_array_equal(got, img)  # row 0 on top, as written
