"""ctypes mirror of ``include/atrc_cuda.h`` (struct layouts and prototypes).

Layouts are checked at load time against ``atrc_abi_struct_sizes``.
"""
from __future__ import annotations

import ctypes as C

c_float_p = C.POINTER(C.c_float)
c_double_p = C.POINTER(C.c_double)


class AtrcTransform(C.Structure):
    _fields_ = [("m", C.c_float * 12), ("inv", C.c_float * 12)]


class AtrcMeshDesc(C.Structure):
    _fields_ = [("triangle_count", C.c_uint64), ("vertices", c_float_p)]


class AtrcGeometryDesc(C.Structure):
    _fields_ = [("type", C.c_int32), ("mesh", C.c_int32), ("transform", AtrcTransform),
                ("p", (C.c_float * 3) * 4), ("uv", (C.c_float * 2) * 4), ("radius", C.c_float),
                ("pad_", C.c_int32)]


class AtrcEntityDesc(C.Structure):
    _fields_ = [("geometry", C.c_int32), ("has_instance", C.c_int32), ("instance", AtrcTransform),
                ("double_sided", C.c_int32), ("material", C.c_int32), ("medium_in", C.c_int32),
                ("medium_out", C.c_int32), ("emit_radiance", C.c_float * 3), ("no_denoise", C.c_int32),
                ("power", C.c_float), ("pad_", C.c_int32)]


class AtrcTexture2DDesc(C.Structure):
    _fields_ = [("type", C.c_int32), ("texel", C.c_float * 3), ("width", C.c_int32), ("height", C.c_int32),
                ("data", c_float_p), ("nearest", C.c_int32), ("uv_transform", C.c_float * 6),
                ("wrap_u", C.c_int32), ("wrap_v", C.c_int32), ("inv_gamma", C.c_float), ("grid_count", C.c_int32),
                ("texel2", C.c_float * 3), ("tex3d", C.c_int32)]


class AtrcTexture3DDesc(C.Structure):
    _fields_ = [("type", C.c_int32), ("texel", C.c_float * 3), ("width", C.c_int32), ("height", C.c_int32),
                ("depth", C.c_int32), ("channels", C.c_int32), ("data", c_float_p), ("nearest", C.c_int32),
                ("uvw_transform", C.c_float * 12), ("uvw_perm", C.c_int32 * 3), ("wrap", C.c_int32 * 3),
                ("inv_gamma", C.c_float), ("max_real", C.c_float)]


class AtrcMaterialDesc(C.Structure):
    _fields_ = [("type", C.c_int32), ("tex", C.c_int32 * 13), ("normal_map", C.c_int32), ("bssrdf", C.c_int32 * 3)]


class AtrcMediumDesc(C.Structure):
    _fields_ = [("type", C.c_int32), ("sigma_a", C.c_float * 3), ("sigma_s", C.c_float * 3), ("g", C.c_float),
                ("max_scattering_count", C.c_int32), ("transform", AtrcTransform), ("density", C.c_int32),
                ("albedo", C.c_int32), ("g_tex", C.c_int32), ("white_for_indirect", C.c_int32)]


class AtrcEnvDesc(C.Structure):
    _fields_ = [("type", C.c_int32), ("tex", C.c_int32), ("no_importance_sampling", C.c_int32),
                ("power", C.c_float), ("top", C.c_float * 3), ("bottom", C.c_float * 3)]


class AtrcSceneDesc(C.Structure):
    _fields_ = [("abi_version", C.c_uint32), ("aggregate", C.c_int32), ("aggregate_max_leaf_size", C.c_int32),
                ("bvh_builder", C.c_int32),
                ("meshes", C.POINTER(AtrcMeshDesc)), ("mesh_count", C.c_uint32),
                ("geometries", C.POINTER(AtrcGeometryDesc)), ("geometry_count", C.c_uint32),
                ("entities", C.POINTER(AtrcEntityDesc)), ("entity_count", C.c_uint32),
                ("materials", C.POINTER(AtrcMaterialDesc)), ("material_count", C.c_uint32),
                ("textures2d", C.POINTER(AtrcTexture2DDesc)), ("texture2d_count", C.c_uint32),
                ("textures3d", C.POINTER(AtrcTexture3DDesc)), ("texture3d_count", C.c_uint32),
                ("media", C.POINTER(AtrcMediumDesc)), ("medium_count", C.c_uint32),
                ("env", AtrcEnvDesc)]


class AtrcCameraDesc(C.Structure):
    _fields_ = [("pos", C.c_float * 3), ("dst", C.c_float * 3), ("up", C.c_float * 3), ("fov", C.c_float),
                ("lens_radius", C.c_float), ("focal_distance", C.c_float)]


class AtrcRenderDesc(C.Structure):
    _fields_ = [("width", C.c_int32), ("height", C.c_int32), ("spp", C.c_int32), ("min_depth", C.c_int32),
                ("max_depth", C.c_int32), ("cont_prob", C.c_float), ("specular_depth", C.c_int32),
                ("use_mis", C.c_int32), ("filter_type", C.c_int32), ("filter_radius", C.c_float),
                ("filter_alpha", C.c_float), ("eps", C.c_float), ("seed", C.c_uint64), ("first_spp", C.c_int32),
                ("spp_count", C.c_int32), ("camera", AtrcCameraDesc), ("path_pool", C.c_int32),
                ("count_traversal", C.c_int32), ("task_grid_size", C.c_int32), ("sort_mode", C.c_int32),
                ("disney_fixed", C.c_int32), ("renderer", C.c_int32),
                ("ao_sample_count", C.c_int32), ("ao_max_distance", C.c_float), ("ao_low", C.c_float * 3),
                ("ao_high", C.c_float * 3), ("ao_background", C.c_float * 3), ("isect_mode", C.c_int32)]


class AtrcFilm(C.Structure):
    _fields_ = [("value", c_double_p), ("weight", c_double_p), ("value_sq", c_double_p), ("albedo", c_double_p),
                ("normal", c_double_p), ("denoise", c_double_p), ("on_device", C.c_int32), ("pad_", C.c_int32)]


class AtrcRenderStats(C.Structure):
    _fields_ = [("seconds", C.c_double), ("kernel_seconds", C.c_double), ("samples", C.c_uint64),
                ("rays_closest", C.c_uint64), ("rays_shadow", C.c_uint64), ("iterations", C.c_uint64),
                ("kernel_launches", C.c_uint64), ("watchdog_flags", C.c_uint64), ("extend_seconds", C.c_double),
                ("shadow_seconds", C.c_double), ("shade_seconds", C.c_double), ("h2d_bytes", C.c_uint64),
                ("d2h_bytes", C.c_uint64), ("extend_launches", C.c_uint64), ("shadow_launches", C.c_uint64),
                ("nodes_closest", C.c_uint64), ("tris_closest", C.c_uint64), ("ents_closest", C.c_uint64),
                ("nodes_shadow", C.c_uint64), ("tris_shadow", C.c_uint64), ("ents_shadow", C.c_uint64)]


class AtrcRay(C.Structure):
    _fields_ = [("o", C.c_float * 3), ("t_min", C.c_float), ("d", C.c_float * 3), ("t_max", C.c_float)]


class AtrcHit(C.Structure):
    _fields_ = [("t", C.c_float), ("entity", C.c_int32), ("prim", C.c_int32), ("u", C.c_float)]


class AtrcDeviceInfo(C.Structure):
    _fields_ = [("name", C.c_char * 128), ("sm_count", C.c_int32), ("cc_major", C.c_int32),
                ("cc_minor", C.c_int32), ("pad_", C.c_int32), ("global_mem_bytes", C.c_uint64)]


class AtrcTuning(C.Structure):
    _fields_ = [("path_pool", C.c_int32), ("sort_mode", C.c_int32), ("gen_blocks_per_sm", C.c_int32),
                ("gen_threads", C.c_int32), ("finish_threads", C.c_int32), ("trials", C.c_int32),
                ("ms_per_msample", C.c_double), ("default_ms_per_msample", C.c_double), ("extend_fetch", C.c_int32),
                ("queue_order", C.c_int32), ("shadow_fetch", C.c_int32), ("shadow_sort", C.c_int32)]


class AtrcGuideDesc(C.Structure):
    _fields_ = [("log2_table", C.c_int32), ("base_resolution", C.c_int32), ("max_resolution", C.c_int32),
                ("batch", C.c_int32), ("record_capacity", C.c_int32), ("learning_rate", C.c_float),
                ("max_depth", C.c_int32), ("max_select", C.c_float), ("seed", C.c_uint64),
                ("target_clamp", C.c_float), ("pad_", C.c_int32)]


class AtrcGuideInfo(C.Structure):
    _fields_ = [("weights", C.c_uint64), ("table_floats", C.c_uint64), ("levels", C.c_int32), ("inputs", C.c_int32),
                ("hidden", C.c_int32), ("outputs", C.c_int32), ("lobes", C.c_int32), ("steps", C.c_int32),
                ("log2_table", C.c_int32), ("pad_", C.c_int32), ("grid_lo", C.c_float * 3),
                ("grid_inv_extent", C.c_float * 3), ("grid_res", C.c_int32 * 16),
                ("max_select", C.c_float), ("pad2_", C.c_float)]


class AtrcBvhBuildInfo(C.Structure):
    _fields_ = [("seconds", C.c_double), ("sah_cost", C.c_double), ("nodes", C.c_uint64), ("rounds", C.c_int32),
                ("max_depth", C.c_int32)]


STRUCT_ORDER = [AtrcSceneDesc, AtrcMeshDesc, AtrcGeometryDesc, AtrcEntityDesc, AtrcTexture2DDesc,
                AtrcTexture3DDesc, AtrcMaterialDesc, AtrcMediumDesc, AtrcEnvDesc, AtrcRenderDesc, AtrcFilm,
                AtrcRenderStats, AtrcRay, AtrcHit, AtrcDeviceInfo, AtrcTuning, AtrcBvhBuildInfo]

PROGRESS_FN = C.CFUNCTYPE(None, C.c_double, C.c_void_p)
CANCEL_FN = C.CFUNCTYPE(C.c_int, C.c_void_p)

# name -> (restype, argtypes)
PROTOTYPES = {
    "atrc_abi_version": (C.c_int, []),
    "atrc_abi_struct_sizes": (C.c_int, [C.POINTER(C.c_uint64), C.c_int]),
    "atrc_last_error": (C.c_char_p, []),
    "atrc_config_load_file": (C.c_int, [C.c_char_p, C.POINTER(C.c_void_p)]),
    "atrc_config_load_string": (C.c_int, [C.c_char_p, C.c_char_p, C.POINTER(C.c_void_p)]),
    "atrc_config_destroy": (None, [C.c_void_p]),
    "atrc_config_scene": (C.c_int, [C.c_void_p, C.POINTER(C.POINTER(AtrcSceneDesc))]),
    "atrc_config_rendering_count": (C.c_int, [C.c_void_p, C.POINTER(C.c_int)]),
    "atrc_config_rendering": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(AtrcRenderDesc), C.c_char_p, C.c_size_t]),
    "atrc_config_post_processors": (C.c_int, [C.c_void_p, C.c_int, C.c_char_p, C.c_size_t,
                                              C.POINTER(C.c_size_t)]),
    "atrc_cuda_device_init": (C.c_int, [C.c_int, C.POINTER(AtrcDeviceInfo)]),
    "atrc_cuda_scene_create": (C.c_int, [C.POINTER(AtrcSceneDesc), C.POINTER(C.c_void_p)]),
    "atrc_cuda_scene_destroy": (None, [C.c_void_p]),
    "atrc_cuda_trace_rays": (C.c_int, [C.c_void_p, C.POINTER(AtrcRay), C.c_size_t, C.POINTER(AtrcHit), C.c_int,
                                       C.c_int]),
    "atrc_cuda_trace_rays_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p, C.c_int, C.c_int]),
    "atrc_cuda_render": (C.c_int, [C.c_void_p, C.POINTER(AtrcRenderDesc), C.POINTER(AtrcFilm),
                                   CANCEL_FN, PROGRESS_FN, C.c_void_p, C.POINTER(AtrcRenderStats)]),
    "atrc_cuda_stream_read_gbs": (C.c_int, [C.c_int, C.c_uint64, C.c_int, C.POINTER(C.c_double)]),
    "atrc_cuda_render_noalloc": (C.c_int, [C.c_void_p, C.POINTER(AtrcRenderDesc), C.POINTER(AtrcFilm),
                                           C.POINTER(AtrcRenderStats)]),
    "atrc_film_resolve": (C.c_int, [C.POINTER(AtrcFilm), C.c_int, C.c_int, c_float_p]),
    "atrc_save_png_bytes": (C.c_int, [C.c_char_p, C.c_void_p, C.c_int, C.c_int]),
    "atrc_cuda_film_resolve": (C.c_int, [C.POINTER(AtrcFilm), C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]),
    "atrc_cuda_post_apply": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int32, C.c_float]),
    "atrc_cuda_encode_ldr": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_float, C.c_void_p]),
    "atrc_cuda_post_process": (C.c_int, [C.POINTER(AtrcFilm), C.c_int, C.c_int, C.c_char_p, C.c_char_p, C.c_char_p,
                                         C.c_size_t]),
    "atrc_cuda_autotune": (C.c_int, [C.c_void_p, C.POINTER(AtrcRenderDesc), C.c_int32, C.POINTER(AtrcTuning)]),
    "atrc_cuda_get_tuning": (C.c_int, [C.c_void_p, C.POINTER(AtrcTuning)]),
    "atrc_guide_default_desc": (C.c_int, [C.POINTER(AtrcGuideDesc)]),
    "atrc_guide_create": (C.c_int, [C.c_int, c_float_p, c_float_p, C.POINTER(AtrcGuideDesc), C.POINTER(C.c_void_p)]),
    "atrc_guide_destroy": (None, [C.c_void_p]),
    "atrc_guide_info": (C.c_int, [C.c_void_p, C.POINTER(AtrcGuideInfo)]),
    "atrc_guide_set_max_select": (C.c_int, [C.c_void_p, C.c_float]),
    "atrc_guide_params": (C.c_int, [C.c_void_p, c_float_p, c_float_p, C.c_int]),
    "atrc_guide_eval": (C.c_int, [C.c_void_p, c_float_p, C.c_size_t, c_float_p]),
    "atrc_guide_train": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_float)]),
    "atrc_guide_pdf": (C.c_int, [C.c_void_p, c_float_p, c_float_p, C.c_size_t, c_float_p, c_float_p]),
    "atrc_guide_train_records": (C.c_int, [C.c_void_p, c_float_p, C.c_size_t, C.c_int, C.POINTER(C.c_float)]),
    "atrc_guide_gradients": (C.c_int, [C.c_void_p, c_float_p, C.c_size_t, c_float_p, c_float_p, c_float_p]),
    "atrc_guide_records": (C.c_int, [C.c_void_p, c_float_p, C.c_size_t, C.POINTER(C.c_size_t)]),
    "atrc_cuda_scene_bounds": (C.c_int, [C.c_void_p, c_float_p, c_float_p]),
    "atrc_cuda_subsurface_probe": (C.c_int, [C.c_void_p, c_float_p, c_float_p, C.c_int32, C.c_uint64, c_float_p,
                                             c_float_p]),
    "atrc_bvh_build": (C.c_int, [C.c_int32, C.c_int32, c_float_p, C.c_uint64, C.POINTER(AtrcBvhBuildInfo)]),
    "atrc_bvh_cluster_tree": (C.c_int, [C.c_int32, c_float_p, C.c_uint64, C.POINTER(C.c_uint32),
                                        C.POINTER(C.c_int32), C.POINTER(C.c_int32), c_float_p,
                                        C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    "atrc_cuda_render_batch": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(AtrcRenderDesc), C.c_int32,
                                         C.POINTER(AtrcFilm), C.POINTER(C.c_double), C.POINTER(AtrcRenderStats)]),
    "atrc_cuda_render_guided": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(AtrcRenderDesc), C.c_int32,
                                          C.POINTER(AtrcFilm), C.POINTER(AtrcRenderStats)]),
    "atrc_cuda_set_tuning": (C.c_int, [C.c_void_p, C.POINTER(AtrcTuning)]),
}
