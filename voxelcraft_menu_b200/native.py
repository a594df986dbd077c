"""ctypes binding of libvoxmarch.so (include/voxmarch.h, include/voxmarch_world.h).

The library is built in-tree by voxelcraft_menu_b200/build.py.  Loading fails
loudly when it is missing: there is no CPU fallback for any march entry point.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "libvoxmarch.so"

c_f3 = C.c_float * 3
c_u3 = C.c_uint32 * 3
c_i3 = C.c_int32 * 3


class VmFrame(C.Structure):
    """GpuFrame (src/render/mod.rs:399-459), 352 bytes."""
    _fields_ = [
        ("cam_pos", c_f3), ("time", C.c_float), ("cam_fwd", c_f3), ("tan_half_fov", C.c_float),
        ("cam_right", c_f3), ("aspect", C.c_float), ("cam_up", c_f3), ("far", C.c_float),
        ("sun_dir", c_f3), ("daylight", C.c_float), ("res", C.c_uint32 * 2), ("tiles", C.c_uint32 * 2),
        ("chunk_count", C.c_uint32), ("camera_chunk", C.c_uint32), ("flags", C.c_uint32), ("max_pairs", C.c_uint32),
        ("fog_density", C.c_float), ("fog_falloff", C.c_float), ("shadow_dist", C.c_float), ("ambient", C.c_float),
        ("fog_scatter", C.c_float), ("fog_g", C.c_float), ("fog_height", C.c_float), ("mip_bias", C.c_float),
        ("grid_min", c_i3), ("sea_level", C.c_float), ("grid_dim", c_u3), ("water_absorb", C.c_float),
        ("jitter", C.c_float * 2), ("taa_feedback", C.c_float), ("frame_index", C.c_uint32),
        ("cloud_cover", C.c_float), ("cloud_height", C.c_float), ("cloud_scale", C.c_float), ("cloud_speed", C.c_float),
        ("godray_strength", C.c_float), ("godray_steps", C.c_uint32), ("godray_dist", C.c_float),
        ("cloud_shadow", C.c_float), ("tint_strength", C.c_float), ("tint_seed", C.c_int32),
        ("tint_freq_t", C.c_float), ("tint_freq_h", C.c_float), ("wave_amp", C.c_float), ("wave_scale", C.c_float),
        ("wave_speed", C.c_float), ("wave_reflect_slope", C.c_float), ("shaft_origin", C.c_float * 2),
        ("shaft_texel", C.c_float), ("shaft_soft", C.c_float), ("cloud_patch", C.c_float), ("cloud_relief", C.c_float),
        ("haze_warm", C.c_float), ("zenith_deep", C.c_float), ("prev_view_proj", C.c_float * 16),
    ]


class VmChunk(C.Structure):
    """GpuChunk (src/render/mod.rs:469-488), 96 bytes."""
    _fields_ = [
        ("aabb_min", c_f3), ("voxel_size", C.c_float), ("aabb_max", c_f3), ("lod", C.c_uint32),
        ("origin", c_f3), ("fade", C.c_float), ("root", C.c_uint32 * 4), ("attr_base", C.c_uint32),
        ("attr_flags", C.c_uint32), ("light_base", C.c_uint32), ("light_flags", C.c_uint32),
        ("dry_mask", C.c_uint32 * 2), ("reserved", C.c_uint32 * 2),
    ]


assert C.sizeof(VmFrame) == 352 and VmFrame.prev_view_proj.offset == 288
assert C.sizeof(VmChunk) == 96

# numpy view of a chunk list
CHUNK_DTYPE = np.dtype({
    "names": ["aabb_min", "voxel_size", "aabb_max", "lod", "origin", "fade", "root", "attr_base", "attr_flags",
              "light_base", "light_flags", "dry_mask", "reserved"],
    "formats": [("<f4", 3), "<f4", ("<f4", 3), "<u4", ("<f4", 3), "<f4", ("<u4", 4), "<u4", "<u4", "<u4", "<u4",
                ("<u4", 2), ("<u4", 2)],
    "offsets": [0, 12, 16, 28, 32, 44, 48, 64, 68, 72, 76, 80, 88],
    "itemsize": 96,
})


class VmwRecipe(C.Structure):
    _fields_ = [
        ("size", c_u3), ("octaves", C.c_uint32), ("seed", C.c_uint32), ("base", C.c_float),
        ("amplitude", C.c_float), ("base_freq", C.c_float), ("water_level", C.c_int32), ("water_depth", C.c_int32),
        ("tree_permille", C.c_uint32), ("glass_permille", C.c_uint32), ("island_permille", C.c_uint32),
        ("tuft_permille", C.c_uint32),
    ]


class VmwCamera(C.Structure):
    _fields_ = [
        ("pos", c_f3), ("yaw", C.c_float), ("pitch", C.c_float), ("use_basis", C.c_uint32), ("fwd", c_f3),
        ("right", c_f3), ("up", c_f3), ("fov_y", C.c_float), ("width", C.c_uint32), ("height", C.c_uint32),
        ("far", C.c_float), ("sun_dir", c_f3), ("daylight", C.c_float), ("flags", C.c_uint32),
        ("jitter", C.c_float * 2), ("frame_index", C.c_uint32), ("sea_level", C.c_float),
        ("offscreen_shadows", C.c_uint32), ("grid_dim", c_u3), ("grid_min_set", C.c_uint32), ("grid_min", c_i3),
        ("max_chunks", C.c_uint32),
    ]


class VmwChunkInfo(C.Structure):
    _fields_ = [
        ("root", C.c_uint32 * 4), ("attr_uniform", C.c_uint32), ("attr_value", C.c_uint32), ("aabb_min", c_i3),
        ("aabb_max", c_i3), ("solid_count", C.c_uint32), ("leaf_count", C.c_uint32), ("dry_mask", C.c_uint64),
        ("has_water", C.c_uint32), ("has_foliage", C.c_uint32), ("has_cutout", C.c_uint32),
        ("has_glass", C.c_uint32), ("has_emitter", C.c_uint32),
    ]


class VmwPoolStats(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in ("n_inners", "n_leaves", "n_bricks", "live_inners", "live_leaves",
                                          "referenced_inners", "referenced_leaves", "used_words", "n_chunks")]


class VmCaps(C.Structure):
    _fields_ = [("max_width", C.c_uint32), ("max_height", C.c_uint32), ("max_chunks", C.c_uint32),
                ("max_views", C.c_uint32), ("max_batch_pixels", C.c_uint64)]


class VmStats(C.Structure):
    _fields_ = [("counters", C.c_uint32 * 8), ("pairs_selected", C.c_uint32), ("pairs_deferred", C.c_uint32),
                ("pairs_recovered", C.c_uint32), ("max_pairs", C.c_uint32), ("truncated", C.c_uint32),
                ("device_error", C.c_uint32)]


class VmTraffic(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in ("chunk_records", "l1_fetches", "leaf_fetches", "attr_fetches",
                                          "palette_decodes", "grid_lookups", "iters", "rays_primary",
                                          "rays_shadow", "rays_secondary", "list_entries")] + \
               [("stage_iters", C.c_uint64 * 3), ("stage_chunks", C.c_uint64 * 3), ("stage_bytes", C.c_uint64 * 3)]


class VmDevicePtrs(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in ("vis", "shadow", "sec_key", "sec_t", "hiz", "batch_vis", "batch_shadow",
                                          "stream")]


P = C.POINTER
vp = C.c_void_p

# (name, restype, argtypes) for every exported entry point
_SIGNATURES = [
    # drop-in march ABI (include/voxmarch.h)
    ("vm_create", C.c_int, [C.c_int, P(VmCaps), P(vp)]),
    ("vm_destroy", None, [vp]),
    ("vm_last_error", C.c_char_p, [vp]),
    ("vm_set_stream", C.c_int, [vp, vp]),
    ("vm_upload_world", C.c_int, [vp, vp, C.c_uint64, vp, C.c_uint64, vp, C.c_uint64]),
    ("vm_update_pool", C.c_int, [vp, C.c_int, C.c_uint64, vp, C.c_uint64]),
    ("vm_upload_chunks", C.c_int, [vp, vp, C.c_uint32, vp, C.c_uint64]),
    ("vm_set_frame", C.c_int, [vp, P(VmFrame)]),
    ("vm_select", C.c_int, [vp]),
    ("vm_march", C.c_int, [vp]),
    ("vm_primary_shadow", C.c_int, [vp]),
    ("vm_secondary", C.c_int, [vp]),
    ("vm_soften_shadows", C.c_int, [vp, C.c_uint32, C.c_float]),
    ("vm_render", C.c_int, [vp]),
    ("vm_set_tuning", C.c_int, [vp, C.c_int, C.c_int, C.c_int]),
    ("vm_set_packet", C.c_int, [vp, C.c_int]),
    ("vm_set_spec", C.c_int, [vp, C.c_uint32]),
    ("vm_water_sec", C.c_int, [vp, C.c_uint32]),
    ("vm_read_water_sec", C.c_int, [vp, vp, vp, vp, vp]),
    ("vm_upload_atlas", C.c_int, [vp, vp, C.c_uint32, C.c_uint32, C.c_uint32]),
    ("vm_upload_block_faces", C.c_int, [vp, vp, C.c_uint32]),
    ("vm_upload_probes", C.c_int, [vp, vp, C.c_uint32, C.c_uint32, C.c_uint32]),
    ("vm_upload_shaft", C.c_int, [vp, vp, C.c_uint32]),
    ("vm_resolve", C.c_int, [vp, C.c_uint32]),
    ("vm_read_color", C.c_int, [vp, vp]),
    ("vm_read_vis", C.c_int, [vp, vp]),
    ("vm_read_hiz", C.c_int, [vp, vp]),
    ("vm_write_hiz", C.c_int, [vp, vp]),
    ("vm_read_shadow", C.c_int, [vp, vp]),
    ("vm_read_secondary", C.c_int, [vp, vp, vp]),
    ("vm_read_heatmap", C.c_int, [vp, vp]),
    ("vm_read_shadow_mask", C.c_int, [vp, vp]),
    ("vm_read_reflection", C.c_int, [vp, vp, vp]),
    ("vm_read_expanded", C.c_int, [vp, vp, vp, vp, vp, vp]),
    ("vm_stats_read", C.c_int, [vp, P(VmStats)]),
    ("vm_render_counted", C.c_int, [vp, P(VmTraffic)]),
    ("vm_render_events", C.c_int, [vp, P(vp)]),
    ("vm_read_async", C.c_int, [vp, vp, vp]),
    ("vm_read_async_r16f", C.c_int, [vp, vp, vp]),
    ("vm_wait_render", C.c_int, [vp, vp]),
    ("vm_batch_set", C.c_int, [vp, C.c_uint32, vp, vp, vp, vp, vp]),
    ("vm_batch_run", C.c_int, [vp, C.c_int]),
    ("vm_batch_read", C.c_int, [vp, vp, vp]),
    ("vm_batch_pixels", C.c_uint64, [vp]),
    ("vm_batch_read_secondary", C.c_int, [vp, vp, vp]),
    ("vm_batch_counted", C.c_int, [vp, C.c_int, P(VmTraffic)]),
    ("vm_shade_gbuffer", C.c_int, [vp, vp, vp]),
    ("vm_shade_forward", C.c_int, [vp, C.c_uint64, vp, vp, vp, vp, vp, vp]),
    ("vm_shade_backward", C.c_int, [vp, C.c_uint64, vp, vp, vp, vp, vp, vp, vp]),
    ("vm_device_buffers", C.c_int, [vp, P(VmDevicePtrs)]),
    ("vm_sync", C.c_int, [vp]),
    ("vm_render_static", C.c_int, [P(VmFrame), vp, C.c_uint32, vp, C.c_uint64, vp, C.c_uint64, vp, C.c_uint64,
                                   vp, C.c_uint64, vp, vp, vp, vp]),
    ("vm_static_last_error", C.c_char_p, []),
    # host world store (include/voxmarch_world.h)
    ("vmw_create", vp, []),
    ("vmw_destroy", None, [vp]),
    ("vmw_insert_dense", C.c_int, [vp, C.c_uint8, C.c_int32, C.c_int32, C.c_int32, vp]),
    ("vmw_build_tree", C.c_int, [vp, C.c_uint32, vp, vp, vp, vp, vp]),
    ("vmw_insert_tree", C.c_int, [vp, C.c_uint8, C.c_int32, C.c_int32, C.c_int32, vp, vp, vp, vp, vp]),
    ("vm_encode_trees", C.c_int, [vp, C.c_uint32, C.c_uint32, vp, vp, vp, vp, vp, vp]),
    ("vmw_remove", C.c_int, [vp, C.c_uint8, C.c_int32, C.c_int32, C.c_int32]),
    ("vmw_get_block", C.c_uint32, [vp, C.c_int32, C.c_int32, C.c_int32]),
    ("vmw_get_chunk_info", C.c_int, [vp, C.c_uint8, C.c_int32, C.c_int32, C.c_int32, P(VmwChunkInfo)]),
    ("vmw_set_fade", C.c_int, [vp, C.c_uint8, C.c_int32, C.c_int32, C.c_int32, C.c_float]),
    ("vmw_pool_stats", None, [vp, P(VmwPoolStats)]),
    ("vmw_inners", vp, [vp]),
    ("vmw_leaves", vp, [vp]),
    ("vmw_bricks", vp, [vp]),
    ("vmw_generate", C.c_int, [vp, P(VmwRecipe)]),
    ("vmw_recipe_dense", C.c_int, [P(VmwRecipe), C.c_int32, C.c_int32, C.c_int32, vp]),
    ("vmw_recipe_dense_all", C.c_int, [P(VmwRecipe), vp]),
    ("vmw_recipe_dense_lod", C.c_int, [P(VmwRecipe), C.c_uint32, C.c_int32, C.c_int32, C.c_int32, vp]),
    ("vmw_recipe_height", C.c_int32, [P(VmwRecipe), C.c_int32, C.c_int32]),
    ("vmw_camera_basis", None, [C.c_float, C.c_float, vp, vp, vp]),
    ("vmw_pairs_for", C.c_uint32, [C.c_uint32, C.c_uint32]),
    ("vmw_build_view", C.c_int, [vp, P(VmwCamera), P(VmFrame), vp, C.c_uint32, P(C.c_uint32), vp]),
    ("vmw_halton_jitter", None, [C.c_uint64, vp]),
    ("vmw_atlas_bytes", C.c_uint64, [C.c_uint32]),
    ("vmw_build_atlas", C.c_int, [C.c_uint32, vp]),
    ("vmw_block_faces", C.c_int, [vp, C.c_uint32]),
    ("vmw_probe_field", C.c_int, [C.c_uint32, vp]),
    ("vmw_shaft_envelope", C.c_int, [vp, vp, vp, C.c_float, vp]),
    ("vmw_look_defaults", None, [vp, C.c_int32]),
]

EXPORTED = [s[0] for s in _SIGNATURES]

_lib = None


def lib() -> C.CDLL:
    """The loaded libvoxmarch.so; raises if it was not built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing: run `python -m voxelcraft_menu_b200.build` "
                               "(there is no CPU fallback for the march)")
        L = C.CDLL(str(LIB_PATH))
        for name, res, args in _SIGNATURES:
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def ptr(a: np.ndarray) -> C.c_void_p:
    assert a.flags["C_CONTIGUOUS"]
    return C.c_void_p(a.ctypes.data)
