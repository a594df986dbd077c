"""Material inputs of the resolve (vm_upload_atlas, vm_upload_block_faces,
vm_upload_probes, vm_upload_shaft) for callers without the engine's own, and
the engine's default look of a frame.

The engine passes its own atlas (src/render/mod.rs:2159-2222), face table
(src/block.rs:265-276), probe field (src/render/mod.rs:2248-2300) and shaft
pass output; these builders stand in for them in the tests, the benchmarks
and the smoke check (include/voxmarch_world.h).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from .native import lib, ptr

TEX_COUNT = 27
ATLAS_SIZE, ATLAS_MIPS = 16, 4
PROBE_SHAPE = (128, 768, 128)        # x, 6 slabs of 128 in y, z
SHAFT_DIM = 512

# frame flags the resolve reads (src/render/mod.rs:140-262)
FLAG_AO = 8
FLAG_TINT = 128
FLAG_FOLIAGE = 256
FLAG_TERRAIN_SHAFTS = 8192
FLAG_TEX_VARIATION = 16384
FLAG_DISTANT_SHADOWS = 32768
FLAG_FLAT_SECONDARY = 1048576
FLAG_PROBE_TAP = 16777216
FLAG_PROBE_AMBIENT = 33554432
FLAG_PROBE_CUBE = 67108864
FLAG_PROBE_BOUNCE = 134217728
FLAG_LIGHT_RGB = 268435456
FLAG_PROBE_SUN = 536870912
FLAG_PROBE_SUN_HIGH = 1073741824
FLAG_SKY_TINT = 2147483648
# the engine's default configuration's resolve flags (src/scene.rs:422-520 with
# src/config.rs:276-380: AO, tint + biomes, terrain shafts, texture variation,
# distant shadows, flat secondary light, probe cube / bounce / sun, RGB light,
# sky tint)
LOOK_FLAGS = (FLAG_AO | FLAG_TINT | FLAG_TERRAIN_SHAFTS | FLAG_TEX_VARIATION | FLAG_DISTANT_SHADOWS |
              FLAG_FLAT_SECONDARY | FLAG_PROBE_CUBE | FLAG_PROBE_BOUNCE | FLAG_LIGHT_RGB | FLAG_PROBE_SUN |
              FLAG_SKY_TINT)

# spec_hi bits (FLAG_HI_*, src/render/mod.rs:196-300) the resolve reads
HI_SKY_SPECULAR, HI_SHORE_WET, HI_SHORE_FOAM, HI_WATER_SEC, HI_CAUSTICS = 1, 8, 16, 32, 64
HI_GLASS_REFLECT, HI_TINT_BALANCE, HI_WATER_LOOK = 128, 512, 4096
HI_SKY_LOOK, HI_SKY_COOL, HI_FOLIAGE_RICH, HI_CANOPY_RELIEF = 1024, 2048, 8192, 16384
HI_COMPACT_SHADE_HIT, HI_LEGACY_LIGHTING = 131072, 1048576
# src/scene.rs:341-411 with the default configuration and a sea: sky specular,
# shore wetting and foam, the half-resolution water legs
HI_DEFAULT = HI_SKY_SPECULAR | HI_SHORE_WET | HI_SHORE_FOAM | HI_WATER_SEC


def atlas(seed: int = 1) -> np.ndarray:
    """The library's procedural atlas in the engine's upload format: uint8
    RGBA (sRGB), mips 16, 8, 4, 2 one after the other."""
    out = np.empty(int(lib().vmw_atlas_bytes(TEX_COUNT)), np.uint8)
    if lib().vmw_build_atlas(seed, ptr(out)):
        raise RuntimeError("vmw_build_atlas failed")
    return out


def block_faces() -> np.ndarray:
    """The engine's face table: 8 words per block id, layer | perm << 16."""
    out = np.empty(26 * 8, np.uint32)
    if lib().vmw_block_faces(ptr(out), out.size):
        raise RuntimeError("vmw_block_faces failed")
    return out


def probe_field(seed: int = 1) -> np.ndarray:
    """A probe field: uint16 binary16 RGBA, 128 x 768 x 128 texels ([z][y][x][4])."""
    out = np.empty(PROBE_SHAPE[0] * PROBE_SHAPE[1] * PROBE_SHAPE[2] * 4, np.uint16)
    if lib().vmw_probe_field(seed, ptr(out)):
        raise RuntimeError("vmw_probe_field failed")
    return out


def shaft_envelope(recipe, sun_dir, origin, texel: float = 4.0) -> np.ndarray:
    """The terrain sun envelope of a recipe on the 512 x 512 window at origin (x, z)."""
    out = np.empty(SHAFT_DIM * SHAFT_DIM, np.float32)
    sun = np.asarray(sun_dir, np.float32)
    org = np.asarray(origin, np.float32)
    if lib().vmw_shaft_envelope(C.byref(recipe.c()), ptr(sun), ptr(org), float(texel), ptr(out)):
        raise RuntimeError("vmw_shaft_envelope failed")
    return out


def apply_defaults(frame, seed: int) -> None:
    """The engine's default fog, clouds, god rays, tint and shaft window on a frame."""
    lib().vmw_look_defaults(C.byref(frame), int(seed))


def sun_visibility(shadow: np.ndarray, mask: np.ndarray | None = None, soft_rays: bool = False) -> np.ndarray:
    """The sun visibility the resolve reads per pixel (the engine's primary_sun,
    an r8unorm target): the soft-shadow mask, else 1 - blocked, rounded to
    the 8-bit target in float32."""
    if mask is not None:
        m = np.asarray(mask, np.float32)
    elif soft_rays:
        m = np.float32(1.0) - np.asarray(shadow, np.float32)
    else:
        m = np.where(np.asarray(shadow) > 0, np.float32(0.0), np.float32(1.0)).astype(np.float32)
    m = np.clip(m, np.float32(0.0), np.float32(1.0)).astype(np.float32)
    return (np.floor(m * np.float32(255.0) + np.float32(0.5)) / np.float32(255.0)).astype(np.float32)
