"""Host-side world store and the synthetic workloads.

`World` wraps the library's world store (include/voxmarch_world.h): chunks
encoded in the engine's tree format (build_local, src/voxel/tree.rs:89-204)
and packed into the three pools the march reads; `World.view()` is the
engine's per-frame `build_chunk_list` plus the GpuFrame fill
(src/render/mod.rs:1447-1564, 1640-1707).
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field

import numpy as np

from . import native
from .native import VmFrame, VmwCamera, VmwChunkInfo, VmwPoolStats, VmwRecipe, lib, ptr

# GpuFrame.flags bits (src/render/mod.rs:144-270, common.wgsl:142-162)
FLAG_HIZ = 1
FLAG_HEATMAP = 2
FLAG_SHADOWS = 4
FLAG_WATER_REFLECT = 16
FLAG_WATER_REFRACT = 32
FLAG_UNDERWATER = 64
FLAG_WAVES = 512
FLAG_WATER_FAR = 2097152
FLAG_WATER_DARK = 4194304

NO_CHUNK = 0xFFFFFFFF
GRID_X, GRID_Y, GRID_Z = 32, 8, 32
MAX_CHUNKS = 8191
TILE = 8

# block ids (src/block.rs:3-35)
AIR, STONE, DIRT, GRASS, SAND, GRAVEL, LOG, LEAVES, PLANKS, COBBLE, GLASS, GLOWSTONE, BEDROCK, WATER = range(14)
PINE_LEAVES, TALL_GRASS = 16, 18


def dense_index(x, y, z):
    """src/voxel/tree.rs:8-10"""
    return x | (z << 6) | (y << 12)


@dataclass
class Recipe:
    size: tuple = (256, 128, 256)
    octaves: int = 4
    seed: int = 1
    base: float = 48.0
    amplitude: float = 40.0
    base_freq: float = 1.0 / 64.0
    water_level: int = 64
    water_depth: int = 0
    tree_permille: int = 10
    glass_permille: int = 0
    island_permille: int = 0
    tuft_permille: int = 0

    def c(self) -> VmwRecipe:
        r = VmwRecipe()
        r.size[:] = self.size
        r.octaves, r.seed, r.base, r.amplitude, r.base_freq = self.octaves, self.seed, self.base, self.amplitude, self.base_freq
        r.water_level, r.water_depth = self.water_level, self.water_depth
        r.tree_permille, r.glass_permille, r.island_permille = self.tree_permille, self.glass_permille, self.island_permille
        r.tuft_permille = self.tuft_permille
        return r


def recipe_small_terrain() -> Recipe:
    """256x128x256 world: 4-octave value-noise heightfield (base 48, amplitude 40,
    seed 1), water below y=64, trees on 1% of dry surface columns."""
    return Recipe()


def recipe_large_terrain() -> Recipe:
    """1024x256x1024 world: same recipe with 6 octaves and seed 7, plus ~3% glass
    in the top two surface layers."""
    return Recipe(size=(1024, 256, 1024), octaves=6, seed=7, glass_permille=30)


def recipe_sparse_world() -> Recipe:
    """4096x256x4096 sparse world (seed 21): terrain islands, a water sheet at
    y=64, trees on 2% of dry columns."""
    return Recipe(size=(4096, 256, 4096), octaves=6, seed=21, base=40.0, amplitude=48.0, water_level=64,
                  water_depth=2, tree_permille=20, island_permille=120)


@dataclass
class Camera:
    pos: tuple
    yaw: float = math.radians(90.0)
    pitch: float = math.radians(-15.0)
    fov_y: float = math.radians(70.0)
    width: int = 640
    height: int = 360
    far: float = 2600.0
    sun_dir: tuple = None
    daylight: float = 1.0
    flags: int = FLAG_SHADOWS | FLAG_WATER_REFRACT
    jitter: tuple = (0.0, 0.0)
    frame_index: int = 0
    sea_level: float = 64.0
    offscreen_shadows: bool = True
    basis: tuple = None          # (fwd, right, up) overrides yaw/pitch
    grid_dim: tuple = None
    grid_min: tuple = None
    max_chunks: int = 0

    def c(self) -> VmwCamera:
        cam = VmwCamera()
        cam.pos[:] = self.pos
        cam.yaw, cam.pitch, cam.fov_y = self.yaw, self.pitch, self.fov_y
        if self.basis is not None:
            cam.use_basis = 1
            cam.fwd[:], cam.right[:], cam.up[:] = self.basis
        cam.width, cam.height, cam.far = self.width, self.height, self.far
        sun = self.sun_dir if self.sun_dir is not None else default_sun()
        cam.sun_dir[:] = sun
        cam.daylight, cam.flags = self.daylight, self.flags
        cam.jitter[:] = self.jitter
        cam.frame_index, cam.sea_level = self.frame_index, self.sea_level
        cam.offscreen_shadows = 1 if self.offscreen_shadows else 0
        if self.grid_dim is not None:
            cam.grid_dim[:] = self.grid_dim
        if self.grid_min is not None:
            cam.grid_min_set = 1
            cam.grid_min[:] = self.grid_min
        cam.max_chunks = self.max_chunks
        return cam


def default_sun() -> tuple:
    """normalize(0.4, 0.8, 0.3) in float32, as the frame carries it."""
    v = np.array([0.4, 0.8, 0.3], np.float32)
    return tuple((v / np.sqrt(np.float32((v * v).sum()))).astype(np.float32).tolist())


@dataclass
class View:
    """One frame's march inputs: the GpuFrame, the chunk list and the grid."""
    frame: VmFrame
    chunks: np.ndarray          # CHUNK_DTYPE, visible chunks first
    grid: np.ndarray            # uint32, NO_CHUNK where empty

    @property
    def res(self):
        return int(self.frame.res[0]), int(self.frame.res[1])

    @property
    def n_pixels(self):
        return int(self.frame.res[0]) * int(self.frame.res[1])


class World:
    """The engine's voxel world store (src/voxel/world.rs:16-29)."""

    def __init__(self):
        self._L = lib()
        self._h = self._L.vmw_create()
        if not self._h:
            raise RuntimeError("vmw_create failed")

    def close(self):
        if self._h:
            self._L.vmw_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- building -------------------------------------------------------
    @classmethod
    def generate(cls, recipe: Recipe) -> "World":
        w = cls()
        rc = w._L.vmw_generate(w._h, C.byref(recipe.c()))
        if rc:
            raise ValueError(f"vmw_generate failed ({rc}); sizes must be multiples of 64")
        w.recipe = recipe
        return w

    def insert_dense(self, key: tuple, dense: np.ndarray, lod: int = 0):
        """World::insert_local(key, build_local(dense)); dense is u16[64^3],
        index x | z<<6 | y<<12."""
        d = np.ascontiguousarray(dense, dtype=np.uint16).reshape(-1)
        assert d.size == 64 ** 3
        rc = self._L.vmw_insert_dense(self._h, lod, key[0], key[1], key[2], ptr(d))
        if rc:
            raise RuntimeError("insert failed")

    def remove(self, key: tuple, lod: int = 0) -> bool:
        return self._L.vmw_remove(self._h, lod, *key) == 0

    def get_block(self, x: int, y: int, z: int) -> int:
        return int(self._L.vmw_get_block(self._h, x, y, z))

    def chunk_info(self, key: tuple, lod: int = 0):
        info = VmwChunkInfo()
        if self._L.vmw_get_chunk_info(self._h, lod, key[0], key[1], key[2], C.byref(info)):
            return None
        return info

    def set_fade(self, key: tuple, fade: float, lod: int = 0):
        """The chunk's LOD cross-fade (RenderItem::fade, src/lod.rs:56-80)."""
        rc = self._L.vmw_set_fade(self._h, lod, key[0], key[1], key[2], fade)
        if rc:
            raise KeyError(key) if rc == 1 else ValueError(fade)

    def pool_stats(self) -> VmwPoolStats:
        s = VmwPoolStats()
        self._L.vmw_pool_stats(self._h, C.byref(s))
        return s

    def pools(self):
        """Copies of the inner (n x 4 u32), leaf (n x 2 u32) and brick (u32) pools."""
        s = self.pool_stats()

        def grab(p, n):
            if n == 0:
                return np.zeros(0, np.uint32)
            return np.ctypeslib.as_array(C.cast(p, C.POINTER(C.c_uint32)), shape=(n,)).copy()

        inners = grab(self._L.vmw_inners(self._h), s.n_inners * 4).reshape(-1, 4)
        leaves = grab(self._L.vmw_leaves(self._h), s.n_leaves * 2).reshape(-1, 2)
        bricks = grab(self._L.vmw_bricks(self._h), s.n_bricks)
        return inners, leaves, bricks

    # -- per frame --------------------------------------------------------
    def view(self, cam: Camera) -> View:
        frame = VmFrame()
        s = self.pool_stats()
        cap = max(int(s.n_chunks), 1)
        chunks = np.zeros(cap, native.CHUNK_DTYPE)
        gd = cam.grid_dim or (GRID_X, GRID_Y, GRID_Z)
        grid = np.zeros(int(np.prod(gd)), np.uint32)
        n = C.c_uint32(0)
        rc = self._L.vmw_build_view(self._h, C.byref(cam.c()), C.byref(frame), ptr(chunks), cap, C.byref(n), ptr(grid))
        if rc:
            raise RuntimeError(f"vmw_build_view failed ({rc})")
        return View(frame=frame, chunks=chunks[: n.value].copy(), grid=grid)


def camera_basis(yaw: float, pitch: float):
    """src/player.rs:122-126 + src/scene.rs:334-339"""
    f, r, u = (np.zeros(3, np.float32) for _ in range(3))
    lib().vmw_camera_basis(yaw, pitch, ptr(f), ptr(r), ptr(u))
    return f, r, u


def pairs_for(tiles_x: int, tiles_y: int) -> int:
    """src/render/mod.rs:27-30"""
    return int(lib().vmw_pairs_for(tiles_x, tiles_y))


def halton_jitter(index: int):
    """src/math.rs:119-134"""
    out = np.zeros(2, np.float32)
    lib().vmw_halton_jitter(index, ptr(out))
    return float(out[0]), float(out[1])


def recipe_dense_chunks(recipe: Recipe) -> np.ndarray:
    """Every dense chunk of the recipe's world (n x 64^3 u16), chunk i at
    (i % nx, i // nx % ny, i // (nx ny)), the order World.generate inserts."""
    n = (recipe.size[0] // 64) * (recipe.size[1] // 64) * (recipe.size[2] // 64)
    out = np.empty((n, 64 ** 3), np.uint16)
    if lib().vmw_recipe_dense_all(C.byref(recipe.c()), ptr(out)):
        raise RuntimeError("vmw_recipe_dense_all failed")
    return out


def recipe_mixed_lod() -> Recipe:
    """512x128x512 terrain (the small world's noise, water and trees) for the
    mixed level-of-detail layout."""
    return Recipe(size=(512, 128, 512))


def mixed_lod_layout():
    """(lod, chunk cell, fade) of a world mixing the engine's LOD levels: lod-0
    chunks over x, z in [0, 256), of which the 2x2x2 block over [128, 256)^2
    fades in (0.6) over its fading-out lod-1 parent (-0.6); lod-1 chunks
    (voxels of 2) over x in [256, 512), z in [0, 256); lod-2 chunks (voxels of
    4) over z in [256, 512).  Chunk cells are in units of the level's chunk
    size (64 << lod)."""
    items = []
    for cz in range(4):
        for cy in range(2):
            for cx in range(4):
                fading = cx >= 2 and cz >= 2
                items.append((0, (cx, cy, cz), 0.6 if fading else 1.0))
    items.append((1, (1, 0, 1), -0.6))
    for cz in range(2):
        for cx in range(2, 4):
            items.append((1, (cx, 0, cz), 1.0))
    for cx in range(2):
        items.append((2, (cx, 0, 1), 1.0))
    return items


def layout_dense(recipe: Recipe, lod: int, key: tuple) -> np.ndarray:
    """Dense blocks of one chunk of a layout: the recipe's full-resolution
    chunk for lod 0, its sampled coarse chunk otherwise."""
    if lod == 0:
        out = np.empty(64 ** 3, np.uint16)
        if lib().vmw_recipe_dense(C.byref(recipe.c()), key[0], key[1], key[2], ptr(out)):
            raise ValueError("vmw_recipe_dense failed")
        return out
    return recipe_dense_lod(recipe, lod, key)


def build_layout(world, recipe: Recipe, layout) -> None:
    """Insert every chunk of layout [(lod, key, fade)] into world and set its fade."""
    for lod, key, fade in layout:
        world.insert_dense(key, layout_dense(recipe, lod, key), lod=lod)
    for lod, key, fade in layout:
        if fade != 1.0:
            world.set_fade(key, fade, lod=lod)
    world.recipe = recipe


def recipe_dense_lod(recipe: Recipe, lod: int, key: tuple) -> np.ndarray:
    """The recipe's chunk of level lod at chunk cell key of that level (u16[64^3])."""
    out = np.empty(64 ** 3, np.uint16)
    if lib().vmw_recipe_dense_lod(C.byref(recipe.c()), lod, key[0], key[1], key[2], ptr(out)):
        raise ValueError("vmw_recipe_dense_lod failed")
    return out


def surface_height(recipe: Recipe, x: int, z: int) -> int:
    return int(lib().vmw_recipe_height(C.byref(recipe.c()), x, z))


def small_terrain_camera(width=640, height=360, **kw) -> Camera:
    """The 256x128x256 world's camera: (128,110,20), looking +z, pitched -15 deg,
    vertical fov 70 deg."""
    return Camera(pos=(128.0, 110.0, 20.0), width=width, height=height, **kw)


def penumbra_camera(width=640, height=360, **kw) -> Camera:
    """A low camera over the 256x128x256 world, (60.5, 79.5, 60.5), looking +z,
    pitched -45 deg: close enough to the ground that tree and hill shadows
    have penumbrae wider than a pixel for the bilateral shadow filter."""
    kw.setdefault("pitch", math.radians(-45.0))
    return Camera(pos=(60.5, 79.5, 60.5), width=width, height=height, **kw)


def large_terrain_camera(recipe: Recipe, width=1920, height=1080, dx=0.0, **kw) -> Camera:
    """The 1024x256x1024 world's camera: centre column, 30 above the surface,
    looking +z, pitched -15 deg; dx shifts it along x (0.5 for the Hi-Z frame)."""
    h = surface_height(recipe, 512, 512)
    return Camera(pos=(512.0 + dx, float(h + 30), 512.0), width=width, height=height, **kw)
