"""ctypes binding of the oracle's world producer (oracle/producer.cpp, in
liboracle.so) -- test infrastructure.

`OracleWorld` restates the engine's CPU world producers (build_local, the run
and word pools, World::insert_local, build_chunk_list) independently of the
product's world store.  Only tests/, __graft_entry__.smoke() and bench.py's
CPU legs use it: as the producer of the oracle's own inputs, and as the
checker of the product's encoder and world store.  It reuses the product's
plain ctypes structures and dataclasses (Recipe, Camera, View) but never
loads the product library.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from voxelcraft_menu_b200.native import CHUNK_DTYPE, VmFrame, VmwCamera, VmwChunkInfo, VmwPoolStats, VmwRecipe
from voxelcraft_menu_b200.world import GRID_X, GRID_Y, GRID_Z, Recipe, View

from .oracle import lib as _oracle_lib

vp = C.c_void_p
P = C.POINTER

_SIGS = {
    "orw_create": (vp, []),
    "orw_destroy": (None, [vp]),
    "orw_insert_dense": (C.c_int, [vp, C.c_uint8, C.c_int32, C.c_int32, C.c_int32, vp]),
    "orw_build_tree": (C.c_int, [vp, C.c_uint32, vp, vp, vp, vp, vp]),
    "orw_insert_tree": (C.c_int, [vp, C.c_uint8, C.c_int32, C.c_int32, C.c_int32, vp, vp, vp, vp, vp]),
    "orw_remove": (C.c_int, [vp, C.c_uint8, C.c_int32, C.c_int32, C.c_int32]),
    "orw_set_fade": (C.c_int, [vp, C.c_uint8, C.c_int32, C.c_int32, C.c_int32, C.c_float]),
    "orw_get_block": (C.c_uint32, [vp, C.c_int32, C.c_int32, C.c_int32]),
    "orw_get_chunk_info": (C.c_int, [vp, C.c_uint8, C.c_int32, C.c_int32, C.c_int32, P(VmwChunkInfo)]),
    "orw_l1_node": (C.c_int, [vp, C.c_uint8, C.c_int32, C.c_int32, C.c_int32, C.c_uint32, vp]),
    "orw_pool_stats": (None, [vp, P(VmwPoolStats)]),
    "orw_inners": (vp, [vp]),
    "orw_leaves": (vp, [vp]),
    "orw_bricks": (vp, [vp]),
    "orw_generate": (C.c_int, [vp, P(VmwRecipe)]),
    "orw_recipe_dense": (C.c_int, [P(VmwRecipe), C.c_int32, C.c_int32, C.c_int32, vp]),
    "orw_recipe_dense_all": (C.c_int, [P(VmwRecipe), vp]),
    "orw_recipe_dense_lod": (C.c_int, [P(VmwRecipe), C.c_uint32, C.c_int32, C.c_int32, C.c_int32, vp]),
    "orw_recipe_height": (C.c_int32, [P(VmwRecipe), C.c_int32, C.c_int32]),
    "orw_camera_basis": (None, [C.c_float, C.c_float, vp, vp, vp]),
    "orw_pairs_for": (C.c_uint32, [C.c_uint32, C.c_uint32]),
    "orw_build_view": (C.c_int, [vp, P(VmwCamera), P(VmFrame), vp, C.c_uint32, P(C.c_uint32), vp]),
    "orw_halton_jitter": (None, [C.c_uint64, vp]),
}
_bound = None


def lib():
    global _bound
    if _bound is None:
        L = _oracle_lib()
        for n, (r, a) in _SIGS.items():
            f = getattr(L, n)
            f.restype, f.argtypes = r, a
        _bound = L
    return _bound


def _ptr(a: np.ndarray):
    assert a.flags["C_CONTIGUOUS"]
    return C.c_void_p(a.ctypes.data)


class OracleWorld:
    """The engine's world store restated (src/voxel/world.rs:16-29)."""

    def __init__(self):
        self._L = lib()
        self._h = self._L.orw_create()
        self.recipe = None

    def close(self):
        if self._h:
            self._L.orw_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @classmethod
    def generate(cls, recipe: Recipe) -> "OracleWorld":
        w = cls()
        if w._L.orw_generate(w._h, C.byref(recipe.c())):
            raise ValueError("orw_generate failed")
        w.recipe = recipe
        return w

    def insert_dense(self, key: tuple, dense: np.ndarray, lod: int = 0):
        d = np.ascontiguousarray(dense, dtype=np.uint16).reshape(-1)
        assert d.size == 64 ** 3
        if self._L.orw_insert_dense(self._h, lod, key[0], key[1], key[2], _ptr(d)):
            raise RuntimeError("insert failed")

    def insert_tree(self, key: tuple, info, l1, leaves, attrs, palette, lod: int = 0):
        rc = self._L.orw_insert_tree(self._h, lod, key[0], key[1], key[2], _ptr(info), _ptr(l1) if l1.size else None,
                                     _ptr(leaves) if leaves.size else None, _ptr(attrs) if attrs.size else None,
                                     _ptr(palette) if palette.size else None)
        if rc:
            raise RuntimeError("orw_insert_tree rejected the chunk")

    def remove(self, key: tuple, lod: int = 0) -> bool:
        return self._L.orw_remove(self._h, lod, *key) == 0

    def set_fade(self, key: tuple, fade: float, lod: int = 0):
        if self._L.orw_set_fade(self._h, lod, key[0], key[1], key[2], fade):
            raise KeyError(key)

    def get_block(self, x: int, y: int, z: int) -> int:
        return int(self._L.orw_get_block(self._h, x, y, z))

    def chunk_info(self, key: tuple, lod: int = 0):
        info = VmwChunkInfo()
        if self._L.orw_get_chunk_info(self._h, lod, key[0], key[1], key[2], C.byref(info)):
            return None
        return info

    def l1_node(self, key: tuple, l1b: int, lod: int = 0):
        """Inner node (mask u64, run_ptr, leaf_prefix) or None (src/voxel/world.rs:225)."""
        out = np.zeros(4, np.uint32)
        rc = self._L.orw_l1_node(self._h, lod, key[0], key[1], key[2], l1b, _ptr(out))
        if rc < 0:
            raise KeyError(key)
        if rc == 0:
            return None
        return (int(out[0]) | (int(out[1]) << 32), int(out[2]), int(out[3]))

    def pool_stats(self) -> VmwPoolStats:
        s = VmwPoolStats()
        self._L.orw_pool_stats(self._h, C.byref(s))
        return s

    def pools(self):
        s = self.pool_stats()

        def grab(p, n):
            if n == 0:
                return np.zeros(0, np.uint32)
            return np.ctypeslib.as_array(C.cast(p, C.POINTER(C.c_uint32)), shape=(n,)).copy()

        return (grab(self._L.orw_inners(self._h), s.n_inners * 4).reshape(-1, 4),
                grab(self._L.orw_leaves(self._h), s.n_leaves * 2).reshape(-1, 2),
                grab(self._L.orw_bricks(self._h), s.n_bricks))

    def view(self, cam) -> View:
        frame = VmFrame()
        cap = max(int(self.pool_stats().n_chunks), 1)
        chunks = np.zeros(cap, CHUNK_DTYPE)
        gd = cam.grid_dim or (GRID_X, GRID_Y, GRID_Z)
        grid = np.zeros(int(np.prod(gd)), np.uint32)
        n = C.c_uint32(0)
        rc = self._L.orw_build_view(self._h, C.byref(cam.c()), C.byref(frame), _ptr(chunks), cap, C.byref(n),
                                    _ptr(grid))
        if rc:
            raise RuntimeError(f"orw_build_view failed ({rc})")
        return View(frame=frame, chunks=chunks[: n.value].copy(), grid=grid)


def recipe_dense(recipe: Recipe, lod: int, key: tuple) -> np.ndarray:
    out = np.empty(64 ** 3, np.uint16)
    L = lib()
    rc = (L.orw_recipe_dense(C.byref(recipe.c()), key[0], key[1], key[2], _ptr(out)) if lod == 0 else
          L.orw_recipe_dense_lod(C.byref(recipe.c()), lod, key[0], key[1], key[2], _ptr(out)))
    if rc:
        raise ValueError("recipe dense failed")
    return out


def build_layout(recipe: Recipe, layout) -> OracleWorld:
    """An OracleWorld of the chunks of layout [(lod, key, fade)]."""
    w = OracleWorld()
    for lod, key, fade in layout:
        w.insert_dense(key, recipe_dense(recipe, lod, key), lod=lod)
    for lod, key, fade in layout:
        if fade != 1.0:
            w.set_fade(key, fade, lod=lod)
    w.recipe = recipe
    return w


def surface_height(recipe: Recipe, x: int, z: int) -> int:
    return int(lib().orw_recipe_height(C.byref(recipe.c()), x, z))


def build_tree(dense: np.ndarray, palette_cap: int = 16384):
    """build_local of one dense chunk in the flat encoder layout:
    (info, l1, leaves, attrs, palette) trimmed to their lengths."""
    from voxelcraft_menu_b200.encode import INFO_DTYPE, L1_DTYPE, TREE_L1, TREE_LEAVES
    info = np.zeros(1, INFO_DTYPE)
    l1 = np.zeros(TREE_L1, L1_DTYPE)
    leaves = np.zeros(TREE_LEAVES, np.uint64)
    attrs = np.zeros(TREE_LEAVES, np.uint32)
    pal = np.zeros(palette_cap, np.uint32)
    d = np.ascontiguousarray(dense, np.uint16).reshape(-1)
    if lib().orw_build_tree(_ptr(d), palette_cap, _ptr(info), _ptr(l1), _ptr(leaves), _ptr(attrs), _ptr(pal)):
        raise RuntimeError("orw_build_tree failed")
    n = info[0]
    return (info, l1[: n["n_l1"]].copy(), leaves[: n["n_leaves"]].copy(), attrs[: n["n_attrs"]].copy(),
            pal[: min(int(n["n_palette"]), palette_cap)].copy())
