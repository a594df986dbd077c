"""Layout producers, checked with the reference's own fixtures and assertions
(tests/tree.rs, tests/full_march.rs, tests/emitter_gate.rs, tests/pairs.rs,
tests/camera.rs, tests/shadow_grid.rs): the oracle's restatement of the
engine's encoder, pools and chunk list (oracle/producer.cpp) and the
product's world store (csrc/store.cpp) each pass them, and the two agree on
every block, chunk record and grid cell."""
import math

import numpy as np
import pytest

from oracle.producer import OracleWorld
from oracle import producer as OP
from voxelcraft_menu_b200 import world as W
from voxelcraft_menu_b200.world import Camera, World, dense_index

PRODUCERS = {"product": World, "oracle": OracleWorld}


@pytest.fixture(params=sorted(PRODUCERS))
def producer(request):
    return PRODUCERS[request.param]


def l1_node(w, key, l1b):
    """World::l1_node (src/voxel/world.rs:225-234) read through the packed
    pools: (mask, run_ptr, leaf_prefix), or None when the cell is empty."""
    rec = w.chunk_info(key)
    root = rec.root[0] | (rec.root[1] << 32)
    if not (root >> l1b) & 1:
        return None
    if rec.root[2] & 0x80000000:
        return ((1 << 64) - 1, 0x80000000, l1b * 64)
    inners, _, _ = w.pools()
    n = inners[rec.root[2] + bin(root & ((1 << l1b) - 1)).count("1")]
    return (int(n[0]) | (int(n[1]) << 32), int(n[2]), int(n[3]))

X, Y, Z = np.meshgrid(np.arange(64, dtype=np.uint32), np.arange(64, dtype=np.uint32),
                      np.arange(64, dtype=np.uint32), indexing="ij")


def dense_from(f):
    """tests/tree.rs:9-19: f(x, y, z) over the 64^3 cube, dense index x | z<<6 | y<<12."""
    ids = f(X, Y, Z).astype(np.uint16)
    d = np.zeros(64 ** 3, np.uint16)
    d[dense_index(X, Y, Z).ravel()] = ids.ravel()
    return d


def hash3(x, y, z, seed):
    """tests/tree.rs:21-27 (wrapping u32 arithmetic)."""
    x, y, z = (np.asarray(a, np.uint64) for a in (x, y, z))
    m = np.uint64(0xFFFFFFFF)
    h = ((x * np.uint64(0x8da6b343)) & m) ^ ((y * np.uint64(0xd8163841)) & m) ^ ((z * np.uint64(0xcb1ab31f)) & m) \
        ^ np.uint64(seed)
    h ^= h >> np.uint64(13)
    h = (h * np.uint64(0x5bd1e995)) & m
    return (h ^ (h >> np.uint64(15))) & m


def terrain(seed):
    """tests/tree.rs:29-50"""
    def f(x, y, z):
        fx = (x.astype(np.float32) + np.float32(seed * 13.0)) * np.float32(0.11)
        fz = (z.astype(np.float32) + np.float32(seed * 7.0)) * np.float32(0.09)
        h = (np.float32(30.0) + np.float32(10.0) * np.sin(fx) * np.cos(fz)
             + np.float32(4.0) * np.cos(fx * np.float32(3.1))).astype(np.uint32)
        out = np.full(x.shape, W.STONE, np.uint32)
        out[hash3(x, y, z, seed + 1) % 41 == 0] = W.GLOWSTONE
        out[hash3(x, y, z, seed) % 23 == 0] = W.GRAVEL if hasattr(W, "GRAVEL") else 5
        out[y + 4 >= h] = W.DIRT
        out[y + 1 == h] = W.GRASS
        cave = (y > 8) & (y + 6 < h) & (hash3(x // 3, y // 3, z // 3, seed) % 11 == 0)
        out[cave] = W.AIR
        out[y >= h] = W.AIR
        return out
    return f


def world_matches(w, key, dense):
    o = np.array(key) * 64
    got = np.array([w.get_block(int(o[0] + x), int(o[1] + y), int(o[2] + z))
                    for y in range(64) for z in range(64) for x in range(64)], np.uint16)
    want = np.array([dense[dense_index(x, y, z)] for y in range(64) for z in range(64) for x in range(64)], np.uint16)
    return np.array_equal(got, want)


def assert_pools_empty(w):
    s = w.pool_stats()
    assert s.live_leaves == 0 and s.live_inners == 0
    assert s.referenced_leaves == 0 and s.referenced_inners == 0
    assert s.used_words == 0


def test_local_roundtrip(producer):
    """tests/tree.rs:77-92"""
    d = dense_from(terrain(1))
    w = producer()
    w.insert_dense((0, 0, 0), d)
    assert w.chunk_info((0, 0, 0)).solid_count > 0
    assert world_matches(w, (0, 0, 0), d)


def test_world_roundtrip_and_aabb(producer):
    """tests/tree.rs:94-109"""
    d = dense_from(terrain(2))
    w = producer()
    w.insert_dense((3, 1, -2), d)
    assert world_matches(w, (3, 1, -2), d)
    rec = w.chunk_info((3, 1, -2))
    assert rec.aabb_min[1] == 0
    assert rec.aabb_max[1] <= 45
    assert rec.aabb_min[0] == 0 and rec.aabb_max[0] == 64
    assert w.get_block(0, -1, 0) == W.AIR
    assert w.get_block(1000, 10, 1000) == W.AIR
    w.remove((3, 1, -2))
    assert_pools_empty(w)


def test_identical_chunks_share_runs(producer):
    """tests/tree.rs:111-135"""
    d = dense_from(terrain(3))
    w = producer()
    w.insert_dense((0, 0, 0), d)
    s0 = w.pool_stats()
    assert s0.live_leaves > 0 and s0.live_inners > 0
    w.insert_dense((5, 0, 5), d)
    s1 = w.pool_stats()
    assert s1.live_leaves == s0.live_leaves, "second identical chunk must add no leaf data"
    assert s1.live_inners == s0.live_inners, "second identical chunk must add no inner data"
    assert s1.referenced_inners / s1.live_inners >= 2.0 - 1e-9
    assert world_matches(w, (5, 0, 5), d)
    w.remove((0, 0, 0))
    assert w.pool_stats().live_leaves == s0.live_leaves
    assert world_matches(w, (5, 0, 5), d)
    w.remove((5, 0, 5))
    assert_pools_empty(w)


def test_uniform_chunk_costs_nothing(producer):
    """tests/tree.rs:137-152"""
    d = dense_from(lambda x, y, z: np.full(x.shape, W.STONE))
    w = producer()
    w.insert_dense((0, 0, 0), d)
    rec = w.chunk_info((0, 0, 0))
    assert rec.root[2] & 0x80000000, "root must be full"
    assert rec.attr_uniform == 1 and rec.attr_value == W.STONE
    s = w.pool_stats()
    assert s.live_leaves == 0 and s.live_inners == 0 and s.used_words == 0
    assert w.get_block(17, 33, 60) == W.STONE


def test_empty_chunk(producer):
    """tests/tree.rs:154-157 (the insertion half; edits are not on the march path)"""
    d = dense_from(lambda x, y, z: np.zeros(x.shape))
    w = producer()
    w.insert_dense((0, 0, 0), d)
    rec = w.chunk_info((0, 0, 0))
    assert rec.root[0] == 0 and rec.root[1] == 0
    assert w.get_block(1, 2, 3) == W.AIR


def test_many_block_types_attribute_recovery(producer):
    """tests/tree.rs:231-246 (every palette width: up to 25 ids per leaf)"""
    d = dense_from(lambda x, y, z: np.where(y > 40, 0, 1 + (x * 7 + y * 3 + z * 5) % 25))
    w = producer()
    w.insert_dense((0, 0, 0), d)
    assert world_matches(w, (0, 0, 0), d)
    w.remove((0, 0, 0))
    assert_pools_empty(w)


def test_water_line_packing_and_stratification(producer):
    """tests/tree.rs:281-314"""
    d = dense_from(lambda x, y, z: np.where(y <= 9, W.DIRT, np.where(y <= 12, W.WATER, W.AIR)))
    w = producer()
    w.insert_dense((0, 0, 0), d)
    rec = w.chunk_info((0, 0, 0))
    for l1b in range(64):
        n = l1_node(w, (0, 0, 0), l1b)
        if n is None:
            continue
        _mask, run_ptr, prefix = n
        wl = prefix >> 28
        if run_ptr & 0x80000000:
            assert wl == 15, "full solid cell must report 15"
        else:
            assert wl == 9, "mixed cell keeps the land top"
        assert (prefix & 0x0FFFFFFF) == (prefix & ~0xF0000000 & 0xFFFFFFFF)
    assert rec.dry_mask == (rec.root[0] | (rec.root[1] << 32))
    assert rec.dry_mask != 0


def test_water_only_cells_report_fifteen_and_leave_the_dry_mask(producer):
    """tests/tree.rs:316-345"""
    d = dense_from(lambda x, y, z: np.where(y <= 4, W.STONE, np.where(y <= 30, W.WATER, W.AIR)))
    w = producer()
    w.insert_dense((0, 0, 0), d)
    nodes = [l1_node(w, (0, 0, 0), b) for b in range(64)]
    nodes = [n for n in nodes if n is not None]
    water_only = sum(1 for m, rp, pre in nodes if pre >> 28 == 15 and not rp & 0x80000000)
    assert water_only == 16
    dry_solid = sum(1 for m, rp, pre in nodes if pre >> 28 == 15 and rp & 0x80000000)
    carrying_top = sum(1 for m, rp, pre in nodes if pre >> 28 == 4)
    assert dry_solid + carrying_top == 16
    rec = w.chunk_info((0, 0, 0))
    root_mask = rec.root[0] | (rec.root[1] << 32)
    assert bin(rec.dry_mask).count("1") == 16
    assert rec.dry_mask != root_mask
    assert bin(root_mask).count("1") == 32


def test_full_mixed_root(producer):
    """tests/full_march.rs:7-40: water above stone collapses to a full root whose
    dry mask holds exactly the bottom 32 cells."""
    d = dense_from(lambda x, y, z: np.where(y < 32, W.STONE, W.WATER))
    w = producer()
    w.insert_dense((0, 0, 0), d)
    rec = w.chunk_info((0, 0, 0))
    assert rec.root[2] & 0x80000000
    assert rec.has_water
    assert rec.dry_mask not in (0, (1 << 64) - 1)
    assert bin(rec.dry_mask).count("1") == 32


def test_seabed_sets_its_line_and_open_sea_carries_fifteen(producer):
    """tests/emitter_gate.rs:108-140"""
    d = dense_from(lambda x, y, z: np.where(y <= 8, W.STONE, np.where(y <= 40, W.WATER, W.AIR)))
    w = producer()
    w.insert_dense((0, 0, 0), d)
    rec = w.chunk_info((0, 0, 0))
    assert not rec.root[2] & 0x80000000
    for l1b in range(64):
        yn = (l1b >> 2) & 3
        n = l1_node(w, (0, 0, 0), l1b)
        if yn == 0:
            assert n[2] >> 28 == 8
        elif yn == 3:
            assert n is None
        else:
            assert n[2] >> 28 == 15


def test_prefix_mask_and_nibble():
    """tests/emitter_gate.rs:102-106,143-148"""
    prefix_mask = 0x0FFFFFFF
    assert prefix_mask > 64 * 64
    assert prefix_mask & 0xF0000000 == 0


def test_pairs_for_matches_the_engine():
    """tests/pairs.rs:12-77"""
    tiles = lambda w, h: ((w + 7) // 8, (h + 7) // 8)
    for w, h in [(1280, 720), (1920, 1080), (2560, 1440)]:
        assert W.pairs_for(*tiles(w, h)) == 1 << 20
    for w, h, demand in [(3840, 2160, 1_313_456), (5120, 2880, 2_325_513)]:
        assert W.pairs_for(*tiles(w, h)) > demand
    tx, ty = tiles(7680, 4320)
    assert tx * ty <= 1 << 19
    tx, ty = tiles(8192, 4320)
    assert tx * ty > 1 << 19
    assert W.pairs_for(*tiles(7680, 4320)) > 2_325_513


def test_halton_jitter_covers_the_pixel_and_repeats():
    """tests/camera.rs:125-157"""
    seen = []
    s = np.zeros(2)
    for i in range(8):
        j = W.halton_jitter(i)
        assert -0.5 < j[0] <= 0.5 and -0.5 < j[1] <= 0.5
        assert j != (0.0, 0.0)
        assert not any(abs(a - j[0]) < 1e-6 and abs(b - j[1]) < 1e-6 for a, b in seen)
        seen.append(j)
        s += j
        assert j == W.halton_jitter(i + 8)
    assert np.linalg.norm(s / 8) < 0.1


def test_camera_basis_is_orthonormal_and_looks_along_yaw():
    """src/player.rs:122-126 and src/scene.rs:334-339"""
    f, r, u = W.camera_basis(np.radians(90.0), np.radians(-15.0))
    assert abs(f[0]) < 1e-6 and f[1] < 0 and f[2] > 0
    for v in (f, r, u):
        assert abs(np.linalg.norm(v) - 1) < 1e-6
    assert abs(np.dot(f, r)) < 1e-6 and abs(np.dot(f, u)) < 1e-6 and abs(np.dot(r, u)) < 1e-6
    assert u[1] > 0


def test_generated_world_matches_its_recipe():
    """The synthetic terrain: heights, water below 64, surface blocks."""
    rec = W.recipe_small_terrain()
    w = World.generate(rec)
    assert w.pool_stats().n_chunks == 4 * 2 * 4
    for (x, z) in [(3, 5), (100, 200), (255, 0), (17, 130)]:
        h = W.surface_height(rec, x, z)
        assert 48 <= h < 88
        assert w.get_block(x, h - 1, z) in (W.GRASS, W.LOG, W.LEAVES)
        assert w.get_block(x, h - 3, z) == W.DIRT
        assert w.get_block(x, h - 6, z) == W.STONE
        if h < 64:
            assert w.get_block(x, 63, z) == W.WATER
        assert w.get_block(x, 64 + 60, z) in (W.AIR,)


def test_view_chunk_list_is_sorted_and_grid_indexes_it():
    """build_chunk_list (src/render/mod.rs:1447-1564): visible chunks sorted by
    AABB distance, shadow-only chunks after them, the grid names list indices."""
    w = World.generate(W.recipe_small_terrain())
    v = w.view(W.small_terrain_camera())
    f = v.frame
    cam = np.array(f.cam_pos[:])
    ch = v.chunks
    d = np.linalg.norm(np.maximum(np.maximum(ch["aabb_min"] - cam, cam - ch["aabb_max"]), 0), axis=1)
    vis = d[: f.chunk_count]
    assert np.all(np.diff(vis) >= -1e-4)
    used = v.grid[v.grid != W.NO_CHUNK]
    assert used.size == len(ch) and np.array_equal(np.sort(used), np.arange(len(ch)))
    assert f.tiles[0] == 80 and f.tiles[1] == 45
    assert f.max_pairs == 1 << 20


# ---- the shadow casters' grid: tests/shadow_grid.rs --------------------------
# build_chunk_list + partition_for_grid (src/render/mod.rs:88-138,1447-1564):
# the frame's list is the frustum-visible chunks (frame.chunk_count of them)
# followed by the off-screen chunks that cover a cell of the grid lattice,
# which only shadow and secondary rays reach.

def _partition(w, yaw_deg, offscreen=True, grid_dim=None, pos=(128.5, 110.0, 128.5)):
    cam = Camera(pos=pos, yaw=math.radians(yaw_deg), pitch=math.radians(-14.0), width=1280, height=720,
                 offscreen_shadows=offscreen, grid_dim=grid_dim)
    v = w.view(cam)
    keys = [(int(c["origin"][0]) // 64, int(c["origin"][1]) // 64, int(c["origin"][2]) // 64, int(c["lod"]))
            for c in v.chunks]
    n_vis = int(v.frame.chunk_count)
    gd = grid_dim or (W.GRID_X, W.GRID_Y, W.GRID_Z)
    gmin = (math.floor(pos[0] / 64.0) - gd[0] // 2, 0, math.floor(pos[2] / 64.0) - gd[2] // 2)
    return keys[:n_vis], keys[n_vis:], gmin, gd


def _grid_span(key, gmin, gd):
    """mod.rs:93-107 for a chunk key (x, y, z, lod)"""
    span = 1 << key[3]
    lo = [max(key[i] * span - gmin[i], 0) for i in range(3)]
    hi = [min(key[i] * span - gmin[i] + span, gd[i]) for i in range(3)]
    return (lo, hi) if all(l < h for l, h in zip(lo, hi)) else None


@pytest.fixture(scope="module")
def small_world():
    return World.generate(W.recipe_small_terrain())


def test_the_grid_set_is_the_same_at_every_yaw(small_world):
    """shadow_grid.rs:78-103"""
    ref = None
    for gd in (None, (4, 2, 2)):
        ref = None
        for yaw in (0.0, 45.0, 90.0, 135.0, 180.0, 225.0, 265.0, 315.0):
            vis, off, gmin, g = _partition(small_world, yaw, grid_dim=gd)
            got = sorted(k for k in vis + off if _grid_span(k, gmin, g))
            if ref is None:
                ref = got
            assert got == ref, f"grid {g}: the grid-eligible set changed at yaw {yaw}"
        assert ref


def test_the_drawn_set_still_depends_on_the_yaw(small_world):
    """shadow_grid.rs:105-131"""
    seen = []
    for yaw in (0.0, 90.0, 180.0, 265.0):
        vis, off, _, _ = _partition(small_world, yaw)
        assert vis, f"nothing drawn at yaw {yaw}"
        assert off, f"nothing shadow-only at yaw {yaw}"
        seen.append(sorted(vis))
    assert any(a != b for a, b in zip(seen, seen[1:])), "the frustum cull is not running"


def test_the_control_leaves_exactly_the_frustum_culled_set(small_world):
    """shadow_grid.rs:133-149"""
    on_vis, on_off, _, _ = _partition(small_world, 265.0)
    off_vis, off_off, _, _ = _partition(small_world, 265.0, offscreen=False)
    assert not off_off, "the control left a shadow-only tail"
    assert on_off, "the feature added no shadow-only tail"
    assert on_vis == off_vis, "the control changed the drawn list"


def test_every_shadow_only_chunk_reaches_the_lattice(small_world):
    """shadow_grid.rs:151-165, on the full lattice and on one smaller than
    the world"""
    for gd in (None, (4, 2, 2)):
        _, off, gmin, g = _partition(small_world, 265.0, grid_dim=gd)
        for k in off:
            span = _grid_span(k, gmin, g)
            assert span is not None, f"{k} is in the tail and covers no grid cell"
            lo, hi = span
            assert all(0 <= l < h <= n for l, h, n in zip(lo, hi, g))
