"""Pins of the oracle itself: the reference's key / predicate fixtures
(tests/cutout.rs, tests/waterline.rs, tests/physics.rs), known answers on
hand-built chunks, and a cross-check of the hierarchical march against a
unit-voxel DDA (the engine's Player::pick, src/player.rs:334-393)."""
import math

import numpy as np
import pytest

from oracle.oracle import Oracle, leaf_solid
from voxelcraft_menu_b200 import world as W
from voxelcraft_menu_b200.world import Camera, Recipe, World, dense_index


def cube(f):
    x, y, z = np.meshgrid(np.arange(64), np.arange(64), np.arange(64), indexing="ij")
    d = np.zeros(64 ** 3, np.uint16)
    d[dense_index(x, y, z).ravel()] = f(x, y, z).astype(np.uint16).ravel()
    return d


def one_chunk_oracle(dense, cam_pos=(32.5, 50.0, 32.5), flags=W.FLAG_SHADOWS | W.FLAG_WATER_REFRACT):
    w = World()
    w.insert_dense((0, 0, 0), dense)
    v = w.view(Camera(pos=cam_pos, width=64, height=64, flags=flags, grid_min=(-1, 0, -1), grid_dim=(3, 2, 3)))
    return w, v, Oracle(v, *w.pools())


# ---- key packing: tests/cutout.rs:15-60 ----------------------------------
def test_micro_bits_fit_the_key_and_round_trip():
    w, v, o = one_chunk_oracle(cube(lambda x, y, z: y < 5))
    for vx in ([0, 0, 0], [63, 63, 63], [1, 62, 33], [63, 0, 7]):
        for m in ([0, 0, 0], [3, 3, 3], [1, 2, 3], [0, 3, 1]):
            k = o.make_key(10.0, 3, 5, vx, m)
            low = k & 0xFFFFFF
            b = [(low >> 16) & 0xFF, (low >> 8) & 0xFF, low & 0xFF]
            assert [c & 63 for c in b] == vx
            assert [c >> 6 for c in b] == m
            assert (k >> 24) & 0x1FFF == 5 and (k >> 37) & 7 == 3
            assert k >> 40 == o.depth_key(10.0)
    for vx in ([0, 0, 0], [63, 63, 63], [12, 5, 40]):
        assert o.make_key(0.0, 0, 0, vx, [0, 0, 0]) & 0xFFFFFF == (vx[0] << 16) | (vx[1] << 8) | vx[2]


def test_depth_key_is_monotone_and_24_bits():
    w, v, o = one_chunk_oracle(cube(lambda x, y, z: y < 5))
    far = v.frame.far
    assert o.depth_key(0.0) == 16777215
    assert o.depth_key(far) == 0
    assert o.depth_key(2 * far) == 0
    ts = np.linspace(0, far, 257, dtype=np.float32)
    ks = [o.depth_key(float(t)) for t in ts]
    assert all(a >= b for a, b in zip(ks, ks[1:]))


# ---- water-line skip: tests/waterline.rs:3-99 ------------------------------
def predicate_v2(wl, ly, rd):
    """the skip formula of common.wgsl:721-735 as tests/waterline.rs:7-17 states it"""
    dx, dy, dz = rd
    if wl >= 15 or float(ly) <= float(wl):
        return False
    if dy >= 0.0:
        return True
    h = max(abs(dx), abs(dz))
    return h > 1e-6 and (ly - wl) > 16.0 * (abs(dy) / h)


def test_waterline_degenerate_rays():
    """tests/waterline.rs:85-99"""
    assert not predicate_v2(8, 15, (0.0, -1.0, 0.0))
    assert predicate_v2(8, 15, (0.9, 0.0, 0.44))
    assert predicate_v2(8, 15, (0.2, 0.8, 0.1))
    s9, c9 = math.sin(math.radians(9)), math.cos(math.radians(9))
    assert not predicate_v2(8, 10, (c9, -s9, 0.0))
    assert predicate_v2(8, 11, (c9, -s9, 0.0))


def test_water_line_skip_never_dives_through_the_land():
    """A water-blind (shadow) ray descending over a submerged slab must stop on
    the slab, whatever its slope: the oracle's march against a unit DDA that
    treats water as empty (the property tests/waterline.rs:29-59 states).

    The engine's predicate treats the line's own voxel layer as above the land
    (`ly - drop > wl` while that layer spans [wl, wl+1)), so a skipped 16^3
    cell may let a grazing ray cross the slab's top voxel layer unseen.  What
    it guarantees, and what is pinned here: a ray that reaches below the top
    layer is stopped no later than there, and no hit comes before the true
    first contact."""
    wl = 8  # land top inside the bottom L1 band
    d = cube(lambda x, y, z: np.where(y <= wl, W.STONE, np.where(y <= 40, W.WATER, W.AIR)))
    w, v, o = one_chunk_oracle(d)
    hits = late = 0
    for e10 in range(5, 800, 7):
        elev = math.radians(e10 / 10.0)
        for start_y in (10.5, 12.5, 15.5, 20.5, 30.5):
            rd = np.array([math.cos(elev), -math.sin(elev), 0.013], np.float32)
            rd /= np.float32(np.sqrt(np.float32((rd * rd).sum())))
            ro = np.array([0.25, start_y, 31.5], np.float32)
            h = o.march_chunk(0, ro, rd, 1000.0, skip_water=True, skip_glass=True, sun_ray=True)
            # ground truth: first non-water solid along the ray (fine sampling)
            ts = np.arange(0, 200, 0.002, dtype=np.float64)
            p = ro[None, :].astype(np.float64) + ts[:, None] * rd[None, :].astype(np.float64)
            inside = np.all((p >= 0) & (p < 64), axis=1)
            solid = inside & (np.floor(p[:, 1]) <= wl)
            deep = inside & (np.floor(p[:, 1]) <= wl - 1)
            if h.hit:
                assert solid.any() and h.t >= ts[np.argmax(solid)] - 0.01
                assert h.voxel[1] <= wl
            if deep.any():
                hits += 1
                assert h.hit, f"elev {e10/10} y {start_y}: passed below the slab's top layer"
                assert h.t <= ts[np.argmax(deep)] + 0.01
                late += h.t > ts[np.argmax(solid)] + 0.01
    assert hits > 100
    assert late < hits // 2


# ---- known answers ---------------------------------------------------------
FLOOR = 20


def test_looking_down_at_the_floor_finds_its_top_face():
    """tests/physics.rs:239-252 on the march: straight down onto a floor."""
    d = cube(lambda x, y, z: np.where(y < FLOOR, W.STONE, W.AIR))
    w, v, o = one_chunk_oracle(d)
    eye = FLOOR + 2.0 + 1.62
    fwd = np.array([0.0, -1.0, 1e-3], np.float32)
    h = o.march_chunk(0, [32.5, eye, 32.5], fwd, 2600.0)
    assert h.hit and list(h.voxel) == [32, FLOOR - 1, 32]
    assert h.normal == 3, "top face of the block below (+Y)"
    assert abs(h.t - (eye - FLOOR)) < 1e-4
    pick = o.pick([32.5, eye, 32.5], fwd, 64, 5.0)
    assert pick is not None and pick[0] == (32, FLOOR - 1, 32) and pick[1] == (0, 1, 0)


@pytest.mark.parametrize("axis", range(6))
def test_axis_rays_hit_the_expected_face(axis):
    """Rays along each axis into a solid box report the entered face."""
    d = cube(lambda x, y, z: (x >= 20) & (x < 40) & (y >= 20) & (y < 40) & (z >= 20) & (z < 40))
    w, v, o = one_chunk_oracle(d)
    a, sgn = axis >> 1, (1 if axis & 1 else -1)
    ro = np.array([30.5, 30.5, 30.5], np.float32)
    ro[a] = 30.5 - sgn * 25.0          # outside the box, looking back at it
    rd = np.full(3, 1e-6, np.float32)
    rd[a] = sgn
    h = o.march_chunk(0, ro, rd, 2600.0)
    want_face = a * 2 + (0 if sgn > 0 else 1)
    assert h.hit and h.normal == want_face
    assert h.voxel[a] == (20 if sgn > 0 else 39)
    assert abs(h.t - (15.0 - 0.5 * sgn)) < 1e-4   # faces at 20 and 40, start 25 from the centre 30.5


def shadow_world(slab_id):
    return cube(lambda x, y, z: np.where(y < 10, W.STONE, np.where((y >= 20) & (y < 22), slab_id, W.AIR)))


@pytest.mark.parametrize("slab,blocks", [(W.STONE, True), (W.GLASS, False), (W.WATER, False),
                                          (W.GLOWSTONE, False), (W.DIRT, True)])
def test_sun_ray_transparency(slab, blocks):
    """shadow_ray_t marches with skip_water / skip_glass / sun_ray: water and
    glass are transparent and emitters cast no shadow (common.wgsl:624-668)."""
    w, v, o = one_chunk_oracle(shadow_world(slab))
    sun = np.array(W.default_sun(), np.float32)
    t = o.shadow_ray_t([30.5, 10.02, 30.5], sun, 220.0)
    if blocks:
        assert t > 0 and abs(t - (20 - 10.02) / sun[1]) < 0.1
    else:
        assert t == -1.0


def test_primary_rays_see_glass_and_water_surfaces():
    for slab in (W.GLASS, W.WATER):
        w, v, o = one_chunk_oracle(shadow_world(slab))
        h = o.march_chunk(0, [30.5, 40.0, 30.5], [1e-6, -1.0, 1e-6], 2600.0)
        assert h.hit and h.voxel[1] == 21 and h.normal == 3


def test_water_interface_inside_water_is_not_a_surface():
    """A primary ray that starts inside a water body only stops at the first
    water face that borders non-water (world_block_at repair,
    common.wgsl:800-813): here the sea floor."""
    d = cube(lambda x, y, z: np.where(y < 10, W.STONE, np.where(y < 40, W.WATER, W.AIR)))
    w, v, o = one_chunk_oracle(d, cam_pos=(30.5, 50.0, 30.5))
    h = o.march_chunk(0, [30.5, 30.5, 30.5], [0.3, -0.9, 0.3], 2600.0)
    assert h.hit and h.voxel[1] == 9, "the water cells around the start are interior"


def test_leaf_cutout_hits_land_on_solid_micro_cells():
    """cutout_march (common.wgsl:537-577): a leaf hit's micro cell is filled
    per leaf_solid's hash; misses pass through the leaf voxel."""
    d = cube(lambda x, y, z: np.where((y >= 20) & (y < 24), W.LEAVES, W.AIR))
    w, v, o = one_chunk_oracle(d)
    rng = np.random.default_rng(5)
    n_hit = 0
    for _ in range(300):
        ro = np.array([rng.uniform(5, 59), 40.0, rng.uniform(5, 59)], np.float32)
        rd = np.array([rng.uniform(-0.3, 0.3), -1.0, rng.uniform(-0.3, 0.3)], np.float32)
        rd /= np.float32(np.sqrt(np.float32((rd * rd).sum())))
        h = o.march_chunk(0, ro, rd, 2600.0)
        if h.hit:
            n_hit += 1
            assert leaf_solid(list(h.voxel), list(h.micro))
            assert 20 <= h.voxel[1] < 24
    assert n_hit > 250


def test_hierarchical_march_equals_unit_dda_on_opaque_worlds():
    """trace_world (common.wgsl:1205) through the 64-tree vs a unit-voxel walk
    over block lookups (src/player.rs:334-393) on an opaque world: same first
    voxel and entry face."""
    rec = Recipe(size=(256, 128, 256), water_level=-1, tree_permille=0)
    w = World.generate(rec)
    v = w.view(W.small_terrain_camera())
    o = Oracle(v, *w.pools())
    rng = np.random.default_rng(1)
    checked = agree = 0
    for _ in range(1500):
        ro = np.array([rng.uniform(10, 246), rng.uniform(90, 126), rng.uniform(10, 246)], np.float32)
        rd = rng.normal(size=3).astype(np.float32)
        rd[1] = -abs(rd[1]) - 0.05
        rd /= np.float32(np.sqrt(np.float32((rd * rd).sum())))
        hit, t, normal, vox, ci = o.trace_world(ro, rd, 150.0, False)
        p = o.pick(ro, rd, 4000, 150.0)
        if not hit and p is None:
            continue
        checked += 1
        assert hit and p is not None, "one side found a voxel the other missed"
        c = v.chunks[ci]
        world_vox = tuple(int(c["origin"][i]) + vox[i] for i in range(3))
        axis = normal >> 1
        sign = 1 if normal & 1 else -1
        nvec = [0, 0, 0]
        nvec[axis] = sign
        if world_vox == p[0] and tuple(nvec) == p[1]:
            agree += 1
        assert abs(t - p[2]) < 1e-3
    assert checked > 800
    assert agree >= checked - 2, f"{checked - agree} rays disagree"


def test_hiz_does_not_change_the_visibility():
    """The two-phase Hi-Z (tile_select.wgsl:79-86, march.wgsl:57-76,
    tile_select.wgsl:94-110) only culls pairs that cannot win the atomicMax."""
    w = World.generate(W.recipe_small_terrain())
    inn, lea, bri = w.pools()
    v0 = w.view(W.small_terrain_camera(flags=W.FLAG_SHADOWS))
    vis0, hiz0, c0 = Oracle(v0, inn, lea, bri).frame_vis()
    v1 = w.view(W.small_terrain_camera(flags=W.FLAG_SHADOWS | W.FLAG_HIZ))
    o1 = Oracle(v1, inn, lea, bri)
    visA, hizA, cA = o1.frame_vis(hiz_in=np.zeros(o1.ntiles, np.uint32))
    visB, hizB, cB = o1.frame_vis(hiz_in=hizA)
    assert np.array_equal(vis0, visA) and np.array_equal(vis0, visB)
    assert cB[1] > 0, "the second frame defers pairs"
    assert cB[5] <= cB[1]


# ---- the underwater reach: tests/submerged.rs --------------------------------
# The engine pins tile_select's reach (tile_select.wgsl:116-133) by reading its
# shader source; here the same properties are checked on the oracle's per-tile
# chunk lists (or_tile_pairs): the reach applies only when both
# FLAG_UNDERWATER and FLAG_WATER_FAR are set, it is decided by where the
# tile's most upward corner ray leaves the water (frame.sea_level), and the
# cull compares each chunk's box distance with it.

def _tile_lists(flags, pos=(128.5, 62.0, 2.5), pitch=0.0):
    w = World.generate(W.recipe_small_terrain())
    v = w.view(Camera(pos=pos, pitch=math.radians(pitch), width=320, height=200, flags=flags))
    v.frame.flags = flags          # exactly these flags, whatever the camera's medium
    o = Oracle(v, *w.pools())
    f = v.frame
    return v, o, {t: o.tile_pairs(t)[0] for t in range(int(f.tiles[0]) * int(f.tiles[1]))}


def _box_distance(p, c):
    lo, hi = np.asarray(c["aabb_min"], np.float64), np.asarray(c["aabb_max"], np.float64)
    d = np.maximum(np.maximum(lo - p, 0.0), p - hi)
    return float(np.sqrt((d * d).sum()))


def test_reach_needs_both_flags():
    """submerged.rs: FLAG_WATER_FAR alone would clamp a dry camera; the
    reach tests both flags in one expression."""
    base = W.FLAG_SHADOWS
    _, _, ref = _tile_lists(base)
    for extra in (W.FLAG_WATER_FAR, W.FLAG_UNDERWATER):
        _, _, got = _tile_lists(base | extra)
        assert all(np.array_equal(got[t], ref[t]) for t in ref), f"flag {extra} alone changed the tile lists"


def test_reach_culls_by_box_distance_below_the_water_only():
    """submerged.rs: the cull reads the per-tile reach (dmin >= reach), and
    the reach follows the water path: tiles whose corner rays all point down
    never leave the water and lose every chunk at WATER_FAR_DIST or beyond;
    tiles whose most upward corner ray reaches sea_level within that
    distance keep the full view distance."""
    base = W.FLAG_SHADOWS
    v, o, ref = _tile_lists(base)
    _, _, got = _tile_lists(base | W.FLAG_UNDERWATER | W.FLAG_WATER_FAR)
    cam = np.asarray(v.frame.cam_pos, np.float64)
    tx, ty = int(v.frame.tiles[0]), int(v.frame.tiles[1])
    dropped_any = False
    for t in ref:
        kept = set(got[t].tolist())
        assert kept <= set(ref[t].tolist())
        row = t // tx
        for ci in set(ref[t].tolist()) - kept:
            dropped_any = True
            assert row > ty // 2, f"tile {t} (an upward row) lost chunk {ci}"
            assert _box_distance(cam, v.chunks[ci]) >= 128.0 - 1e-3
        if row > ty // 2 + 1:                 # corner rays all below the horizon: reach 128
            for ci in kept:
                assert _box_distance(cam, v.chunks[ci]) < 128.0 + 1e-3 or ci == v.frame.camera_chunk
        if row < ty // 2 - 1:                 # upward rows: sea level within 2 / up < 128
            assert np.array_equal(got[t], ref[t])
    assert dropped_any, "the camera sees chunks beyond the reach"


def test_water_far_dist_is_shorter_than_the_view_distance():
    """submerged.rs: 128 <= WATER_FAR_DIST < the default view distance
    (2600, src/lod.rs:44)."""
    from pathlib import Path
    import re
    src = (Path(__file__).resolve().parents[1] / "voxelcraft_menu_b200" / "csrc" / "vm_types.h").read_text()
    reach = float(re.search(r"#define VM_WATER_FAR_DIST ([0-9.]+)f", src).group(1))
    assert 128.0 <= reach < 2600.0
