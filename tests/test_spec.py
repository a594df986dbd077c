"""The engine's pipeline specialisations of the march (make_spec,
src/render/mod.rs:2355-2689; VM_SPEC_* bits, vm_set_spec).

The world is the 256x128x256 terrain with one chunk rebuilt to carry
glowstone pillars (emitters: SPEC_EMITTER_GATHER), glass pillars (SPEC_GLASS)
and tall-grass tufts (SPEC_FOLIAGE) on its surface; its trees exercise the leaf cutout and fill, its
y = 0 chunks have full roots (SPEC_FULL_MARCH) and, from an underwater
camera, its water the Snell bend.  One water chunk cross-fades (fade 0.5), so
where the dither skips it the next chunk's march starts inside water: the
water-interface repair (SPEC_WATER_REPAIR) decides those pixels.  CPU: each non-default setting
changes the oracle's frame.  GPU: every setting equals the oracle through
vm_render and the engine passes."""
import math

import numpy as np
import pytest

from oracle import oracle as O
from oracle.oracle import Oracle
from voxelcraft_menu_b200 import world as W
from voxelcraft_menu_b200.world import Camera, World

KEY = (2, 1, 1)          # chunk cell whose blocks get emitters and tufts
FADED = (2, 0, 0)        # water chunk drawn with a dither
GLOWSTONE, TALL_GRASS, GLASS = 11, 18, 10

SPECS = {
    "default": O.SPEC_DEFAULT,
    "no_full_march": O.SPEC_DEFAULT & ~O.SPEC_FULL_MARCH,
    "no_full_march_legacy_water": O.SPEC_DEFAULT & ~(O.SPEC_FULL_MARCH | O.SPEC_WATER_REPAIR),
    "legacy_water": O.SPEC_DEFAULT & ~O.SPEC_WATER_REPAIR,
    "no_leaf_cutout": O.SPEC_DEFAULT & ~O.SPEC_LEAF_CUTOUT,
    "no_glass": O.SPEC_DEFAULT & ~O.SPEC_GLASS,
    "no_emitter_gather": O.SPEC_DEFAULT & ~O.SPEC_EMITTER_GATHER,
    "no_foliage": O.SPEC_DEFAULT & ~O.SPEC_FOLIAGE,
    "no_leaf_thin": O.SPEC_DEFAULT & ~O.SPEC_LEAF_THIN,
    "snell_bend": O.SPEC_DEFAULT | O.SPEC_SNELL_BEND,
}


def special_chunk(rec):
    """The recipe's chunk KEY with glowstone pillars and a meadow of tufts on
    its dry surface columns (dense index x | z<<6 | y<<12)."""
    d = W.layout_dense(rec, 0, KEY).reshape(64, 64, 64)        # [y, z, x]
    air = d == W.AIR
    below_solid = np.zeros_like(air)
    below_solid[1:] = (d[:-1] != W.AIR) & (d[:-1] != W.WATER)
    surface = air & below_solid                                 # first air block above dry ground
    ys, zs, xs = np.nonzero(surface)
    rng = np.random.default_rng(7)
    pick = rng.random(ys.size)
    tufts = pick < 0.35
    d[ys[tufts], zs[tufts], xs[tufts]] = TALL_GRASS
    for y, z, x in zip(ys[pick > 0.985], zs[pick > 0.985], xs[pick > 0.985]):
        d[y:min(y + 4, 64), z, x] = GLOWSTONE
    for y, z, x in zip(ys[(pick > 0.95) & (pick < 0.97)], zs[(pick > 0.95) & (pick < 0.97)],
                       xs[(pick > 0.95) & (pick < 0.97)]):
        d[y:min(y + 3, 64), z, x] = GLASS
    return d.reshape(-1)


@pytest.fixture(scope="module")
def world():
    rec = W.recipe_small_terrain()
    w = World.generate(rec)
    d = special_chunk(rec)
    w.insert_dense(KEY, d)
    w.set_fade(FADED, 0.5)
    return w, w.pools()


def cam_over(**kw):
    c = dict(pos=(160.0, 100.0, 20.0), yaw=math.radians(90.0), pitch=math.radians(-25.0), width=320, height=180)
    c.update(kw)
    return Camera(**c)


def cam_under():
    rec = W.recipe_small_terrain()
    for x in range(0, 256, 8):
        if W.surface_height(rec, x, 128) < 56:
            break
    flags = W.FLAG_SHADOWS | W.FLAG_WATER_REFRACT | W.FLAG_UNDERWATER
    return Camera(pos=(x + 0.5, 61.5, 128.5), pitch=math.radians(25.0), width=320, height=180, flags=flags)


def oracle_frame(view, pools, spec):
    o = Oracle(view, *pools, spec=spec)
    vis, _, _ = o.frame_vis()
    sh = o.shadow(vis)
    sk, st = o.secondary(vis)
    return vis, sh, sk, st


def test_the_world_has_emitters_tufts_leaves_and_full_roots(world):
    w, pools = world
    v = w.view(cam_over())
    ch = v.chunks
    assert (ch["attr_flags"] & (1 << 5)).any(), "an emitter chunk"
    assert (ch["attr_flags"] & (1 << 2)).any(), "a foliage chunk"
    assert (ch["attr_flags"] & (1 << 3)).any(), "a cutout chunk"
    assert ((ch["root"][:, 2] & 0x80000000) != 0).any(), "a full root"


@pytest.mark.parametrize("name", [n for n in SPECS if n not in ("default", "snell_bend")])
def test_each_setting_changes_the_oracle_frame(world, name):
    w, pools = world
    v = w.view(cam_over())
    base = oracle_frame(v, pools, SPECS["default"])
    got = oracle_frame(v, pools, SPECS[name])
    assert any(not np.array_equal(a, b) for a, b in zip(base, got)), f"{name} changed nothing"


def test_snell_bend_changes_the_underwater_frame(world):
    w, pools = world
    v = w.view(cam_under())
    assert not np.array_equal(oracle_frame(v, pools, SPECS["default"])[0],
                              oracle_frame(v, pools, SPECS["snell_bend"])[0])


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(SPECS))
def test_setting_matches_the_oracle(world, name):
    from voxelcraft_menu_b200.march import Marcher
    w, pools = world
    spec = SPECS[name]
    m = Marcher(320, 180)
    m.upload_world(*pools)
    m.set_spec(spec)
    for cam in (cam_over(), cam_under()):
        v = w.view(cam)
        vis, sh, sk, st = oracle_frame(v, pools, spec)
        m.upload_view(v)
        for run in (m.render, m.render_passes):
            run()
            assert np.array_equal(m.read_vis(), vis), f"{name} {run.__name__}: vis"
            assert np.array_equal(m.read_shadow(), sh), f"{name} {run.__name__}: shadow"
            gk, gt = m.read_secondary()
            assert np.array_equal(gk, sk), f"{name} {run.__name__}: secondary key"
            assert np.array_equal(gt, st), f"{name} {run.__name__}: secondary t"
    m.close()


@pytest.mark.gpu
def test_unknown_spec_bits_are_rejected():
    from voxelcraft_menu_b200.march import MarchError, Marcher
    m = Marcher(64, 64)
    with pytest.raises(MarchError) as e:
        m.set_spec(1 << 12)
    assert e.value.code == 1
    m.close()
