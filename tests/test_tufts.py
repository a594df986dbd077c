"""Foliage tufts (TALL_GRASS, GRASS_TALL, REEDS): the cross quads of
cross_quad (common.wgsl:425-487), alpha-tested against the atlas at the ray's
texture level, traced by every march whose skip_foliage is off (the primary
march and trace_world's water / glass legs) and transparent to sun rays.

CPU: the recipe's tufts, the oracle without an atlas (tufts transparent: the
march equals the same world's with the tufts removed), and with one (hits on
the cross normals inside the tuft voxels).  GPU: the wavefront pipeline, the
engine pass sequence and the batch equal the oracle bit for bit; with wind
sway (whose shear is a sum of sines) within 0.5% of the pixels, all of them
cross-quad hits on one side; without an atlas tufts stay transparent."""
import math

import numpy as np
import pytest

from oracle.oracle import SPEC_DEFAULT, Oracle, engine_atlas
from voxelcraft_menu_b200 import look as LK
from voxelcraft_menu_b200 import world as W

SPEC_WIND_SWAY = 512
TUFTS = (18, 24, 25)


def tuft_recipe():
    r = W.recipe_small_terrain()
    r.tuft_permille = 300
    return r


@pytest.fixture(scope="module")
def tufted():
    rec = tuft_recipe()
    w = W.World.generate(rec)
    plain = W.recipe_small_terrain()
    w0 = W.World.generate(plain)
    return rec, w, w.pools(), w0, w0.pools()


def low_camera(width=320, height=180, **kw):
    # close over a dry meadow, looking along the ground
    return W.Camera(pos=(150.0, 92.0, 60.0), yaw=math.radians(60.0), pitch=math.radians(-12.0), width=width,
                    height=height, **kw)


def key_normals(vis):
    return (vis >> np.uint64(37)) & np.uint64(7)


def test_recipe_places_tufts_on_dry_grass(tufted):
    rec, w, _, w0, _ = tufted
    n = 0
    for x in range(0, 256, 3):
        for z in range(0, 256, 3):
            h = W.surface_height(rec, x, z)
            b = w.get_block(x, h, z)
            if b in TUFTS:
                n += 1
                assert w.get_block(x, h - 1, z) == 3          # on grass
                assert h - 1 >= rec.water_level               # dry
            assert w0.get_block(x, h, z) not in TUFTS
    assert n > 100


def test_oracle_without_an_atlas_sees_through_tufts(tufted):
    rec, w, pools, w0, pools0 = tufted
    cam = low_camera()
    v, v0 = w.view(cam), w0.view(cam)
    vis = Oracle(v, *pools).frame_vis()[0]
    vis0 = Oracle(v0, *pools0).frame_vis()[0]
    assert np.array_equal(vis, vis0)
    assert not (key_normals(vis) >= 6).any()


def test_oracle_with_an_atlas_hits_cross_quads(tufted):
    rec, w, pools, _, _ = tufted
    v = w.view(low_camera())
    o = Oracle(v, *pools, atlas=LK.atlas(1), faces=LK.block_faces())
    vis = o.frame_vis()[0]
    cross = key_normals(vis) >= 6
    assert cross.sum() > 200
    # a cross hit's voxel holds a tuft, its t lies inside that voxel's box
    for p in np.flatnonzero(cross)[::97]:
        k = int(vis[p])
        ci, vx, vy, vz = (k >> 24) & 0x1FFF, (k >> 16) & 63, (k >> 8) & 63, k & 63
        assert o.block_at(ci, [vx, vy, vz]) in TUFTS
    # sun rays pass through tufts: the shadow is the one of the world without an atlas
    o0 = Oracle(v, *pools)
    vis0 = o0.frame_vis()[0]
    keep = ~cross & (vis == vis0)
    assert np.array_equal(o.shadow(vis)[keep], o0.shadow(vis0)[keep])


@pytest.mark.gpu
@pytest.mark.parametrize("spec,source", [(SPEC_DEFAULT, "library"), (SPEC_DEFAULT, "engine"),
                                         (SPEC_DEFAULT | SPEC_WIND_SWAY, "engine")])
def test_tufts_match_the_oracle(tufted, spec, source):
    from voxelcraft_menu_b200.march import Marcher
    rec, w, pools, _, _ = tufted
    atlas, faces = (engine_atlas() if source == "engine" else LK.atlas(1)), LK.block_faces()
    v = w.view(low_camera(480, 270, flags=W.FLAG_SHADOWS | W.FLAG_WATER_REFRACT))
    v.frame.time, v.frame.cloud_speed = 12.5, 3.0
    o = Oracle(v, *pools, spec=spec, atlas=atlas, faces=faces)
    vis, _, _ = o.frame_vis()
    sh = o.shadow(vis)
    sk, st = o.secondary(vis)
    assert (key_normals(vis) >= 6).sum() > 300
    m = Marcher(480, 270)
    try:
        m.set_spec(spec)
        m.upload_world(*pools)
        m.upload_view(v)
        m.upload_look(atlas, faces)
        def check(gv, gs, what):
            if not sway:
                assert np.array_equal(gv, vis), what
                assert np.array_equal(gs, sh), what
                return
            # the sway shear comes from sinf (CUDA's against the host's): a
            # last-bit difference can move a quad edge across a pixel
            diff = gv != vis
            assert diff.mean() < 0.005, f"{what}: {diff.sum()} pixels differ"
            assert ((key_normals(gv[diff]) >= 6) | (key_normals(vis[diff]) >= 6)).all(), what
            assert np.array_equal(gs[~diff], sh[~diff]), what

        sway = (spec & SPEC_WIND_SWAY) != 0
        m.render()
        check(m.read_vis(), m.read_shadow(), "pipeline")
        if not sway:
            gk, gt = m.read_secondary()
            assert np.array_equal(gk, sk) and np.array_equal(gt, st)
        m.render_passes()
        check(m.read_vis(), m.read_shadow(), "engine passes")
        m.batch_set([v, w.view(low_camera(96, 96))])
        m.batch_run()
        bv, bs = m.batch_read()
        check(bv[:v.n_pixels], bs[:v.n_pixels], "batch")
        assert m.stats().device_error == 0
    finally:
        m.close()


@pytest.mark.gpu
def test_tufts_without_an_atlas_are_transparent(tufted):
    from voxelcraft_menu_b200.march import Marcher
    rec, w, pools, w0, pools0 = tufted
    v = w.view(low_camera(320, 180))
    m = Marcher(320, 180)
    try:
        m.upload_world(*pools)
        m.upload_view(v)
        m.render()
        vis = m.read_vis()
    finally:
        m.close()
    assert np.array_equal(vis, Oracle(w0.view(low_camera(320, 180)), *pools0).frame_vis()[0])
