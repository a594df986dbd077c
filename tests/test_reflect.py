"""The reflect leg of water hits (water_reflect_leg, resolve.wgsl:1044-1058).

CPU: the oracle traces one reflect ray per water hit closer than 1024 voxels
when FLAG_WATER_REFLECT is set, none for other blocks and none without the
flag; a ray that leaves a +Y water face rises (a hit above the surface, or
the 768-voxel distance).  On waved surfaces (FLAG_WAVES on +Y faces) the leg
follows water_ctx's mirror_t: with the engine's default wave_reflect_slope of
0 it is the flat surface's, with a positive slope the wave normal's.
GPU: the reflect keys and distances of the wavefront pipeline and of the
engine pass sequence equal the oracle's bit for bit (flat and default waves;
with a positive reflect slope, whose wave field runs through cos and exp,
at most 0.5% of the legs may differ); the flag leaves the frame's other
outputs unchanged."""
import numpy as np
import pytest

from oracle.oracle import Oracle
from voxelcraft_menu_b200 import world as W

REFL = W.FLAG_SHADOWS | W.FLAG_WATER_REFRACT | W.FLAG_WATER_REFLECT
WAVE_OPTS = 1024 | 2048 | 4096        # FLAG_WAVE_ANISO | FLAG_WAVE_SHOAL | FLAG_WAVE_FILL


@pytest.fixture(scope="module")
def small():
    w = W.World.generate(W.recipe_small_terrain())
    return w, w.pools()


def water_pixels(o, vis):
    ids = np.array([o.block_at(int(k >> 24) & 0x1FFF, [int(k >> 16) & 63, int(k >> 8) & 63, int(k) & 63])
                    if k else 0 for k in vis], np.uint32)
    return ids == W.WATER


def test_oracle_reflect_rays(small):
    w, pools = small
    v = w.view(W.small_terrain_camera(flags=REFL))
    o = Oracle(v, *pools)
    vis, _, _ = o.frame_vis()
    k, t = o.reflection(vis)
    water = water_pixels(o, vis)
    traced = (k >> np.uint64(63)) & np.uint64(1) == 1
    assert water.sum() > 1000
    assert traced.sum() > 0.9 * water.sum()          # water within 1024 voxels: all of this view's
    assert not traced[~water].any()
    assert (k[~traced] == 0).all() and (t[~traced] == 0).all()
    hit = (k >> np.uint64(62)) & np.uint64(1) == 1
    assert ((t[traced & ~hit] == 768.0)).all() and (t[traced & hit] < 768.0).all()
    nid = (vis >> np.uint64(37)) & np.uint64(7)
    assert (nid[traced] == 3).mean() > 0.5          # mostly the lakes' +Y faces
    # without the flag, nothing; with waves, no +Y face is traced
    v2 = w.view(W.small_terrain_camera(flags=W.FLAG_SHADOWS | W.FLAG_WATER_REFRACT))
    k2, _ = Oracle(v2, *pools).reflection(vis)
    assert (k2 == 0).all()
    # waves at the default reflect slope 0: the flat legs; a positive slope
    # moves some +Y legs and no other face's
    waves = W.FLAG_WAVES | WAVE_OPTS
    v3 = w.view(W.small_terrain_camera(flags=REFL | waves))
    k3, t3 = Oracle(v3, *pools).reflection(vis)
    # the waved direction is renormalised (normalize(x, max(y, 0), z)): the
    # same voxels, distances within float rounding
    assert np.array_equal(k3, k) and np.allclose(t3, t, rtol=1e-5, atol=0.0)
    v3.frame.wave_reflect_slope, v3.frame.time = 0.35, 1.7
    k4, t4 = Oracle(v3, *pools).reflection(vis)
    py = nid == 3
    assert np.array_equal(k4[~py], k[~py])
    assert (k4[py] != k[py]).sum() > 100
    assert ((k4 >> np.uint64(63)) & np.uint64(1) == 1)[py & water].all()


@pytest.mark.gpu
@pytest.mark.parametrize("waves", ["flat", "waves", "waves_all", "slope"])
def test_gpu_reflect_matches_oracle(small, waves):
    from voxelcraft_menu_b200.march import Marcher
    w, pools = small
    flags = REFL | {"flat": 0, "waves": W.FLAG_WAVES, "waves_all": W.FLAG_WAVES | WAVE_OPTS,
                    "slope": W.FLAG_WAVES | WAVE_OPTS}[waves]
    v = w.view(W.small_terrain_camera(flags=flags))
    if waves == "slope":
        v.frame.wave_reflect_slope, v.frame.time = 0.35, 1.7
    o = Oracle(v, *pools)
    ovis, _, _ = o.frame_vis()
    ok, ot = o.reflection(ovis)
    m = Marcher(640, 360, device=0)
    try:
        m.upload_world(*pools)
        m.upload_view(v)
        for run in (m.render, m.render_passes):
            run()
            assert np.array_equal(m.read_vis(), ovis)
            k, t = m.read_reflection()
            if waves == "slope":
                traced = ((ok >> np.uint64(63)) & np.uint64(1)).sum()
                assert np.array_equal(k != 0, ok != 0), "the same pixels trace a leg"
                assert (k != ok).sum() <= 0.005 * traced, f"{run.__name__}: {(k != ok).sum()} of {traced} differ"
            else:
                assert np.array_equal(k, ok), f"{run.__name__}: {(k != ok).sum()} reflect keys differ"
                assert np.array_equal(t, ot), f"{run.__name__}: reflect t differs"
            assert m.stats().device_error == 0
        # the flag adds the reflect legs and changes nothing else
        vis, sh, (sk, st) = m.read_vis(), m.read_shadow(), m.read_secondary()
        v0 = w.view(W.small_terrain_camera(flags=flags & ~W.FLAG_WATER_REFLECT))
        v0.frame.wave_reflect_slope, v0.frame.time = v.frame.wave_reflect_slope, v.frame.time
        m.upload_view(v0)
        m.render()
        assert np.array_equal(m.read_vis(), vis) and np.array_equal(m.read_shadow(), sh)
        k0, t0 = m.read_secondary()
        assert np.array_equal(k0, sk) and np.array_equal(t0, st)
        with pytest.raises(RuntimeError):
            m.read_reflection()                      # the last frame had no FLAG_WATER_REFLECT
    finally:
        m.close()


@pytest.mark.gpu
def test_gpu_reflect_1080p_large_terrain():
    from voxelcraft_menu_b200.march import Marcher
    rec = W.recipe_large_terrain()
    w = W.World.generate(rec)
    pools = w.pools()
    v = w.view(W.large_terrain_camera(rec, flags=REFL))
    m = Marcher(1920, 1080, device=0)
    try:
        m.upload_world(*pools)
        m.upload_view(v)
        m.render()
        vis = m.read_vis()
        k, t = m.read_reflection()
    finally:
        m.close()
    o = Oracle(v, *pools)
    ok, ot = o.reflection(vis)
    assert np.array_equal(k, ok) and np.array_equal(t, ot)
    assert ((k >> np.uint64(63)) & np.uint64(1)).sum() > 10000
