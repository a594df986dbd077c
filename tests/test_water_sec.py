"""The engine's schedule of the water legs (water_sec, resolve.wgsl:1468-1535;
vm_water_sec): one refract and one reflect leg per 2x2 pixel block (its
water pixel nearest the camera), WATER_SEC_SHIFT = 1, kept as a parity mode
beside the per-hit legs.

CPU: the oracle picks the nearest water pixel of each block (ties to the
first in x-major order) and its refract leg is that pixel's per-hit refract
leg; blocks without water have none.  GPU: vm_water_sec equals the oracle
(bit for bit for flat water and default waves; with a positive reflect
slope at most 0.5% of the reflect legs differ), at shifts 0, 1 and 2."""
import numpy as np
import pytest

from oracle.oracle import Oracle
from voxelcraft_menu_b200 import world as W

FLAGS = W.FLAG_SHADOWS | W.FLAG_WATER_REFRACT | W.FLAG_WATER_REFLECT
WAVES = W.FLAG_WAVES | 1024 | 2048 | 4096


@pytest.fixture(scope="module")
def small():
    w = W.World.generate(W.recipe_small_terrain())
    return w, w.pools()


def test_blocks_take_their_nearest_water_pixel(small):
    w, pools = small
    v = w.view(W.small_terrain_camera(flags=FLAGS, width=320, height=180))
    o = Oracle(v, *pools)
    vis, _, _ = o.frame_vis()
    sk, st = o.secondary(vis)
    rk, rt, mk, mt = o.water_sec(vis, 1)
    assert rk.shape == (90, 160)
    # a block's refract leg is the per-hit refract leg of one of its water pixels
    sk2, st2 = sk.reshape(90, 2, 160, 2), st.reshape(90, 2, 160, 2)
    water = ((sk >> np.uint64(63)) & np.uint64(1) == 1) & ((sk >> np.uint64(61)) & np.uint64(1) == 0)
    wblk = water.reshape(90, 2, 160, 2).any(axis=(1, 3))
    assert ((rk != 0) == wblk).all()
    match = (sk2 == rk[:, None, :, None]) & (st2 == rt[:, None, :, None])
    assert match.any(axis=(1, 3))[wblk].all()
    # shift 0: every water pixel is its own block
    rk0, rt0, _, _ = o.water_sec(vis, 0)
    wk = np.where(water, sk, 0).reshape(180, 320)
    assert np.array_equal(rk0, wk)
    assert (mk != 0).sum() > 1000


@pytest.mark.gpu
@pytest.mark.parametrize("shift", [0, 1, 2])
@pytest.mark.parametrize("waves", ["flat", "waves", "slope"])
def test_gpu_water_sec_matches_oracle(small, shift, waves):
    from voxelcraft_menu_b200.march import Marcher
    w, pools = small
    v = w.view(W.small_terrain_camera(flags=FLAGS | (0 if waves == "flat" else WAVES), width=333, height=187))
    if waves == "slope":
        v.frame.wave_reflect_slope, v.frame.time = 0.35, 1.7
    m = Marcher(333, 187)
    m.upload_world(*pools)
    m.upload_view(v)
    m.render()
    vis = m.read_vis()
    m.water_sec(shift)
    got = m.read_water_sec()
    m.close()
    want = Oracle(v, *pools).water_sec(vis, shift)
    assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1]), "refract legs"
    if waves == "slope":
        assert np.array_equal(got[2] != 0, want[2] != 0)
        assert (got[2] != want[2]).sum() <= 0.005 * max((want[2] != 0).sum(), 1), "reflect legs"
    else:
        assert np.array_equal(got[2], want[2]) and np.array_equal(got[3], want[3]), "reflect legs"
    assert (want[0] != 0).sum() > 100
