"""The bilateral soft-shadow reconstruction (shadow_horizontal +
shadow_vertical, shadow.wgsl:49-116).

CPU: the oracle's binary16 storage rounding equals numpy's float16
conversion (round to nearest even) bit for bit; the oracle's filter leaves
the hard mask alone where the engine would (shadows inactive, no
penumbra wider than half a pixel, no compatible neighbours) and softens
the penumbrae of a low camera.  GPU: the fused kernel's mask matches the
oracle's within MASK_ATOL at every pixel, and within NEAR_ATOL at all
but a NEAR_FRACTION of them.  The two use different expf, so a weight may
differ in its last bits: a soft pixel's mask then differs by a few float
ulps and, rarely, a horizontal result rounds to the neighbouring binary16
value (2^-11 near 1), the largest difference this leaves in the mask."""
import math

import numpy as np
import pytest

from oracle.oracle import SPEC_DEFAULT, SPEC_SOFT_RAYS, Oracle, f16_round
from voxelcraft_menu_b200 import world as W

MASK_ATOL = 1e-3            # |GPU - oracle| at every pixel
NEAR_ATOL = 2e-6            # |GPU - oracle| at all pixels but ...
NEAR_FRACTION = 1e-3        # ... this fraction


@pytest.fixture(scope="module")
def small():
    w = W.World.generate(W.recipe_small_terrain())
    return w, w.pools()


def hard_mask(dist):
    return (1.0 - (f16_round(dist) > 0.0)).astype(np.float32)


# -- CPU: the oracle -----------------------------------------------------------

def test_f16_round_matches_numpy():
    rng = np.random.default_rng(5)
    x = (rng.standard_normal(100000) * 10.0 ** rng.integers(-9, 6, 100000)).astype(np.float32)
    edges = np.array([0.0, -0.0, 0.001, 65504.0, 65519.99, 65520.0, 1e5, 2.0 ** -24, 2.0 ** -25, 3 * 2.0 ** -25,
                      6.1e-5, 1.0 + 2.0 ** -11, 1.0 + 3 * 2.0 ** -11, np.inf, -np.inf], np.float32)
    bits = np.arange(0, 2 ** 32, 65537, dtype=np.uint64).astype(np.uint32).view(np.float32)
    x = np.concatenate([x, edges, bits])
    with np.errstate(over="ignore", invalid="ignore"):
        ref = x.astype(np.float16).astype(np.float32)
    got = f16_round(x)
    same = (got.view(np.uint32) == ref.view(np.uint32)) | (np.isnan(got) & np.isnan(ref))
    assert same.all(), x[~same][:8]


def test_oracle_inactive_shadows_give_the_hard_mask(small):
    w, pools = small
    v = w.view(W.penumbra_camera())
    o = Oracle(v, *pools)
    vis, _, _ = o.frame_vis()
    dist = o.shadow(vis)
    v.frame.daylight = 0.0          # shadow_active() false: both passes copy occ
    h, mask = Oracle(v, *pools).soften(vis, dist, 8, 3.0)
    assert np.array_equal(mask, hard_mask(dist))
    assert (h[:, 1] == 0).all()


def test_oracle_softens_penumbrae(small):
    w, pools = small
    v = w.view(W.penumbra_camera())
    o = Oracle(v, *pools)
    vis, _, _ = o.frame_vis()
    dist = o.shadow(vis)
    hard = hard_mask(dist)
    for limit, pen in ((4, 1.5), (8, 3.0)):
        h, mask = o.soften(vis, dist, limit, pen)
        assert ((mask >= 0) & (mask <= 1)).all()
        soft = (mask > 0) & (mask < 1)
        assert soft.sum() > 500
        assert (h[:, 1] <= limit).all()
        sky = vis == 0                             # no guide: the hard value
        assert np.array_equal(mask[sky], hard[sky])
        changed = mask != hard
        assert changed.any() and (np.abs(mask - hard)[changed] <= 1).all()
    # wider penumbra and radius limit soften more pixels
    _, m4 = o.soften(vis, dist, 4, 1.5)
    _, m8 = o.soften(vis, dist, 8, 3.0)
    assert ((m8 > 0) & (m8 < 1)).sum() > ((m4 > 0) & (m4 < 1)).sum()


def test_oracle_no_shadow_means_fully_lit(small):
    w, pools = small
    v = w.view(W.penumbra_camera())
    o = Oracle(v, *pools)
    vis, _, _ = o.frame_vis()
    _, mask = o.soften(vis, np.zeros(o.npix, np.float32), 8, 3.0)
    assert (mask == 1.0).all()


# -- GPU: the fused kernel against the oracle ----------------------------------

def gpu_mask(pools, v, limit, pen):
    from voxelcraft_menu_b200.march import Marcher
    m = Marcher(int(v.frame.res[0]), int(v.frame.res[1]), device=0)
    try:
        m.upload_world(*pools)
        m.upload_view(v)
        m.render()
        m.soften_shadows(limit, pen)
        return m.read_vis(), m.read_shadow(), m.read_shadow_mask()
    finally:
        m.close()


def assert_close(mask, ref):
    d = np.abs(mask - ref)
    assert d.max() <= MASK_ATOL, f"max |GPU - oracle| {d.max()}"
    far = (d > NEAR_ATOL).mean()
    assert far <= NEAR_FRACTION, f"{far:.2e} of the pixels differ by more than {NEAR_ATOL}"


@pytest.mark.gpu
@pytest.mark.parametrize("limit,pen", [(4, 1.5), (8, 3.0), (8, 1.0), (1, 1.5)])
def test_gpu_soften_matches_oracle(small, limit, pen):
    w, pools = small
    v = w.view(W.penumbra_camera())
    vis, dist, mask = gpu_mask(pools, v, limit, pen)
    o = Oracle(v, *pools)
    ovis, _, _ = o.frame_vis()
    assert np.array_equal(vis, ovis)
    assert np.array_equal(dist, o.shadow(ovis))
    _, ref = o.soften(vis, dist, limit, pen)
    assert_close(mask, ref)
    if limit >= 4:
        assert ((mask > 0) & (mask < 1)).sum() > 500


@pytest.mark.gpu
@pytest.mark.parametrize("size", [(1920, 1080), (333, 171)])
def test_gpu_soften_ragged_and_1080p(small, size):
    # 1080p: 60 x 34 tiles, the last row cut at 1080 = 33 * 32 + 24; 333 x 171: both edges ragged
    w, pools = small
    v = w.view(W.penumbra_camera(width=size[0], height=size[1]))
    vis, dist, mask = gpu_mask(pools, v, 8, 3.0)
    _, ref = Oracle(v, *pools).soften(vis, dist, 8, 3.0)
    assert_close(mask, ref)


@pytest.mark.gpu
def test_gpu_soften_inactive_and_far_view(small):
    w, pools = small
    v = w.view(W.small_terrain_camera())          # penumbrae under half a pixel: the hard mask
    vis, dist, mask = gpu_mask(pools, v, 8, 1.5)
    assert np.array_equal(mask, hard_mask(dist))
    v = w.view(W.penumbra_camera())
    v.frame.daylight = 0.0                         # shadow_active() false
    vis, dist, mask = gpu_mask(pools, v, 8, 3.0)
    assert np.array_equal(mask, hard_mask(dist))


@pytest.mark.gpu
def test_gpu_soften_rejects_bad_arguments(small):
    from voxelcraft_menu_b200.march import Marcher
    w, pools = small
    v = w.view(W.penumbra_camera())
    m = Marcher(640, 360, device=0)
    try:
        m.upload_world(*pools)
        m.upload_view(v)
        with pytest.raises(RuntimeError):
            m.read_shadow_mask()                   # before any vm_soften_shadows
        m.render()
        for limit, pen in ((0, 1.5), (9, 1.5), (4, 0.0), (4, math.inf), (4, math.nan)):
            with pytest.raises(RuntimeError):
                m.soften_shadows(limit, pen)
        m.set_spec(SPEC_DEFAULT | SPEC_SOFT_RAYS)
        m.render()
        with pytest.raises(RuntimeError):
            m.soften_shadows(4, 1.5)               # jittered rays: blocked fractions, not distances
    finally:
        m.close()
