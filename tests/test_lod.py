"""Level-of-detail chunks and the LOD cross-fade dither.

The engine draws distant terrain as coarser chunks (ChunkKey.lod, voxels of
1 << lod blocks, src/voxel/chunk.rs:6-53) and cross-fades a finer set in over
its parent with a screen-space dither (RenderItem::fade, src/lod.rs:56-80;
ray_skips, common.wgsl:370-385).  The world here mixes lod 0, 1 and 2 chunks
with one cross-faded region (world.mixed_lod_layout).

CPU: the oracle's frame really exercises those paths (hits in chunks of
voxel size 2 and 4, both sides of the dither in the faded region, dither
pattern moving with the frame index).  GPU: the CUDA path over the product's
world equals the oracle over the oracle producer's own world, bit for bit,
through the pipeline and the engine pass sequence, with and without Hi-Z."""
import math

import numpy as np
import pytest

from oracle import producer as OP
from oracle.oracle import Oracle
from voxelcraft_menu_b200 import world as W
from voxelcraft_menu_b200.world import Camera, World

CAMS = [dict(pos=(128.0, 110.0, 20.0)),
        dict(pos=(300.0, 95.0, 120.0), yaw=math.radians(120.0), pitch=math.radians(-20.0)),
        dict(pos=(190.0, 100.0, 190.0), yaw=math.radians(60.0), pitch=math.radians(-35.0), frame_index=5),
        dict(pos=(190.0, 100.0, 190.0), yaw=math.radians(60.0), pitch=math.radians(-35.0), frame_index=6)]


@pytest.fixture(scope="module")
def worlds():
    rec, lay = W.recipe_mixed_lod(), W.mixed_lod_layout()
    pw = World()
    W.build_layout(pw, rec, lay)
    return pw, OP.build_layout(rec, lay)


def _cam(i, **kw):
    c = dict(width=320, height=180)
    c.update(CAMS[i])
    c.update(kw)
    return Camera(**c)


def _oracle(view, world):
    o = Oracle(view, *world.pools())
    vis, hiz, ctr = o.frame_vis()
    return o, vis, o.shadow(vis), o.secondary(vis)


def test_lod_paths_are_exercised(worlds):
    _, ow = worlds
    v = ow.view(_cam(2))
    o, vis, sh, (sk, st) = _oracle(v, ow)
    ci = ((vis >> np.uint64(24)) & np.uint64(0x1FFF)).astype(np.int64)[vis != 0]
    lods = v.chunks["lod"][ci]
    assert (lods == 0).any() and (lods == 1).any() and (lods == 2).any(), "hits in chunks of voxel size 1, 2 and 4"
    fade = v.chunks["fade"][ci]
    assert (fade == np.float32(0.6)).any() and (fade == np.float32(-0.6)).any(), \
        "the dither shows both the fading-in chunks and their fading-out parent"
    assert (sh > 0).any()


def test_the_dither_moves_with_the_frame_index(worlds):
    _, ow = worlds
    a = _oracle(ow.view(_cam(2)), ow)[1]
    b = _oracle(ow.view(_cam(3)), ow)[1]
    assert (a != b).mean() > 0.01


@pytest.mark.gpu
@pytest.mark.parametrize("i", range(len(CAMS)))
def test_lod_world_matches_the_oracle(worlds, i):
    from voxelcraft_menu_b200.march import Marcher
    pw, ow = worlds
    pv = pw.view(_cam(i))
    ov = ow.view(_cam(i))
    _, vis, sh, (sk, st) = _oracle(ov, ow)
    m = Marcher(320, 180)
    m.upload_world(*pw.pools())
    m.upload_view(pv)
    for run in (m.render, m.render_passes):
        run()
        assert np.array_equal(m.read_vis(), vis), f"{run.__name__}: vis"
        assert np.array_equal(m.read_shadow(), sh), f"{run.__name__}: shadow"
        gk, gt = m.read_secondary()
        assert np.array_equal(gk, sk), f"{run.__name__}: secondary key"
        assert np.array_equal(gt, st), f"{run.__name__}: secondary t"
    assert m.stats().device_error == 0
    m.close()


@pytest.mark.gpu
def test_lod_world_hiz_frames_match_the_oracle(worlds):
    """Frame A, then B half a voxel over with A's Hi-Z: deferred and recovered
    pairs of LOD chunks, through the engine passes."""
    from voxelcraft_menu_b200.march import Marcher
    pw, ow = worlds
    flags = W.FLAG_SHADOWS | W.FLAG_WATER_REFRACT | W.FLAG_HIZ
    ca, cb = _cam(1, flags=flags), _cam(1, flags=flags)
    cb.pos = (cb.pos[0] + 0.5, cb.pos[1], cb.pos[2])
    oa, ob = Oracle(ow.view(ca), *ow.pools()), Oracle(ow.view(cb), *ow.pools())
    vis_a, hiz_a, _ = oa.frame_vis(hiz_in=np.zeros(oa.ntiles, np.uint32))
    vis_b, hiz_b, ctr_b = ob.frame_vis(hiz_in=hiz_a)
    m = Marcher(320, 180)
    m.upload_world(*pw.pools())
    m.upload_view(pw.view(ca))
    m.write_hiz(np.zeros(oa.ntiles, np.uint32))
    m.select(); m.march()
    assert np.array_equal(m.read_vis(), vis_a) and np.array_equal(m.read_hiz(), hiz_a)
    m.upload_view(pw.view(cb))
    m.select(); m.march()
    assert np.array_equal(m.read_vis(), vis_b) and np.array_equal(m.read_hiz(), hiz_b)
    s = m.stats()
    assert s.pairs_deferred == ctr_b[1] and s.pairs_recovered == ctr_b[5]
    m.render()
    assert np.array_equal(m.read_vis(), vis_b)
    m.close()
