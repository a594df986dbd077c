"""The 4096x256x4096 sparse world, soft shadows and jittered frames.

CPU: the jittered sun directions stay inside the 0.02 rad disk and vary per
pixel and frame; the sparse world holds more chunks than one view's 13-bit
chunk field, while each view's own list fits it.  GPU: soft shadows (4 rays
per hit, blocked fraction), Halton-jittered frames and views over the sparse
world match the oracle bit for bit, through the wavefront pipeline, the
engine pass sequence and the batch."""
import math

import numpy as np
import pytest

from oracle.oracle import SPEC_DEFAULT, SPEC_SOFT_RAYS, Oracle
from voxelcraft_menu_b200 import world as W

SOFT = W.FLAG_SHADOWS | W.FLAG_WATER_REFRACT
SOFT_SPEC = SPEC_DEFAULT | SPEC_SOFT_RAYS


@pytest.fixture(scope="module")
def small():
    w = W.World.generate(W.recipe_small_terrain())
    return w, w.pools()


@pytest.fixture(scope="module")
def sparse():
    rec = W.recipe_sparse_world()
    w = W.World.generate(rec)
    return rec, w, w.pools()


def sparse_views(rec, w, n, size, seed=21):
    rng = np.random.default_rng(seed)
    views = []
    for _ in range(n):
        x, z = rng.uniform(300, 3800, 2)
        h = max(W.surface_height(rec, int(x), int(z)), 64)
        views.append(w.view(W.Camera(pos=(float(x), float(h) + 40.0, float(z)), yaw=float(rng.uniform(0, 2 * math.pi)),
                                     pitch=math.radians(-10.0), width=size, height=size, flags=SOFT)))
    return views


def test_soft_directions_stay_in_the_disk(small):
    w, pools = small
    v = w.view(W.small_terrain_camera(width=64, height=36, flags=SOFT))
    o = Oracle(v, *pools, spec=SOFT_SPEC)
    sun = np.array(v.frame.sun_dir, np.float64)
    seen = set()
    for py in range(0, 36, 7):
        for px in range(0, 64, 9):
            for s in range(4):
                d = o.soft_sun_dir(px, py, s).astype(np.float64)
                assert abs(np.linalg.norm(d) - 1.0) < 1e-6
                ang = math.acos(min(1.0, float(d @ sun)))
                assert 0.002 < ang < 0.0201
                seen.add(tuple(np.round(d, 6)))
    assert len(seen) > 40          # rotations differ from pixel to pixel


def test_sparse_world_exceeds_the_chunk_field_per_world_not_per_view(sparse):
    rec, w, pools = sparse
    assert int(w.pool_stats().n_chunks) > 8191
    for v in sparse_views(rec, w, 4, 256):
        assert 0 < len(v.chunks) <= 8191
        assert int(v.frame.chunk_count) <= len(v.chunks)


def test_halton_jitter_sequence():
    js = [W.halton_jitter(i) for i in range(8)]
    assert len(set(js)) == 8
    assert all(-0.5 <= x <= 0.5 and -0.5 <= y <= 0.5 for x, y in js)


@pytest.mark.gpu
def test_soft_shadows_match_the_oracle(small):
    from voxelcraft_menu_b200.march import Marcher
    w, pools = small
    m = Marcher(640, 360)
    m.set_spec(SOFT_SPEC)
    m.upload_world(*pools)
    v = w.view(W.small_terrain_camera(width=320, height=180, flags=SOFT))
    m.upload_view(v)
    m.render()
    vis, sh = m.read_vis(), m.read_shadow()
    m.render_passes()
    assert np.array_equal(m.read_vis(), vis) and np.array_equal(m.read_shadow(), sh)
    o = Oracle(v, *pools, spec=SOFT_SPEC)
    ovis, _, _ = o.frame_vis()
    osh = o.shadow(ovis)
    assert np.array_equal(vis, ovis)
    assert np.array_equal(sh.view(np.uint32), osh.view(np.uint32))
    vals = set(np.unique(sh).tolist())
    assert vals <= {0.0, 0.25, 0.5, 0.75, 1.0}
    assert {0.25, 0.5, 0.75} & vals           # penumbrae exist
    counted = m.render_counted()
    _, tr = o.shadow(ovis, traffic=True)
    assert counted["rays_shadow"] == tr["rays"] and tr["rays"] % 4 == 0 and tr["rays"] > 0


@pytest.mark.gpu
def test_halton_jittered_frames_match_the_oracle(small):
    from voxelcraft_menu_b200.march import Marcher
    w, pools = small
    m = Marcher(640, 360)
    m.set_spec(SOFT_SPEC)
    m.upload_world(*pools)
    for k in (1, 6):
        cam = W.small_terrain_camera(width=160, height=90, flags=SOFT, jitter=W.halton_jitter(k), frame_index=k)
        v = w.view(cam)
        m.upload_view(v)
        m.render()
        o = Oracle(v, *pools, spec=SOFT_SPEC)
        ovis, _, _ = o.frame_vis()
        assert np.array_equal(m.read_vis(), ovis)
        assert np.array_equal(m.read_shadow().view(np.uint32), o.shadow(ovis).view(np.uint32))


@pytest.mark.gpu
def test_sparse_world_views_match_the_oracle(sparse):
    from voxelcraft_menu_b200.march import Marcher
    rec, w, pools = sparse
    views = sparse_views(rec, w, 3, 96)
    m = Marcher(1024, 1024)
    m.set_spec(SOFT_SPEC)
    m.upload_world(*pools)
    m.batch_set(views)
    m.batch_run(secondary=True)
    bv, bs = m.batch_read()
    bk, bt = m.batch_read_secondary()
    off = 0
    for v in views:
        n = v.n_pixels
        o = Oracle(v, *pools, spec=SOFT_SPEC)
        ovis, _, _ = o.frame_vis()
        assert np.array_equal(bv[off:off + n], ovis)
        assert np.array_equal(bs[off:off + n].view(np.uint32), o.shadow(ovis).view(np.uint32))
        sk, st = o.secondary(ovis)
        assert np.array_equal(bk[off:off + n], sk)
        assert np.array_equal(bt[off:off + n].view(np.uint32), st.view(np.uint32))
        off += n
    assert np.count_nonzero(bv) > 0


@pytest.mark.gpu
def test_sparse_soft_gbuffer_and_gradient_match_fp64(sparse):
    """The fit's inputs on the sparse world: soft-shadow G-buffer equal to the
    oracle's, gradient within 1e-4 of the FP64 gradient."""
    torch = pytest.importorskip("torch")
    from oracle import shade_oracle as SO
    from voxelcraft_menu_b200 import shading as S
    from voxelcraft_menu_b200 import views as V
    from voxelcraft_menu_b200.march import Marcher
    rec, w, pools = sparse
    views = V.ragged_views(w, n=3, sizes=(96, 128), flags=SOFT, jitter=W.halton_jitter(3), frame_index=3)
    m = Marcher(1024, 1024)
    m.set_spec(SOFT_SPEC)
    m.upload_world(*pools)
    m.batch_set(views)
    m.batch_run(secondary=True)
    k = S.consts()
    gb = S.gbuffer(m, k, torch)
    got = gb.cpu().numpy().view(S.GBUF_DTYPE)
    want = []
    for v in views:
        o = Oracle(v, *pools, spec=SOFT_SPEC)
        ovis, _, _ = o.frame_vis()
        sk, st = o.secondary(ovis)
        want.append(SO.gbuffer_from_oracle(o, ovis, o.shadow(ovis), sk, st, k.fog_falloff, k.fog_height))
    want = np.concatenate(want)
    assert np.array_equal(got["code"], want["code"])
    assert np.array_equal(got["t"].view(np.uint32), want["t"].view(np.uint32))
    soft = got["code"] & SO.G_SOFT
    assert np.count_nonzero(soft) > 0
    model = SO.Model(got, S.SUN_RGB)
    assert np.count_nonzero((model.lit > 0) & (model.lit < 1)) > 0     # penumbrae reach the shading
    p = S.default_params()
    target = model.forward(S.perturbed(p)).astype(np.float32)
    grad = S.backward(gb, torch.from_numpy(p).cuda(), k, torch, target=torch.from_numpy(target).cuda())
    g64 = model.grad(p.astype(np.float64), target)
    g = grad.cpu().numpy()
    assert np.linalg.norm(g - g64) <= 1e-4 * np.linalg.norm(g64)
