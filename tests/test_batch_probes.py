"""Batched ragged views: cube-face probe captures and player views.

CPU: the view set's construction (probe centres in air, face bases,
resolutions).  GPU: the persistent graph-replayed launch equals the
per-view launches and the oracle, bit for bit, and the counted run reports
the same outputs with its ray counts."""
import numpy as np
import pytest

from voxelcraft_menu_b200 import views as V
from voxelcraft_menu_b200 import world as W


@pytest.fixture(scope="module")
def world():
    return W.World.generate(W.recipe_small_terrain())


def test_face_bases_are_orthonormal_and_distinct():
    fwds = set()
    for face in range(6):
        f, r, u = (np.array(v) for v in V.face_basis(face))
        for a in (f, r, u):
            assert abs(np.linalg.norm(a) - 1.0) < 1e-6
        assert abs(f @ r) < 1e-6 and abs(f @ u) < 1e-6 and abs(r @ u) < 1e-6
        fwds.add(tuple(f))
    assert len(fwds) == 6


def test_probe_view_set(world):
    views = V.probe_views(world, n_probes=20)
    assert len(views) == 120
    res = [int(v.frame.res[0]) for v in views]
    assert set(res) <= set(V.PROBE_RES)
    assert all(int(v.frame.res[0]) == int(v.frame.res[1]) for v in views)
    rng = np.random.default_rng(3)
    for c in V.probe_centres(world, 20, rng):
        assert world.get_block(int(c[0]), int(c[1]), int(c[2])) == W.AIR
    # deterministic for a seed
    again = V.probe_views(world, n_probes=20)
    assert [int(v.frame.res[0]) for v in again] == res
    players = V.player_views(world, n=4, width=64, height=36)
    assert len({round(float(v.frame.cam_fwd[0]), 5) for v in players}) == 4


@pytest.mark.gpu
def test_probe_batch_matches_per_view_and_oracle(world):
    from oracle.oracle import Oracle
    from voxelcraft_menu_b200.march import Marcher
    pools = world.pools()
    views = V.probe_views(world, n_probes=4, res=(32, 64)) + V.player_views(world, n=2, width=160, height=90)
    m = Marcher(1920, 1080)
    m.upload_world(*pools)
    m.batch_set(views)
    m.batch_run()
    bv, bs = m.batch_read()
    m.batch_run(per_view=True)
    pv, ps = m.batch_read()
    assert np.array_equal(bv, pv) and np.array_equal(bs, ps)
    traffic = m.batch_counted()
    cv, cs = m.batch_read()
    assert np.array_equal(bv, cv) and np.array_equal(bs, cs)
    assert traffic["rays_primary"] == sum(v.n_pixels for v in views)
    off, shadow_rays = 0, 0
    for v in views:
        n = v.n_pixels
        o = Oracle(v, *pools)
        vis, _, _ = o.frame_vis()
        sh, tr = o.shadow(vis, traffic=True)
        shadow_rays += tr["rays"]
        assert np.array_equal(bv[off:off + n], vis)
        assert np.array_equal(bs[off:off + n], sh)
        off += n
    assert traffic["rays_shadow"] == shadow_rays


@pytest.mark.gpu
def test_256_probe_faces_and_a_full_hd_player_view_match_the_oracle(world):
    """The largest members of the batched workload: 256x256 cube faces and a
    1920x1080 player view, in one persistent batch, equal the oracle bit for
    bit (visibility and shadow distances)."""
    from oracle.oracle import Oracle
    from voxelcraft_menu_b200.march import Marcher
    pools = world.pools()
    views = V.probe_views(world, n_probes=2, res=(256,)) + V.player_views(world, n=1)
    assert views[-1].res == (1920, 1080)
    m = Marcher(1920, 1080)
    m.upload_world(*pools)
    m.batch_set(views)
    m.batch_run()
    bv, bs = m.batch_read()
    off = 0
    for v in views:
        n = v.n_pixels
        o = Oracle(v, *pools)
        vis, _, _ = o.frame_vis()
        sh = o.shadow(vis)
        assert np.array_equal(bv[off:off + n], vis), f"view {v.res}: visibility differs"
        assert np.array_equal(bs[off:off + n], sh), f"view {v.res}: shadow differs"
        off += n
    assert (bv != 0).mean() > 0.3
    m.close()
