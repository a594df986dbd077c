"""Parity of the CUDA march with the oracle, through the C ABI.

Bar: visibility keys, shadow blocker distances, secondary keys and distances,
voxel indices and faces are compared bit for bit; hit distances are held to
1e-5 relative (and are bit-exact here because both sides follow the same
float contract)."""
import math

import numpy as np
import pytest

from oracle.oracle import Oracle
from voxelcraft_menu_b200 import world as W
from voxelcraft_menu_b200.march import PRIMARY_WARPS, MarchError, Marcher
from voxelcraft_menu_b200.world import Camera, Recipe, World

pytestmark = pytest.mark.gpu

T_RTOL = 1e-5


@pytest.fixture(scope="module")
def small():
    w = World.generate(W.recipe_small_terrain())
    pools = w.pools()
    m = Marcher(1920, 1080)
    m.upload_world(*pools)
    return w, pools, m


@pytest.fixture(scope="module")
def large():
    rec = W.recipe_large_terrain()
    w = World.generate(rec)
    pools = w.pools()
    m = Marcher(1920, 1080)
    m.upload_world(*pools)
    return rec, w, pools, m


def oracle_all(view, pools, hiz_in=None, tiles=None):
    o = Oracle(view, *pools)
    vis, hiz, ctr = o.frame_vis(hiz_in=hiz_in, tiles=tiles)
    sh = o.shadow(vis)
    sk, st = o.secondary(vis)
    return o, vis, hiz, ctr, sh, sk, st


def tile_min_depth(vis, view):
    """build_hiz (march.wgsl:57-76) over a visibility buffer: per 8x8 tile the
    minimum depth key, 0 when a pixel of the tile (or outside the frame) missed."""
    w, h = view.res
    tx, ty = int(view.frame.tiles[0]), int(view.frame.tiles[1])
    d = np.zeros((ty * 8, tx * 8), np.uint32)
    d[:h, :w] = (vis >> np.uint64(40)).astype(np.uint32).reshape(h, w)
    return d.reshape(ty, 8, tx, 8).min(axis=(1, 3)).reshape(-1)


def assert_same(got, want, what):
    if not np.array_equal(got, want):
        bad = np.flatnonzero(got != want)
        raise AssertionError(f"{what}: {bad.size} of {got.size} differ; first at {bad[:5]}: "
                             f"got {got[bad[:5]]}, want {want[bad[:5]]}")


def test_engine_passes_match_the_oracle(small):
    w, pools, m = small
    v = w.view(W.small_terrain_camera())
    m.upload_view(v)
    m.render_passes()
    o, vis, hiz, ctr, sh, sk, st = oracle_all(v, pools)
    assert_same(m.read_vis(), vis, "vis")
    assert_same(m.read_shadow(), sh, "shadow")
    gk, gt = m.read_secondary()
    assert_same(gk, sk, "secondary key")
    assert_same(gt, st, "secondary t")
    s = m.stats()
    assert s.device_error == 0
    assert s.pairs_selected == ctr[4] and s.counters[3] == ctr[3]
    assert (vis != 0).mean() > 0.3 and (sh > 0).any() and ((sk >> 63) & 1).any()


@pytest.mark.parametrize("warps,level,per_sm,packet", [(4, 0, 0, 1), (4, 1, 0, 1), (4, 2, 1, 1), (4, 3, 0, 1),
                                                        (8, 4, 0, 1), (8, 0, 0, 1), (8, 2, 0, 1), (4, 1, 0, 2),
                                                        (4, 3, 4, 2), (8, 0, 0, 2)])
def test_pipeline_matches_the_oracle(small, warps, level, per_sm, packet):
    w, pools, m = small
    v = w.view(W.small_terrain_camera())
    m.upload_view(v)
    m.set_tuning(warps, level, per_sm, packet)
    m.render()
    o, vis, hiz, ctr, sh, sk, st = oracle_all(v, pools)
    assert_same(m.read_vis(), vis, "vis")
    assert_same(m.read_shadow(), sh, "shadow")
    gk, gt = m.read_secondary()
    assert_same(gk, sk, "secondary key")
    assert_same(gt, st, "secondary t")
    assert m.stats().device_error == 0
    m.set_tuning()


def test_expanded_outputs(small):
    w, pools, m = small
    v = w.view(W.small_terrain_camera())
    m.upload_view(v)
    m.render()
    o = Oracle(v, *pools)
    vis, _, _ = o.frame_vis()
    vox, face, t = m.read_expanded((0, 0, 0), (256, 128, 256))
    ov, of, ot = o.expand(vis, (0, 0, 0), (256, 128, 256))
    assert_same(vox, ov, "voxel index")
    assert_same(face, of, "face")
    hit = ov != 0xFFFFFFFF
    assert np.all(np.abs(t[hit] - ot[hit]) <= T_RTOL * np.abs(ot[hit]))
    # the voxel index names the block the key names
    idx = np.flatnonzero(hit)[:: max(1, hit.sum() // 500)]
    for i in idx:
        x, rest = ov[i] % 256, ov[i] // 256
        z, y = rest % 256, rest // 256
        assert w.get_block(int(x), int(y), int(z)) != W.AIR


def test_hiz_frames_match_the_oracle(small):
    """Frame A, then frame B with the camera moved half a voxel, FLAG_HIZ on:
    the engine's pass sequence keeps every counter of the oracle's."""
    w, pools, m = small
    flags = W.FLAG_SHADOWS | W.FLAG_WATER_REFRACT | W.FLAG_HIZ
    va = w.view(W.small_terrain_camera(flags=flags))
    m.upload_view(va)
    m.write_hiz(np.zeros(int(va.frame.tiles[0]) * int(va.frame.tiles[1]), np.uint32))
    m.select(); m.march()
    oa = Oracle(va, *pools)
    vis_a, hiz_a, ctr_a = oa.frame_vis(hiz_in=np.zeros(oa.ntiles, np.uint32))
    assert_same(m.read_vis(), vis_a, "vis A")
    assert_same(m.read_hiz(), hiz_a, "hiz A")
    cam_b = W.small_terrain_camera(flags=flags)
    cam_b.pos = (cam_b.pos[0] + 0.5, cam_b.pos[1], cam_b.pos[2])
    vb = w.view(cam_b)
    m.upload_view(vb)
    m.select(); m.march()
    vis_b, hiz_b, ctr_b = Oracle(vb, *pools).frame_vis(hiz_in=hiz_a)
    assert_same(m.read_vis(), vis_b, "vis B")
    assert_same(m.read_hiz(), hiz_b, "hiz B")
    s = m.stats()
    assert s.pairs_deferred == ctr_b[1] > 0
    assert s.pairs_recovered == ctr_b[5]
    assert s.pairs_selected == ctr_b[4]
    # and the fused kernel gives the same visibility
    m.render()
    assert_same(m.read_vis(), vis_b, "fused vis B")


def test_heatmap_matches_the_oracle(small):
    w, pools, m = small
    v = w.view(W.small_terrain_camera(flags=W.FLAG_HEATMAP))
    m.upload_view(v)
    m.select(); m.march()
    vis, hiz, ctr, dbg = Oracle(v, *pools).frame_vis(heat=True)
    assert_same(m.read_vis(), vis, "vis")
    assert_same(m.read_heatmap(), dbg, "iteration heatmap")


@pytest.mark.parametrize("res", [(1, 1), (7, 5), (333, 77), (64, 64), (129, 257)])
def test_ragged_resolutions(small, res):
    w, pools, m = small
    v = w.view(W.small_terrain_camera(width=res[0], height=res[1]))
    m.upload_view(v)
    o, vis, hiz, ctr, sh, sk, st = oracle_all(v, pools)
    for warps in PRIMARY_WARPS:
        for packet in (1, 2):
            m.set_tuning(warps, packet=packet)
            m.render()
            assert_same(m.read_vis(), vis, f"pipeline {warps} warps, packet {packet}: vis")
            assert_same(m.read_shadow(), sh, f"pipeline {warps} warps, packet {packet}: shadow")
    m.set_tuning()
    m.render_passes()
    assert_same(m.read_vis(), vis, "passes vis")
    assert_same(m.read_shadow(), sh, "passes shadow")


@pytest.mark.parametrize("yaw,pitch,pos", [(0.0, -30.0, (30.0, 100.0, 130.0)), (200.0, -5.0, (200.0, 70.0, 200.0)),
                                           (45.0, 60.0, (128.0, 66.0, 128.0)), (135.0, -89.0, (60.0, 95.0, 60.0))])
def test_other_cameras(small, yaw, pitch, pos):
    """Cameras looking up, down, along the axes, close to the water and inside
    the terrain's bounding boxes (camera chunk path)."""
    w, pools, m = small
    v = w.view(Camera(pos=pos, yaw=math.radians(yaw), pitch=math.radians(pitch), width=320, height=200))
    m.upload_view(v)
    o, vis, hiz, ctr, sh, sk, st = oracle_all(v, pools)
    m.render()
    assert_same(m.read_vis(), vis, "fused vis")
    assert_same(m.read_shadow(), sh, "fused shadow")
    gk, gt = m.read_secondary()
    assert_same(gk, sk, "fused secondary")
    m.render_passes()
    assert_same(m.read_vis(), vis, "passes vis")


def test_underwater_camera(small):
    w, pools, m = small
    flags = W.FLAG_SHADOWS | W.FLAG_WATER_REFRACT | W.FLAG_UNDERWATER | W.FLAG_WATER_FAR | W.FLAG_WATER_DARK
    rec = W.recipe_small_terrain()
    # find a column under water
    for x in range(0, 256, 8):
        h = W.surface_height(rec, x, 128)
        if h < 58:
            break
    v = w.view(Camera(pos=(x + 0.5, 62.0, 128.5), pitch=math.radians(10.0), width=320, height=200, flags=flags))
    assert v.frame.flags & W.FLAG_UNDERWATER
    m.upload_view(v)
    o, vis, hiz, ctr, sh, sk, st = oracle_all(v, pools)
    m.render()
    assert_same(m.read_vis(), vis, "fused vis")
    m.render_passes()
    assert_same(m.read_vis(), vis, "passes vis")
    assert_same(m.read_shadow(), sh, "shadow")


def test_empty_world_and_empty_view():
    w = World()
    d = np.zeros(64 ** 3, np.uint16)
    w.insert_dense((0, 0, 0), d)
    m = Marcher(64, 64)
    m.upload_world(*w.pools())
    v = w.view(Camera(pos=(10.0, 10.0, 10.0), width=64, height=64))
    assert len(v.chunks) == 0
    m.upload_view(v)
    m.render()
    assert not m.read_vis().any()
    m.render_passes()
    assert not m.read_vis().any()


def test_large_world_reduced_resolution(large):
    rec, w, pools, m = large
    v = w.view(W.large_terrain_camera(rec, width=480, height=270))
    m.upload_view(v)
    o, vis, hiz, ctr, sh, sk, st = oracle_all(v, pools)
    m.render()
    assert_same(m.read_vis(), vis, "vis")
    assert_same(m.read_shadow(), sh, "shadow")
    gk, gt = m.read_secondary()
    assert_same(gk, sk, "secondary key")
    assert_same(gt, st, "secondary t")
    glass = ((sk >> 63) & 1).astype(bool) & ((sk >> 61) & 1).astype(bool)
    water = ((sk >> 63) & 1).astype(bool) & ~((sk >> 61) & 1).astype(bool)
    assert glass.any() and water.any()


def test_large_world_full_hd(large):
    """1920x1080: fused kernel == engine pass sequence on the GPU over every
    pixel, and == the oracle on a band of tiles."""
    rec, w, pools, m = large
    v = w.view(W.large_terrain_camera(rec))
    m.upload_view(v)
    m.render()
    fv, fs = m.read_vis(), m.read_shadow()
    fk, ft = m.read_secondary()
    m.render_passes()
    assert_same(m.read_vis(), fv, "vis fused vs passes")
    assert_same(m.read_shadow(), fs, "shadow fused vs passes")
    pk, pt = m.read_secondary()
    assert_same(pk, fk, "secondary fused vs passes")
    o = Oracle(v, *pools)
    tx = int(v.frame.tiles[0])
    rows = (60 * tx, 64 * tx)            # four tile rows across the horizon
    vis, _, _ = o.frame_vis(tiles=rows)
    sl = slice(60 * 8 * 1920, 64 * 8 * 1920)
    assert_same(fv[sl], vis[sl], "vis band")
    sh = o.shadow(vis, pix=(sl.start, sl.stop))
    assert_same(fs[sl], sh[sl], "shadow band")


def test_large_world_full_frame_a_and_b_match_the_oracle(large):
    """The benchmarked frame pair over every pixel: frame A with FLAG_HIZ and a
    cleared Hi-Z, then frame B with the camera moved half a voxel and A's Hi-Z
    carried over.  Visibility, shadow distances, water / glass keys and
    distances and the Hi-Z equal the oracle's through both the engine pass
    sequence and vm_render; the engine passes also report the oracle's
    deferred / recovered pair counts."""
    rec, w, pools, m = large
    flags = W.FLAG_SHADOWS | W.FLAG_WATER_REFRACT | W.FLAG_HIZ
    cam_a = W.large_terrain_camera(rec, flags=flags)
    va = w.view(cam_a)
    cam_b = W.large_terrain_camera(rec, flags=flags)
    cam_b.pos = (cam_b.pos[0] + 0.5, cam_b.pos[1], cam_b.pos[2])
    vb = w.view(cam_b)
    ntiles = int(va.frame.tiles[0]) * int(va.frame.tiles[1])
    oa = Oracle(va, *pools)
    vis_a, hiz_a, ctr_a = oa.frame_vis(hiz_in=np.zeros(ntiles, np.uint32))
    sh_a = oa.shadow(vis_a)
    sk_a, st_a = oa.secondary(vis_a)
    ob = Oracle(vb, *pools)
    vis_b, hiz_b, ctr_b = ob.frame_vis(hiz_in=hiz_a)
    sh_b = ob.shadow(vis_b)
    sk_b, st_b = ob.secondary(vis_b)
    assert ctr_b[1] > 0, "frame B defers pairs against A's Hi-Z"
    assert (sh_b > 0).any() and (sk_b >> 62 & 1).any()

    def check(tag, vis, sh, sk, st, hiz):
        assert_same(m.read_vis(), vis, f"{tag} vis")
        assert_same(m.read_shadow(), sh, f"{tag} shadow")
        gk, gt = m.read_secondary()
        assert_same(gk, sk, f"{tag} secondary key")
        assert_same(gt, st, f"{tag} secondary t")
        assert_same(m.read_hiz(), hiz, f"{tag} hiz")
        assert m.stats().device_error == 0

    # engine pass sequence
    m.upload_view(va)
    m.write_hiz(np.zeros(ntiles, np.uint32))
    m.render_passes()
    check("passes A", vis_a, sh_a, sk_a, st_a, hiz_a)
    m.upload_view(vb)
    m.render_passes()
    check("passes B", vis_b, sh_b, sk_b, st_b, hiz_b)
    s = m.stats()
    assert s.pairs_deferred == ctr_b[1] and s.pairs_recovered == ctr_b[5] and s.pairs_selected == ctr_b[4]
    # the wavefront pipeline, frame A then B; its Hi-Z output is build_hiz
    # (march.wgsl:57-76) of the final visibility
    m.upload_view(va)
    m.render()
    check("pipeline A", vis_a, sh_a, sk_a, st_a, tile_min_depth(vis_a, va))
    m.upload_view(vb)
    m.render()
    check("pipeline B", vis_b, sh_b, sk_b, st_b, tile_min_depth(vis_b, vb))


def _sun(t):
    """The engine's sun(t) direction (src/scene.rs:10-14) in float32, with
    glam's normalize (v * (1 / length))."""
    a = np.float32((t - 0.25) * np.float32(2.0 * np.pi))
    v = np.array([np.cos(a) * np.float32(0.55), np.sin(a), np.float32(0.42)], np.float32)
    r = np.float32(1.0) / np.sqrt(np.float32((v * v).sum()))
    return tuple((v * r).astype(np.float32).tolist())


@pytest.mark.parametrize("sun", ["t=0.25", (0.0, 0.8, 0.6), (0.6, 0.8, 0.0), (0.0, 1.0, 0.0)])
def test_sun_with_zero_components_matches_the_oracle(small, sun):
    """The engine's sun at t = 0.25 has dir.y == 0 exactly, with daylight 0.375
    and shadows on; axis-aligned suns give infinite reciprocals in x or z.
    Both sides follow IEEE arithmetic from 1 / 0 = inf on."""
    w, pools, m = small
    d = _sun(0.25) if sun == "t=0.25" else sun
    if sun == "t=0.25":
        assert d[1] == 0.0
    v = w.view(W.small_terrain_camera(sun_dir=d, daylight=0.375))
    m.upload_view(v)
    o, vis, hiz, ctr, sh, sk, st = oracle_all(v, pools)
    m.render()
    assert_same(m.read_vis(), vis, "vis")
    assert_same(m.read_shadow(), sh, "shadow")
    gk, gt = m.read_secondary()
    assert_same(gk, sk, "secondary key")
    m.render_passes()
    assert_same(m.read_shadow(), sh, "passes shadow")


def test_batch_matches_single_views(small):
    w, pools, m = small
    rng = np.random.default_rng(3)
    views = []
    for i in range(12):
        res = int(rng.choice([32, 64, 128]))
        pos = (float(rng.uniform(20, 236)), float(rng.uniform(90, 120)), float(rng.uniform(20, 236)))
        views.append(w.view(Camera(pos=pos, yaw=float(rng.uniform(0, 6.28)), pitch=float(rng.uniform(-1.2, 0.3)),
                                   fov_y=math.radians(90.0), width=res, height=res)))
    views.append(w.view(W.small_terrain_camera()))
    m.batch_set(views)
    m.batch_run()
    bv, bs = m.batch_read()
    m.batch_run(per_view=True)
    pv, ps = m.batch_read()
    assert_same(pv, bv, "per-view vs persistent vis")
    assert_same(ps, bs, "per-view vs persistent shadow")
    m.set_tuning(8, 3, 0, 2)
    m.batch_run()
    qv, qs = m.batch_read()
    m.set_tuning()
    assert_same(qv, bv, "8x8-pixel items vs 8x4 vis")
    assert_same(qs, bs, "8x8-pixel items vs 8x4 shadow")
    off = 0
    for v in views:
        n = v.n_pixels
        o = Oracle(v, *pools)
        vis, _, _ = o.frame_vis()
        sh = o.shadow(vis)
        assert_same(bv[off:off + n], vis, "batch vis")
        assert_same(bs[off:off + n], sh, "batch shadow")
        off += n
    m.batch_run()   # graph replay
    bv2, _ = m.batch_read()
    assert_same(bv2, bv, "graph replay")


def test_invalid_frames_are_rejected(small):
    w, pools, m = small
    v = w.view(W.small_terrain_camera())
    m.upload_view(v)
    f = v.frame
    bad = type(f).from_buffer_copy(f)
    bad.tiles[0] = 3
    m.set_frame(bad)
    with pytest.raises(MarchError) as e:
        m.render()
    assert e.value.code == 1
    bad = type(f).from_buffer_copy(f)
    bad.chunk_count = 100000
    m.set_frame(bad)
    with pytest.raises(MarchError):
        m.select()
    big = Marcher(8192, 4320)
    big.upload_world(*pools)
    vb = w.view(W.small_terrain_camera(width=8192, height=4320))
    with pytest.raises(MarchError) as e:
        big.upload_view(vb)
        big.select()
    assert e.value.code == 3, "tile index overflows the pair word"
    big.close()
    m.set_frame(f)


def test_cost_order_and_stage_events_leave_the_output_unchanged(small):
    """Every frame is scheduled by the previous one's measured item costs; the
    order may change from frame to frame, the output may not.  The stage
    events bracket the cull, primary, shadow and secondary kernels."""
    torch = pytest.importorskip("torch")
    w, pools, m = small
    v = w.view(W.small_terrain_camera(width=480, height=270))
    m.upload_view(v)
    m.render()
    vis0, sh0, (k0, t0) = m.read_vis(), m.read_shadow(), m.read_secondary()
    stream = torch.cuda.Stream()
    m._ck(m._L.vm_set_stream(m._h, __import__("ctypes").c_void_p(stream.cuda_stream)))
    try:
        for _ in range(3):
            evs = [torch.cuda.Event(enable_timing=True) for _ in range(5)]
            for e in evs:
                e.record(stream)
            torch.cuda.synchronize()
            m.render_events([e.cuda_event for e in evs])
            torch.cuda.synchronize()
            stages = [evs[i].elapsed_time(evs[i + 1]) for i in range(4)]
            assert all(s >= 0.0 for s in stages) and stages[1] > 0.0
            assert abs(sum(stages) - evs[0].elapsed_time(evs[4])) < 1e-3
            assert_same(m.read_vis(), vis0, "vis after reordering")
            assert_same(m.read_shadow(), sh0, "shadow after reordering")
            k, t = m.read_secondary()
            assert_same(k, k0, "secondary keys after reordering")
            assert_same(t, t0, "secondary t after reordering")
    finally:
        m._ck(m._L.vm_set_stream(m._h, None))


def test_async_read_back_equals_the_synchronous_one(small):
    torch = pytest.importorskip("torch")
    import ctypes as C
    w, pools, m = small
    v = w.view(W.small_terrain_camera(width=333, height=77))
    m.upload_view(v)
    m.render()
    n = v.n_pixels
    vis_h = torch.zeros(n, dtype=torch.int64).pin_memory()
    sh_h = torch.zeros(n, dtype=torch.float32).pin_memory()
    m._ck(m._L.vm_read_async(m._h, C.c_void_p(vis_h.data_ptr()), C.c_void_p(sh_h.data_ptr())))
    m.sync()
    assert_same(vis_h.numpy().view(np.uint64), m.read_vis(), "async vis")
    assert_same(sh_h.numpy(), m.read_shadow(), "async shadow")
    m._ck(m._L.vm_read_async(m._h, None, C.c_void_p(sh_h.data_ptr())))   # either pointer may be NULL
    m.sync()


@pytest.mark.parametrize("res", [(333, 77), (1920, 1080)])
def test_r16f_read_back_is_the_oracle_shadow_in_binary16(small, res):
    """vm_read_async_r16f: the engine's R16F shadow target (shadow.wgsl:1),
    i.e. the oracle's blocker distances rounded to binary16 (nearest even);
    333x77 leaves a ragged tail of the 4-pixel conversion."""
    from oracle.oracle import f16_round
    w, pools, m = small
    v = w.view(W.small_terrain_camera(width=res[0], height=res[1]))
    m.upload_view(v)
    m.render()
    r16 = m.read_shadow_r16f()
    _, _, _, _, sh, _, _ = oracle_all(v, pools)
    assert_same(r16, sh.astype(np.float16).view(np.uint16), "r16f shadow vs numpy binary16 of the oracle")
    assert_same(r16.view(np.float16).astype(np.float32), f16_round(sh), "r16f shadow vs the oracle's f16 rounding")
    assert_same(m.read_shadow(), sh, "float shadow unchanged")


def test_contexts_in_flight_give_each_frame_its_own_output(small):
    """Two contexts alternating with vm_wait_render and asynchronous
    read-backs (the bench's end-to-end loop) return every frame's own
    visibility and R16F shadow."""
    torch = pytest.importorskip("torch")
    import ctypes as C
    w, pools, m = small
    views = [w.view(W.small_terrain_camera(width=320, height=200, yaw=math.radians(yaw)))
             for yaw in (60.0, 90.0, 120.0, 150.0)]
    want = []
    for v in views:
        m.upload_view(v)
        m.render()
        want.append((m.read_vis(), m.read_shadow().astype(np.float16).view(np.uint16)))
    ctxs = [Marcher(320, 200) for _ in range(2)]
    try:
        n = 320 * 200
        host = [(torch.zeros(n, dtype=torch.int64).pin_memory(), torch.zeros(n, dtype=torch.int16).pin_memory())
                for _ in views]
        for c in ctxs:
            c.upload_world(*pools)
        for i, v in enumerate(views):
            c, prev = ctxs[i % 2], ctxs[(i + 1) % 2]
            c.upload_view(v)
            c.wait_render(prev)
            c._ck(c._L.vm_render(c._h))
            vh, sh = host[i]
            c._ck(c._L.vm_read_async_r16f(c._h, C.c_void_p(vh.data_ptr()), C.c_void_p(sh.data_ptr())))
        for c in ctxs:
            c.sync()
        for i, (vh, sh) in enumerate(host):
            assert_same(vh.numpy().view(np.uint64), want[i][0], f"frame {i} vis")
            assert_same(sh.numpy().view(np.uint16), want[i][1], f"frame {i} r16f shadow")
    finally:
        for c in ctxs:
            c.close()
