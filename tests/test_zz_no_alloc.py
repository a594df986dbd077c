"""vm_render_static: the frame march for callers that cannot allocate device
memory (inside a stream capture they do not own, or under an engine that owns
every byte of device memory through its own arenas).  Every buffer is the
caller's; the scratch is a static device array shared by all calls.

Its output must equal the context-based vm_render bit for bit, on two calls in
a row (the second call starts from the first call's leftover scratch).  This
file is collected last so that a failure here cannot hide the others."""
import ctypes as C

import numpy as np
import pytest

from voxelcraft_menu_b200 import native
from voxelcraft_menu_b200 import world as W
from voxelcraft_menu_b200.march import Marcher

pytestmark = pytest.mark.gpu


def _dev(a, torch):
    return torch.from_numpy(np.ascontiguousarray(a).view(np.uint8).copy()).cuda()


def test_static_scratch_matches_the_context_path():
    import torch
    w = W.World.generate(W.recipe_small_terrain())
    inners, leaves, bricks = w.pools()
    v = w.view(W.small_terrain_camera(width=480, height=270))
    m = Marcher(480, 270)
    m.upload_world(inners, leaves, bricks)
    m.upload_view(v)
    m.render()
    want_vis, want_sh = m.read_vis(), m.read_shadow()
    m.close()

    L = native.lib()
    d_ch, d_grid = _dev(v.chunks, torch), _dev(v.grid.astype(np.uint32), torch)
    d_in, d_le, d_br = _dev(inners, torch), _dev(leaves, torch), _dev(bricks, torch)
    npix = v.n_pixels
    stream = torch.cuda.current_stream()
    for call in range(2):
        d_vis = torch.full((npix,), -1, dtype=torch.int64, device="cuda")
        d_sh = torch.full((npix,), -1.0, dtype=torch.float32, device="cuda")
        d_err = torch.zeros(1, dtype=torch.int32, device="cuda")
        rc = L.vm_render_static(C.byref(v.frame), C.c_void_p(d_ch.data_ptr()), len(v.chunks),
                                C.c_void_p(d_grid.data_ptr()), v.grid.size, C.c_void_p(d_in.data_ptr()),
                                inners.shape[0], C.c_void_p(d_le.data_ptr()), leaves.shape[0],
                                C.c_void_p(d_br.data_ptr()), bricks.size, C.c_void_p(d_vis.data_ptr()),
                                C.c_void_p(d_sh.data_ptr()), C.c_void_p(d_err.data_ptr()),
                                C.c_void_p(stream.cuda_stream))
        assert rc == 0, L.vm_static_last_error().decode()
        torch.cuda.synchronize()
        got_vis = d_vis.cpu().numpy().view(np.uint64)
        got_sh = d_sh.cpu().numpy()
        assert np.array_equal(got_vis, want_vis), f"call {call}: visibility differs"
        assert np.array_equal(got_sh, want_sh), f"call {call}: shadow differs"
        assert int(d_err.item()) == 0


def _render_static(L, torch, v, inners, leaves, bricks):
    d_ch, d_grid = _dev(v.chunks, torch), _dev(v.grid.astype(np.uint32), torch)
    d_in, d_le, d_br = _dev(inners, torch), _dev(leaves, torch), _dev(bricks, torch)
    npix = v.n_pixels
    d_vis = torch.full((npix,), -1, dtype=torch.int64, device="cuda")
    d_sh = torch.full((npix,), -1.0, dtype=torch.float32, device="cuda")
    d_err = torch.zeros(1, dtype=torch.int32, device="cuda")
    rc = L.vm_render_static(C.byref(v.frame), C.c_void_p(d_ch.data_ptr()), len(v.chunks),
                            C.c_void_p(d_grid.data_ptr()), v.grid.size, C.c_void_p(d_in.data_ptr()),
                            inners.shape[0], C.c_void_p(d_le.data_ptr()), leaves.shape[0],
                            C.c_void_p(d_br.data_ptr()), bricks.size, C.c_void_p(d_vis.data_ptr()),
                            C.c_void_p(d_sh.data_ptr()), C.c_void_p(d_err.data_ptr()),
                            C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == 0, L.vm_static_last_error().decode()
    torch.cuda.synchronize()
    assert int(d_err.item()) == 0
    return d_vis.cpu().numpy().view(np.uint64), d_sh.cpu().numpy()


def test_static_scratch_tile_lists_longer_than_its_capacity():
    """The static scratch keeps 64 chunks per tile; a tile whose cull keeps
    more is finished by rescanning the chunk list.  A wide view high over the
    1024-chunk terrain has tiles of up to 100 chunks: the output still equals
    the oracle and the context path on two calls in a row."""
    import math
    import torch
    from oracle.oracle import Oracle
    rec = W.recipe_large_terrain()
    w = W.World.generate(rec)
    inners, leaves, bricks = w.pools()
    cam = W.large_terrain_camera(rec, width=96, height=54)
    cam.fov_y, cam.pitch, cam.pos = math.radians(110.0), math.radians(-25.0), (512.0, 200.0, 100.0)
    v = w.view(cam)
    o = Oracle(v, inners, leaves, bricks)
    assert max(len(o.tile_pairs(t)[0]) for t in range(o.ntiles)) > 64
    vis, _, _ = o.frame_vis()
    sh = o.shadow(vis)
    m = Marcher(96, 54)
    m.upload_world(inners, leaves, bricks)
    m.upload_view(v)
    m.render()
    assert np.array_equal(m.read_vis(), vis)
    m.close()
    L = native.lib()
    for call in range(2):
        got_vis, got_sh = _render_static(L, torch, v, inners, leaves, bricks)
        assert np.array_equal(got_vis, vis), f"call {call}: visibility differs from the oracle"
        assert np.array_equal(got_sh, sh), f"call {call}: shadow differs from the oracle"


def test_static_scratch_replays_from_a_cuda_graph():
    """The entry point's reason to exist: recorded into a stream capture the
    caller owns (here a torch CUDA graph) and replayed, it writes the same
    frame as the context path."""
    import torch
    w = W.World.generate(W.recipe_small_terrain())
    inners, leaves, bricks = w.pools()
    v = w.view(W.small_terrain_camera(width=320, height=180))
    m = Marcher(320, 180)
    m.upload_world(inners, leaves, bricks)
    m.upload_view(v)
    m.render()
    want_vis, want_sh = m.read_vis(), m.read_shadow()
    m.close()
    L = native.lib()
    d_ch, d_grid = _dev(v.chunks, torch), _dev(v.grid.astype(np.uint32), torch)
    d_in, d_le, d_br = _dev(inners, torch), _dev(leaves, torch), _dev(bricks, torch)
    npix = v.n_pixels
    d_vis = torch.full((npix,), -1, dtype=torch.int64, device="cuda")
    d_sh = torch.full((npix,), -1.0, dtype=torch.float32, device="cuda")
    d_err = torch.zeros(1, dtype=torch.int32, device="cuda")

    def call(stream):
        return L.vm_render_static(C.byref(v.frame), C.c_void_p(d_ch.data_ptr()), len(v.chunks),
                                  C.c_void_p(d_grid.data_ptr()), v.grid.size, C.c_void_p(d_in.data_ptr()),
                                  inners.shape[0], C.c_void_p(d_le.data_ptr()), leaves.shape[0],
                                  C.c_void_p(d_br.data_ptr()), bricks.size, C.c_void_p(d_vis.data_ptr()),
                                  C.c_void_p(d_sh.data_ptr()), C.c_void_p(d_err.data_ptr()), C.c_void_p(stream))

    side = torch.cuda.Stream()
    with torch.cuda.stream(side):
        assert call(side.cuda_stream) == 0, L.vm_static_last_error().decode()   # warm-up outside the capture
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, capture_error_mode="thread_local"):
        rc = call(torch.cuda.current_stream().cuda_stream)
    assert rc == 0, L.vm_static_last_error().decode()
    d_vis.fill_(-1)
    d_sh.fill_(-1.0)
    torch.cuda.synchronize()
    for _ in range(2):
        g.replay()
        torch.cuda.synchronize()
        assert np.array_equal(d_vis.cpu().numpy().view(np.uint64), want_vis)
        assert np.array_equal(d_sh.cpu().numpy(), want_sh)
        assert int(d_err.item()) == 0
    del g


def test_static_scratch_rejects_oversized_frames():
    import torch
    w = W.World.generate(W.recipe_small_terrain())
    inners, leaves, bricks = w.pools()
    v = w.view(W.small_terrain_camera(width=640, height=480))   # 307200 pixels > 262144
    L = native.lib()
    dummy = torch.zeros(1 << 20, dtype=torch.uint8, device="cuda")
    p = C.c_void_p(dummy.data_ptr())
    rc = L.vm_render_static(C.byref(v.frame), p, len(v.chunks), p, v.grid.size, p, 1, p, 1, p, 1, p, p, p,
                            C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == 8, "VM_E_TOO_LARGE: refused, not a truncated render"
    assert b"262144" in L.vm_static_last_error()
