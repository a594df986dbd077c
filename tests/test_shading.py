"""The differentiable shading stage: forward, adjoint and G-buffer.

CPU: the FP64 model's analytic gradient against FP64 central differences
(h = 1e-4) on synthetic G-buffers.  GPU: the batch's secondary rays and the
G-buffer decoded on the device are compared with the oracle's (bit-exact,
the fog length to 1e-5 relative); the float32 forward is held to 2e-5
absolute of the FP64 model, and the gradient to 1e-4 relative (norm-wise,
overall and per parameter group) of the FP64 gradient."""
import math

import numpy as np
import pytest

from oracle import shade_oracle as SO
from voxelcraft_menu_b200 import shading as S
from voxelcraft_menu_b200 import world as W

GRAD_RTOL = 1e-4
COLOR_ATOL = 2e-5
GROUPS = {"albedo": slice(0, 768), "sun": slice(S.P_SUN, S.P_SUN + 3), "sky": slice(S.P_SKY, S.P_SKY + 3),
          "fog": slice(S.P_FOG, S.P_FOG + 1), "absorb": slice(S.P_ABS, S.P_ABS + 3)}


def synthetic_gbuffer(n, seed):
    rng = np.random.default_rng(seed)
    g = np.zeros(n, S.GBUF_DTYPE)
    ids = np.where(rng.random(n) < 0.3, SO.WATER, rng.integers(1, 40, n))
    code = ids | (rng.integers(0, 8, n) << 8)
    code |= np.where(rng.random(n) < 0.9, SO.G_HIT, 0)
    code |= np.where(rng.random(n) < 0.7, SO.G_LIT, 0)
    code |= np.where(rng.random(n) < 0.8, SO.G_TRACED, 0)
    code |= np.where(rng.random(n) < 0.6, SO.G_HIT2, 0)
    code |= np.where(rng.random(n) < 0.2, SO.G_FLIP, 0)
    code |= rng.integers(1, 40, n) << 16
    code |= rng.integers(0, 8, n) << 24
    g["code"] = code.astype(np.uint32)
    g["t"] = rng.uniform(1.0, 300.0, n)
    g["d"] = rng.uniform(0.0, 96.0, n)
    g["fog"] = rng.uniform(0.0, 1500.0, n)
    return g


def rel_err(got, want):
    return float(np.linalg.norm(got - want) / max(np.linalg.norm(want), 1e-300))


def test_shading_params_layout():
    p = S.default_params()
    assert p.shape == (S.NPARAMS,) and p.dtype == np.float32
    assert np.all((p[:768] >= 0.1) & (p[:768] <= 0.9))
    assert np.allclose(p[S.P_SUN:S.P_SUN + 3], W.default_sun())
    assert p[S.P_FOG] == np.float32(0.002)
    assert np.allclose(p[S.P_ABS:S.P_ABS + 3], (0.45, 0.09, 0.06))
    q = S.perturbed(p)
    r = q.astype(np.float64) / p - 1.0
    assert 0.03 < r.std() < 0.07
    assert S.GBUF_DTYPE.itemsize == S.GBUF_BYTES


@pytest.mark.parametrize("seed", [0, 1])
def test_fp64_gradient_matches_central_differences(seed):
    g = synthetic_gbuffer(3000, seed)
    m = SO.Model(g, S.SUN_RGB)
    p = S.default_params().astype(np.float64)
    target = m.forward(S.perturbed(p.astype(np.float32), seed=12 + seed))
    grad = m.grad(p, target)
    rows = [3 * SO.WATER, 3 * SO.WATER + 2, 3 * 7 + 1, 3 * 20, 3 * 33 + 1]
    idx = rows + list(range(768, 778))
    # plain central differences carry an h^2 truncation term: 1e-4 relative,
    # except for the fog density (0.002, of which h = 1e-4 is 5%)
    fd = m.grad_fd(p, target, idx, h=1e-4)
    for j, i in enumerate(idx):
        if i != S.P_FOG:
            assert abs(fd[j] - grad[i]) <= GRAD_RTOL * max(abs(grad[i]), 1.0), (i, fd[j], grad[i])
    # with the h^2 term cancelled, every parameter agrees to 1e-5, the fog
    # density (an h^4 term of (rho L)^4 / rho^4 scale remains) to 1e-4
    fd = m.grad_fd(p, target, idx, h=1e-4, richardson=True)
    for j, i in enumerate(idx):
        tol = GRAD_RTOL if i == S.P_FOG else 1e-5
        assert abs(fd[j] - grad[i]) <= tol * max(abs(grad[i]), 1.0), (i, fd[j], grad[i])


def test_fp64_gradient_is_zero_at_the_target():
    g = synthetic_gbuffer(500, 5)
    m = SO.Model(g, S.SUN_RGB)
    p = S.default_params().astype(np.float64)
    assert np.abs(m.grad(p, m.forward(p))).max() == 0.0


# ---------------------------------------------------------------------------
# GPU
# ---------------------------------------------------------------------------
@pytest.fixture(scope="module")
def shading_batch():
    torch = pytest.importorskip("torch")
    from oracle.oracle import Oracle
    from voxelcraft_menu_b200.march import Marcher
    w = W.World.generate(W.recipe_small_terrain())
    pools = w.pools()
    m = Marcher(1920, 1080)
    m.upload_world(*pools)
    # two views at 240x135 around the small-terrain camera, one looking over the lake
    views = S.shade_views(w, n=4, width=240, height=135)[::2]
    m.batch_set(views)
    m.batch_run(secondary=True)
    k = S.consts()
    gb = S.gbuffer(m, k, torch)
    torch.cuda.synchronize()
    want, sec = [], []
    for v in views:
        o = Oracle(v, *pools)
        vis, _, _ = o.frame_vis()
        sh = o.shadow(vis)
        sk, st = o.secondary(vis)
        sec.append((sk, st))
        want.append(SO.gbuffer_from_oracle(o, vis, sh, sk, st, k.fog_falloff, k.fog_height))
    return torch, m, gb, np.concatenate(want), sec


def host_gbuffer(gb):
    return gb.cpu().numpy().view(S.GBUF_DTYPE)


@pytest.mark.gpu
def test_batch_secondary_rays_match_the_oracle(shading_batch):
    torch, m, gb, want, sec = shading_batch
    k, t = m.batch_read_secondary()
    assert np.array_equal(k, np.concatenate([s[0] for s in sec]))
    assert np.array_equal(t.view(np.uint32), np.concatenate([s[1] for s in sec]).view(np.uint32))
    # primary + shadow only: the graph of that mode is rebuilt and still agrees
    vis_sec, sh_sec = m.batch_read()
    m.batch_run()
    vis, sh = m.batch_read()
    assert np.array_equal(vis, vis_sec) and np.array_equal(sh, sh_sec)
    m.batch_run(secondary=True)


@pytest.mark.gpu
def test_gbuffer_matches_the_oracle(shading_batch):
    torch, m, gb, want, _ = shading_batch
    got = host_gbuffer(gb)
    assert got.shape == want.shape
    for f in ("code", "t", "d"):
        a, b = got[f].view(np.uint32), want[f].view(np.uint32)
        bad = np.flatnonzero(a != b)
        assert bad.size == 0, f"{f}: {bad.size} differ, first {bad[:5]} got {got[f][bad[:5]]} want {want[f][bad[:5]]}"
    # the fog length is float32 arithmetic with expf on the device, float64 here
    fog, ref = got["fog"].astype(np.float64), want["fog"]
    assert np.all(np.abs(fog - ref) <= 1e-5 * np.abs(ref))
    assert np.array_equal(fog == 0.0, (got["code"] & SO.G_HIT) == 0)
    code = got["code"]
    assert np.count_nonzero(code & SO.G_HIT2) > 100          # the lake is in view and refracted rays hit
    assert np.count_nonzero((code & SO.G_HIT) == 0) > 0       # and some sky


@pytest.mark.gpu
def test_forward_and_loss_match_fp64(shading_batch):
    torch, m, gb, _, _ = shading_batch
    k = S.consts()
    model = SO.Model(host_gbuffer(gb), S.SUN_RGB)
    p = S.default_params()
    pt = torch.from_numpy(p).cuda()
    color, _ = S.forward(gb, pt, k, torch)
    c64 = model.forward(p.astype(np.float64))
    assert np.abs(color.cpu().numpy() - c64).max() <= COLOR_ATOL
    target = torch.from_numpy(model.forward(S.perturbed(p)).astype(np.float32)).cuda()
    color2, loss = S.forward(gb, pt, k, torch, target=target)
    assert torch.equal(color, color2)
    l64 = model.loss(p.astype(np.float64), target.cpu().numpy())
    assert abs(loss.item() - l64) <= 1e-5 * l64


@pytest.mark.gpu
def test_gradient_matches_fp64(shading_batch):
    torch, m, gb, _, _ = shading_batch
    k = S.consts()
    model = SO.Model(host_gbuffer(gb), S.SUN_RGB)
    p = S.default_params()
    target = model.forward(S.perturbed(p)).astype(np.float32)
    grad, loss = S.backward(gb, torch.from_numpy(p).cuda(), k, torch, target=torch.from_numpy(target).cuda(),
                            with_loss=True)
    got = grad.cpu().numpy()
    want = model.grad(p.astype(np.float64), target)
    assert rel_err(got, want) <= GRAD_RTOL
    for name, sl in GROUPS.items():
        assert rel_err(got[sl], want[sl]) <= GRAD_RTOL, name
    l64 = model.loss(p.astype(np.float64), target)
    assert abs(loss.item() - l64) <= 1e-5 * l64


@pytest.mark.gpu
def test_rows_outside_the_column_table(shading_batch):
    """Block ids >= 16 take the shared-atomic path of the adjoint."""
    torch, m, gb, _, _ = shading_batch
    g = host_gbuffer(gb).copy()
    hit = (g["code"] & SO.G_HIT) != 0
    ids = g["code"] & 0xFF
    moved = hit & (ids != SO.WATER) & (np.arange(len(g)) % 3 == 0)
    g["code"] = np.where(moved, (g["code"] & ~np.uint32(0xFF)) | (ids + 100), g["code"]).astype(np.uint32)
    gb2 = torch.from_numpy(g.view(np.uint8).copy()).cuda()
    k = S.consts()
    model = SO.Model(g, S.SUN_RGB)
    p = S.default_params()
    target = model.forward(S.perturbed(p)).astype(np.float32)
    got = S.backward(gb2, torch.from_numpy(p).cuda(), k, torch, target=torch.from_numpy(target).cuda()).cpu().numpy()
    want = model.grad(p.astype(np.float64), target)
    assert np.abs(want[300:400]).max() > 0
    assert rel_err(got, want) <= GRAD_RTOL


@pytest.mark.gpu
def test_autograd_function(shading_batch):
    torch, m, gb, _, _ = shading_batch
    k = S.consts()
    Shade = S.make_function(torch)
    p = torch.from_numpy(S.default_params()).cuda().requires_grad_(True)
    color = Shade.apply(p, gb, k)
    wts = torch.randn(color.shape, device="cuda", generator=torch.Generator("cuda").manual_seed(4))
    (color * wts).sum().backward()
    # the same through the explicit pair (block partial sums are float32,
    # combined in an order that varies from run to run)
    grad = S.backward(gb, p.detach(), k, torch, grad_color=wts)
    assert p.grad.dtype == torch.float32
    assert torch.allclose(p.grad.double(), grad, rtol=1e-5, atol=1e-6)
    # and against FP64: d/dp sum(w * c) is the L2 loss gradient against c - w / 2
    model = SO.Model(host_gbuffer(gb), S.SUN_RGB)
    p64 = p.detach().cpu().double().numpy()
    w64 = wts.cpu().double().numpy()
    want = model.grad(p64, model.forward(p64) - w64 / 2.0)
    assert rel_err(grad.cpu().numpy(), want) <= GRAD_RTOL


@pytest.mark.gpu
def test_adam_fit_reduces_the_loss(shading_batch):
    torch, m, gb, _, _ = shading_batch
    k = S.consts()
    p0 = S.default_params()
    target, _ = S.forward(gb, torch.from_numpy(p0).cuda(), k, torch)
    p = torch.from_numpy(S.perturbed(p0)).cuda().requires_grad_(True)
    opt = torch.optim.Adam([p], lr=2e-3)
    Shade = S.make_function(torch)
    losses = []
    for _ in range(50):
        opt.zero_grad()
        loss = ((Shade.apply(p, gb, k) - target) ** 2).sum()
        loss.backward()
        opt.step()
        losses.append(loss.item())
    assert math.isfinite(losses[-1])
    assert losses[-1] < 0.2 * losses[0]
