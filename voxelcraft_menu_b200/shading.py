"""Differentiable shading over a fixed visibility buffer.

The forward / adjoint kernels (csrc/shade.cu, exported as vm_shade_forward /
vm_shade_backward) are bound here as a torch.autograd.Function for checking
and fitting.  Parameters are one float32 vector of VM_SHADE_NPARAMS entries:
albedo table 256 x 3, sun direction (normalised inside), sky ambient RGB, fog
density, water absorption RGB.  Traversal is never part of the graph: the
G-buffer of a batch (block ids, faces, shadow verdicts, hit distances, water
legs and fog lengths) is computed once, exactly, and the shading is a smooth
function of the parameters on top of it.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import world as W
from .native import lib

NPARAMS = 778
P_SUN, P_SKY, P_FOG, P_ABS = 768, 771, 774, 775
SUN_RGB = tuple(float(np.float32(v) * np.float32(0.78)) for v in (1.0, 0.8469, 0.5647))   # resolve.wgsl:787
GBUF_BYTES = 16
GBUF_DTYPE = np.dtype([("code", "<u4"), ("t", "<f4"), ("d", "<f4"), ("fog", "<f4")])   # vm_shade_gbuf


class ShadeConsts(C.Structure):
    _fields_ = [("sun_rgb", C.c_float * 3), ("fog_falloff", C.c_float), ("fog_height", C.c_float)]


def consts(fog_falloff: float = 0.01, fog_height: float = 64.0) -> ShadeConsts:
    k = ShadeConsts()
    k.sun_rgb[:] = SUN_RGB
    k.fog_falloff, k.fog_height = fog_falloff, fog_height
    return k


def pack_params(albedo, sun, sky, fog_density, absorb) -> np.ndarray:
    p = np.zeros(NPARAMS, np.float32)
    p[:768] = np.asarray(albedo, np.float32).reshape(-1)
    p[P_SUN:P_SUN + 3] = sun
    p[P_SKY:P_SKY + 3] = sky
    p[P_FOG] = fog_density
    p[P_ABS:P_ABS + 3] = absorb
    return p


def default_params(seed: int = 11) -> np.ndarray:
    """Albedo table U(0.1, 0.9) (seed 11), sun normalize(0.4, 0.8, 0.3), sky
    ambient (0.5, 0.7, 1.0), fog density 0.002, water absorption
    (0.45, 0.09, 0.06)."""
    rng = np.random.default_rng(seed)
    return pack_params(rng.uniform(0.1, 0.9, (256, 3)), W.default_sun(), (0.5, 0.7, 1.0), 0.002,
                       (0.45, 0.09, 0.06))


def perturbed(params: np.ndarray, seed: int = 12, scale: float = 0.05) -> np.ndarray:
    """params * (1 + scale * N(0, 1)) (seed 12): the target frames' parameters."""
    rng = np.random.default_rng(seed)
    return (params.astype(np.float64) * (1.0 + scale * rng.standard_normal(params.shape))).astype(np.float32)


def shade_views(world: W.World, cam_pos=(128.0, 110.0, 20.0), n: int = 8, width: int = 960, height: int = 540,
                pitch_deg: float = -15.0):
    """n views at width x height around cam_pos, yaw stepping by 360/n degrees."""
    return [world.view(W.Camera(pos=cam_pos, yaw=math.radians(90.0 + k * 360.0 / n), pitch=math.radians(pitch_deg),
                                width=width, height=height)) for k in range(n)]


def _stream(torch):
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def gbuffer(marcher, k: ShadeConsts, torch):
    """The G-buffer of marcher's current batch (run with secondary=True); the
    fog falloff and height of k fix its fog lengths."""
    n = marcher.batch_pixels()
    g = torch.empty(n * GBUF_BYTES, dtype=torch.uint8, device="cuda")
    marcher._ck(lib().vm_shade_gbuffer(marcher._h, C.byref(k), C.c_void_p(g.data_ptr())))
    marcher.sync()   # the pass runs on the context's stream; torch's stream reads g next
    return g


def forward(gbuf, params, k: ShadeConsts, torch, target=None):
    """Colours (n, 3) float32 and, with target, the L2 loss (float64)."""
    n = gbuf.numel() // GBUF_BYTES
    color = torch.empty((n, 3), dtype=torch.float32, device="cuda")
    loss = torch.zeros(1, dtype=torch.float64, device="cuda") if target is not None else None
    rc = lib().vm_shade_forward(C.c_void_p(gbuf.data_ptr()), n, C.c_void_p(params.data_ptr()), C.byref(k),
                                C.c_void_p(color.data_ptr()),
                                None if target is None else C.c_void_p(target.data_ptr()),
                                None if loss is None else C.c_void_p(loss.data_ptr()), _stream(torch))
    if rc:
        raise RuntimeError(f"vm_shade_forward failed ({rc})")
    return color, loss


def backward(gbuf, params, k: ShadeConsts, torch, grad_color=None, target=None, with_loss=False):
    """dL/dparams (float64) for dL/dcolour = grad_color, or for the L2 loss
    against target; with_loss (target only) also returns that loss (float64),
    from the same fused pass."""
    n = gbuf.numel() // GBUF_BYTES
    grad = torch.zeros(NPARAMS, dtype=torch.float64, device="cuda")
    loss = torch.zeros(1, dtype=torch.float64, device="cuda") if with_loss else None
    rc = lib().vm_shade_backward(C.c_void_p(gbuf.data_ptr()), n, C.c_void_p(params.data_ptr()), C.byref(k),
                                 None if grad_color is None else C.c_void_p(grad_color.data_ptr()),
                                 None if target is None else C.c_void_p(target.data_ptr()),
                                 C.c_void_p(grad.data_ptr()), None if loss is None else C.c_void_p(loss.data_ptr()),
                                 _stream(torch))
    if rc:
        raise RuntimeError(f"vm_shade_backward failed ({rc})")
    return (grad, loss) if with_loss else grad


def make_function(torch):
    """torch.autograd.Function over the forward / adjoint kernels."""

    class Shade(torch.autograd.Function):
        @staticmethod
        def forward(ctx, params, gbuf, k):
            p = params.detach().contiguous()
            color, _ = forward(gbuf, p, k, torch)
            ctx.save_for_backward(p, gbuf)
            ctx.k = k
            return color

        @staticmethod
        def backward(ctx, grad_color):
            p, gbuf = ctx.saved_tensors
            g = backward(gbuf, p, ctx.k, torch, grad_color=grad_color.contiguous().float())
            return g.to(p.dtype), None, None

    return Shade
