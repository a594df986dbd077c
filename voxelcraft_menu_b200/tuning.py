"""Autotuner of the fused march: tile shape (8x8, 16x8, 16x16, 32x16 pixels
per CTA, i.e. 2 to 16 warps per block) and resident CTAs per SM of the
persistent launch.  Every candidate's output is checked against the first
candidate's before its time counts, so tuning can never change results."""
from __future__ import annotations

import hashlib

import numpy as np

from .march import TILE_SHAPES, Marcher


def _time(m: Marcher, run, reps: int = 5) -> float:
    import torch
    stream = torch.cuda.current_stream()
    run()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        run()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def _digest(*arrays) -> str:
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def candidates():
    for v in sorted(TILE_SHAPES):
        for per in (0, 1, 2, 4):
            yield v, per


def autotune_single(m: Marcher, view, warm=None) -> dict:
    """Fastest (variant, ctas_per_sm) for vm_render on `view`."""
    if warm is not None:
        m.upload_view(warm)
        m.render()
    m.upload_view(view)
    ref = None
    best = None
    for v, per in candidates():
        m.set_tuning(v, per)
        ms = _time(m, m.render)
        d = _digest(m.read_vis(), m.read_shadow())
        if ref is None:
            ref = d
        if d != ref:
            raise RuntimeError(f"tile variant {v} / {per} CTAs per SM changed the output")
        if best is None or ms < best["ms"]:
            best = {"variant": v, "ctas_per_sm": per, "ms": ms}
    return best


def autotune_batch(m: Marcher) -> dict:
    """Fastest (variant, ctas_per_sm) for the persistent batched launch."""
    ref = None
    best = None
    for v, per in candidates():
        m.set_tuning(v, per)
        ms = _time(m, m.batch_run, reps=3)
        vis, sh = m.batch_read()
        d = _digest(vis, sh)
        if ref is None:
            ref = d
        if d != ref:
            raise RuntimeError(f"tile variant {v} / {per} CTAs per SM changed the batch output")
        if best is None or ms < best["ms"]:
            best = {"variant": v, "ctas_per_sm": per, "ms": ms}
    return best
