"""Autotuner of the frame pipeline's persistent primary-ray kernel over its
launch shape: warps per block (4, 8), register budget (the resident warps per
SM the allocation must allow, REG_LEVELS), item shape / packet size (pixels
per lane: 1 = 8x4-pixel items, 2 = 8x8, PACKETS) and resident blocks per SM
(the occupancy maximum, or a fixed smaller count).  Every candidate's output
is compared with the first candidate's before its time counts, so tuning can
never change results."""
from __future__ import annotations

import hashlib

import numpy as np

from .march import PACKETS, PRIMARY_WARPS, REG_LEVELS, Marcher


def _time(run, reps: int = 5) -> float:
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


# resident blocks per SM tried besides the occupancy maximum (0), by warps per block
CTAS_PER_SM = {4: (0, 4), 8: (0, 2)}


def candidates():
    for warps in PRIMARY_WARPS:
        for level in REG_LEVELS:
            for packet in PACKETS:
                for per in CTAS_PER_SM[warps]:
                    yield warps, level, per, packet


def _tune(m: Marcher, run, read) -> dict:
    ref = None
    best = None
    for warps, level, per, packet in candidates():
        m.set_tuning(warps, level, per, packet)
        ms = _time(run)
        d = _digest(*read())
        if ref is None:
            ref = d
        if d != ref:
            raise RuntimeError(f"{warps} warps / register level {level} / {per} blocks per SM / packet {packet} "
                               "changed the output")
        if best is None or ms < best["ms"]:
            best = {"warps": warps, "reg_level": level, "ctas_per_sm": per, "packet": packet, "ms": ms}
    return best


def autotune_single(m: Marcher, view, warm=None) -> dict:
    """Fastest launch shape for vm_render on `view`."""
    if warm is not None:
        m.upload_view(warm)
        m.render()
    m.upload_view(view)
    return _tune(m, m.render, lambda: (m.read_vis(), m.read_shadow()))


def autotune_batch(m: Marcher) -> dict:
    """Fastest launch shape for the batched launch."""
    return _tune(m, m.batch_run, m.batch_read)
