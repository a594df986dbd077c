"""Benchmark of the sparse-voxel-tree march on B200.

Workload (one step = one frame): 1920x1080 over the 1024x256x1024 synthetic
terrain (6-octave value noise, seed 7, water below y=64, 1% trees, ~3% glass
in the top two surface layers; 1024 chunks of 64^3), camera 30 above the
centre column looking +z, pitched -15 deg.  Frame A is rendered untimed; the
timed frames use the camera moved half a voxel along x with FLAG_HIZ on.
Every step marches the primary rays, one sun shadow ray per lit-facing hit
and one water-refraction / glass-transmission ray per water / glass hit.

Metric: Grays/s of primary + shadow rays (secondary rays are traced but not
counted).  `value` is measured on device-resident inputs; `e2e` goes through
the C ABI with host buffers (frame + chunk list + grid uploaded, visibility
keys and the shadow buffer in the engine's r16float target format read back
every step; `e2e_f32` reads the shadow back as float).  The library records CUDA events
between its stages during the timed steps (`stage_ms`); `roofline` is the
dominant kernel's algorithmic bytes per launch over its own event time.

More measurements share the JSON line: `shadow_filter` (the bilateral
soft-shadow reconstruction over the timed frame), `reflect` (the timed frame
with a reflect leg per water hit), `encoder` (the dense -> 64-tree encoder
over the terrain's 1024 chunks), `batched` (3072 probe cube faces
of 32^2..256^2 plus four 1920x1080 player views over the 256x128x256 world,
one graph-replayed persistent launch against one launch sequence per view,
primary + shadow), `shading` (forward, adjoint and fused loss + gradient
of the differentiable shading stage over 8 views at 960x540) and `sparse`
(64 ragged views over the 4096x256x4096 world with soft shadows and 8
Halton-jittered frames, then a 50-step Adam fit of the albedo table).

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
                       [--no-batch] [--no-shade] [--no-sparse] [--no-filter] [--no-cpu]
Under torchrun every rank renders its own copy (replicas: the march does not
shard a frame across GPUs); value is the total over ranks / max rank time.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "Grays/s at 1080p (primary + shadow rays)"
UNIT = "Grays/s"
WORKLOAD = ("1920x1080 frames over the 1024x256x1024 terrain (1024 chunks), camera moving 0.5 voxel per frame "
            "(Hi-Z from the frame before)")


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def max_over_ranks(ms, world, device):
    """The largest of the ranks' times: each replica times its own device,
    and the job's step ends when the slowest rank's does.  Every rank calls
    this at the same point (one all-reduce)."""
    if world <= 1:
        return float(ms)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_value(world, rays_per_rank, ms):
    """Whole-job Grays/s: every replica traces the same frame, so the job
    traces world x rays_per_rank rays per step of ms milliseconds."""
    return world * rays_per_rank / (ms * 1e-3) / 1e9


class ClockSampler:
    """SM clocks and throttle reasons sampled during the timed region: NVML
    reads every millisecond or so (read-only queries), else nvidia-smi every
    200 ms."""

    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, index: int):
        self.index = index
        self.samples = []      # (sm_mhz, max_mhz, set of reason names)
        self.source = None
        self._stop = threading.Event()
        self._t = None

    def _nvml(self):
        import pynvml as N
        N.nvmlInit()
        h = N.nvmlDeviceGetHandleByIndex(self.index)
        bits = [N.nvmlClocksEventReasonHwSlowdown, N.nvmlClocksEventReasonHwThermalSlowdown,
                N.nvmlClocksEventReasonSwThermalSlowdown, N.nvmlClocksEventReasonSwPowerCap]
        mx = N.nvmlDeviceGetMaxClockInfo(h, N.NVML_CLOCK_SM)
        self.source = "nvml"
        try:
            while not self._stop.is_set():
                sm = N.nvmlDeviceGetClockInfo(h, N.NVML_CLOCK_SM)
                r = N.nvmlDeviceGetCurrentClocksEventReasons(h)
                self.samples.append((float(sm), float(mx), {n for n, b in zip(self.NAMES, bits) if r & b}))
                self._stop.wait(0.001)
        finally:
            N.nvmlShutdown()

    def _smi(self):
        self.source = "nvidia-smi"
        q = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True,
                                     timeout=5).stdout.strip()
                f = [x.strip() for x in out.split(",")]
                if len(f) >= 6 and f[0].replace(".", "").isdigit():
                    self.samples.append((float(f[0]), float(f[1]),
                                         {n for n, v in zip(self.NAMES, f[2:6]) if "Active" in v and "Not" not in v}))
            except Exception:
                pass
            self._stop.wait(0.2)

    def start(self):
        def run():
            try:
                self._nvml()
            except Exception:
                if not self._stop.is_set():
                    self._smi()
        self._t = threading.Thread(target=run, daemon=True)
        self._t.start()
        time.sleep(0.005)   # first sample before the timed region

    def stop(self):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)
        sm = [x[0] for x in self.samples]
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(x[1] for x in self.samples) if self.samples else None,
                "reasons": sorted(set().union(*[x[2] for x in self.samples])) if self.samples else [],
                "samples": len(self.samples), "source": self.source}


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


FLAGS = 4 | 32 | 1     # FLAG_SHADOWS | FLAG_WATER_REFRACT | FLAG_HIZ


def l2_copy_gbs(dev, mb: int = 24, reps: int = 50) -> float:
    """Measured L2 bandwidth: a device copy between two mb-MB buffers that
    both stay in the 126 MB L2 (read + write bytes over CUDA-event time, best
    of five runs of reps copies, after a warm-up)."""
    import torch
    a = torch.empty(mb << 20, dtype=torch.uint8, device=dev)
    b = torch.empty_like(a)
    for _ in range(10):
        b.copy_(a)
    best = 0.0
    stream = torch.cuda.current_stream(dev)
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            b.copy_(a)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        best = max(best, 2 * a.numel() * reps / (e0.elapsed_time(e1) * 1e-3) / 1e9)
    return best


def build_workload():
    from voxelcraft_menu_b200 import world as W
    rec = W.recipe_large_terrain()
    w = W.World.generate(rec)
    pools = w.pools()
    view_a = w.view(W.large_terrain_camera(rec, flags=FLAGS))
    view_b = w.view(W.large_terrain_camera(rec, flags=FLAGS, dx=0.5))
    return w, pools, view_a, view_b


def mean_traffic(records):
    """Field-wise mean of vm_render_counted records (lists element-wise)."""
    out = {}
    for k, v in records[0].items():
        if isinstance(v, (list, tuple)):
            out[k] = [float(np.mean([r[k][i] for r in records])) for i in range(len(v))]
        else:
            out[k] = float(np.mean([r[k] for r in records]))
    return out


def oracle_workload():
    """The benchmark's frame pair built by the oracle's own producer (the
    engine's encoder, pools and chunk list restated in oracle/producer.cpp):
    the CPU legs never load the product library."""
    from oracle import producer as OP
    from voxelcraft_menu_b200 import world as W
    rec = W.recipe_large_terrain()
    ow = OP.OracleWorld.generate(rec)
    h = OP.surface_height(rec, 512, 512)
    flags = W.FLAG_SHADOWS | W.FLAG_WATER_REFRACT | W.FLAG_HIZ
    va, vb = (ow.view(W.Camera(pos=(512.0 + dx, float(h + 30), 512.0), width=1920, height=1080, flags=flags))
              for dx in (0.0, 0.5))
    return ow, ow.pools(), va, vb


class OracleFrames:
    """The oracle over the whole timed frame: frame B's visibility by the
    engine's pass sequence with frame A's Hi-Z, its shadow rays and its water
    / glass rays -- the work one GPU step does."""

    def __init__(self, pools, va, vb):
        from oracle.oracle import Oracle
        oa = Oracle(va, *pools)
        self.hiz_a = oa.frame_vis(hiz_in=np.zeros(oa.ntiles, np.uint32))[1]
        self.o = Oracle(vb, *pools)
        self.npix = self.o.npix

    def step(self):
        """One frame; returns (seconds, primary + shadow rays)."""
        t0 = time.perf_counter()
        vis, _, _, tr = self.o.frame_vis(hiz_in=self.hiz_a, traffic=True)
        _, tr2 = self.o.shadow(vis, traffic=True)
        self.o.secondary(vis)
        return time.perf_counter() - t0, tr["rays"] + tr2["rays"]


def cpu_sample(pools, va, vb, budget_s=10.0):
    """The oracle (the engine's pass sequence restated on the CPU) over whole
    frames of the timed workload, on every host core, until the budget is
    spent (at least one frame)."""
    fr = OracleFrames(pools, va, vb)
    t_total, rays, frames = 0.0, 0, 0
    while frames == 0 or t_total < budget_s:
        dt, r = fr.step()
        t_total += dt
        rays += r
        frames += 1
    # footnote baseline: the engine's own CPU ray walk (Player::pick, a
    # unit-voxel DDA over block lookups) per pixel of a few pixel rows
    height = int(vb.frame.res[1])
    t0 = time.perf_counter()
    n_pick, hits = fr.o.pick_rows(height // 2 - 64, 128)
    t_pick = time.perf_counter() - t0
    return {"value": rays / t_total / 1e9, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
            "sample": f"oracle (engine pass sequence restated in C++, OpenMP) over {frames} whole frames of the "
                      f"timed workload (frame B with frame A's Hi-Z, shadow and water / glass rays): "
                      f"{rays} primary+shadow rays in {t_total:.1f}s",
            "unit_voxel_walk": {"value": n_pick / t_pick / 1e9, "unit": "Grays/s (primary rays only)",
                                "sample": f"Player::pick (src/player.rs:334-393) restated, per pixel of 128 pixel rows "
                                          f"({n_pick} rays, {hits} hits) in {t_pick:.2f}s on every host core"}}


def reference_arm(args):
    """The engine's path on the CPU: the oracle restatement of its march over
    the same frame, with its world built by the oracle's producer; the whole
    frame every step (the GPU arm's pixel set), on every host core."""
    rank, world, _ = dist_env()
    if rank != 0:
        return
    _, pools, va, vb = oracle_workload()
    fr = OracleFrames(pools, va, vb)
    times, rays = [], 0
    for i in range(args.warmup + args.steps):
        dt, r = fr.step()
        if i >= args.warmup:
            times.append(dt)
            rays = r
    mean = float(np.mean(times))
    value = rays / mean / 1e9
    sample = (f"oracle over the whole frame every step ({fr.npix} pixels, {rays} primary+shadow rays, plus the "
              f"water / glass rays), world and chunk list from the oracle's producer")
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": mean * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic", "impl": "reference",
            "config": {"workload": WORKLOAD, "resolution": [1920, 1080], "chunks": int(len(vb.chunks)),
                       "l2": "host caches (the CPU arm flushes nothing)", "parallelism": "replicas x1"},
            "host_threads": os.cpu_count(),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": os.cpu_count(), "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# The library records five events per frame: before the prepass, after
# k_order, after k_primary, and two after the ray kernels.  The water / glass
# kernel and the shadow kernel run concurrently (the shadow kernel is a
# programmatic dependent launch behind it), so they form one timed stage,
# events 2 -> 4.
STAGES = {"cull": (0, 1), "primary": (1, 2), "shadow+secondary": (2, 4)}
STAGE_KERNELS = {"cull": "k_prepass + k_cull + k_order", "primary": "k_primary",
                 "shadow+secondary": "k_secondary_q + k_shadow (concurrent)"}


def stage_bytes(traffic, npix):
    """Algorithmic bytes per launch of each timed stage: the traversal's
    fetches (the layout's element sizes), plus what the stage reads and
    writes per ray: tile-list entries (2 B) and the visibility key (8 B) and
    queue items (24 B shadow, 40 B secondary) for the primary kernel; the
    queue item read and the 4 B result (12 B for a water / glass ray) for the
    two ray kernels."""
    sb = traffic["stage_bytes"]
    rs, rsec = traffic["rays_shadow"], traffic["rays_secondary"]
    return {
        "primary": sb[0] + 2 * traffic["list_entries"] + 8 * npix + 24 * rs + 40 * rsec,
        "shadow+secondary": sb[1] + (24 + 4) * rs + sb[2] + (40 + 12) * rsec,
    }


def stage_iters(traffic, stage):
    """DDA steps of a timed stage (the primary kernel, or both ray kernels)."""
    it = traffic["stage_iters"]
    return it[0] if stage == "primary" else it[1] + it[2]


def bench_batched(local, steps, warmup):
    """Probe cube captures and player views over the 256x128x256 world: one
    persistent graph-replayed launch against one launch sequence per view."""
    import torch
    from voxelcraft_menu_b200 import tuning
    from voxelcraft_menu_b200 import views as V
    from voxelcraft_menu_b200 import world as W
    from voxelcraft_menu_b200.march import Marcher
    w = W.World.generate(W.recipe_small_terrain())
    views = V.probe_views(w) + V.player_views(w)
    px = sum(v.n_pixels for v in views)
    m = Marcher(1920, 1080, device=local, max_views=len(views), max_batch_pixels=px)
    stream = torch.cuda.current_stream()
    m._ck(m._L.vm_set_stream(m._h, __import__("ctypes").c_void_p(stream.cuda_stream)))
    m.upload_world(*w.pools())
    m.batch_set(views)
    best = tuning.autotune_batch(m)
    m.set_tuning(best["warps"], best["reg_level"], best["ctas_per_sm"], best["packet"])
    traffic = m.batch_counted()
    rays = traffic["rays_primary"] + traffic["rays_shadow"]

    def timed(per_view):
        for _ in range(warmup):
            m.batch_run(per_view=per_view)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(steps):
            m.batch_run(per_view=per_view)
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps

    ms_batch = timed(False)
    out_batch = m.batch_read()
    ms_views = timed(True)
    out_views = m.batch_read()
    identical = all(np.array_equal(a, b) for a, b in zip(out_batch, out_views))
    m.close()
    return {"workload": f"{len(views)} views ({len(views) - 4} probe cube faces of 32^2..256^2 + 4 x 1920x1080 "
                        f"players) over the 256x128x256 world, primary + shadow rays",
            "pixels": px, "rays_per_step": rays, "value": rays / (ms_batch * 1e-3) / 1e9, "unit": UNIT,
            "ms_per_step": ms_batch, "per_view": {"value": rays / (ms_views * 1e-3) / 1e9, "ms_per_step": ms_views},
            "ratio": ms_views / ms_batch, "identical_output": identical, "tuning": best,
            "steps": steps, "warmup": warmup,
            "l2": "not flushed: each step writes 12 B x %d pixels (> 126 MB L2)" % px}


def bench_shading(local, steps, warmup):
    """Forward, adjoint and fused loss + gradient of the shading stage over 8
    views at 960x540 of the 256x128x256 world (one G-buffer, 4.15 Mpx)."""
    import torch
    from voxelcraft_menu_b200 import shading as S
    from voxelcraft_menu_b200 import world as W
    from voxelcraft_menu_b200.march import Marcher
    w = W.World.generate(W.recipe_small_terrain())
    views = S.shade_views(w)
    m = Marcher(1920, 1080, device=local, max_views=len(views), max_batch_pixels=sum(v.n_pixels for v in views))
    stream = torch.cuda.current_stream()
    m._ck(m._L.vm_set_stream(m._h, __import__("ctypes").c_void_p(stream.cuda_stream)))
    m.upload_world(*w.pools())
    m.batch_set(views)
    m.batch_run(secondary=True)
    k = S.consts()
    gb = S.gbuffer(m, k, torch)
    p0 = S.default_params()
    p = torch.from_numpy(p0).cuda()
    target, _ = S.forward(gb, torch.from_numpy(S.perturbed(p0)).cuda(), k, torch)
    gcol = torch.randn_like(target)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")

    def timed(fn):
        for _ in range(warmup):
            fn()
        ms = []
        for _ in range(steps):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fn()
            e1.record(stream)
            torch.cuda.synchronize()
            ms.append(e0.elapsed_time(e1))
        return float(np.mean(ms))

    n = len(views)
    fwd = timed(lambda: S.forward(gb, p, k, torch))
    fwd_loss = timed(lambda: S.forward(gb, p, k, torch, target=target))
    bwd = timed(lambda: S.backward(gb, p, k, torch, grad_color=gcol))
    fused = timed(lambda: S.backward(gb, p, k, torch, target=target, with_loss=True))
    npx = gb.numel() // S.GBUF_BYTES
    m.close()
    return {"workload": "8 views x 960x540 over the 256x128x256 world (4.15 Mpx), 778 parameters",
            "fwd_ms_per_view": fwd / n, "bwd_ms_per_view": bwd / n,
            "fwd_bwd_ms_per_view": (fwd + bwd) / n, "fwd_bwd_over_fwd": (fwd + bwd) / fwd,
            "loss_fwd_ms_per_view": fwd_loss / n, "fused_loss_grad_ms_per_view": fused / n,
            "fused_over_loss_fwd": fused / fwd_loss,
            "fwd_gbs": npx * (16 + 12) / (fwd * 1e-3) / 1e9, "fused_gbs": npx * (16 + 12) / (fused * 1e-3) / 1e9,
            "grad_check": "FP64 oracle gradient and central differences: tests/test_shading.py (rel err <= 1e-4)",
            "l2": "flushed between timed steps (256 MB write)"}


def bench_sparse(local, fit_steps=50):
    """The 4096x256x4096 sparse world (16384 chunk keys, more than one view's
    13-bit chunk field: every view carries its own chunk list and grid
    window): 64 ragged views of 256^2..1024^2 with soft shadows (4 jittered
    sun rays per hit), 8 frames of the Halton(2,3) jitter, then an inverse
    albedo fit of 50 FP32 Adam steps on the shading stage."""
    import torch
    from voxelcraft_menu_b200 import shading as S
    from voxelcraft_menu_b200 import tuning
    from voxelcraft_menu_b200 import views as V
    from voxelcraft_menu_b200 import world as W
    from voxelcraft_menu_b200.march import Marcher
    rec = W.recipe_sparse_world()
    w = W.World.generate(rec)
    flags = W.FLAG_SHADOWS | W.FLAG_WATER_REFRACT
    frames = [V.ragged_views(w, flags=flags, jitter=W.halton_jitter(k), frame_index=k) for k in range(8)]
    n_views = len(frames[0])
    px = sum(v.n_pixels for v in frames[0])
    m = Marcher(1024, 1024, device=local, max_views=n_views, max_batch_pixels=px)
    from voxelcraft_menu_b200.march import SPEC_DEFAULT, SPEC_SOFT_RAYS
    m.set_spec(SPEC_DEFAULT | SPEC_SOFT_RAYS)
    stream = torch.cuda.current_stream()
    m._ck(m._L.vm_set_stream(m._h, __import__("ctypes").c_void_p(stream.cuda_stream)))
    m.upload_world(*w.pools())
    m.batch_set(frames[0])
    best = tuning.autotune_batch(m)
    m.set_tuning(best["warps"], best["reg_level"], best["ctas_per_sm"], best["packet"])
    total_ms, rays, prim, shad = 0.0, 0, 0, 0
    for views in frames:
        m.batch_set(views)
        tr = m.batch_counted()
        prim += tr["rays_primary"]
        shad += tr["rays_shadow"]
        for _ in range(2):
            m.batch_run()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(3):
            m.batch_run()
        e1.record(stream)
        torch.cuda.synchronize()
        total_ms += e0.elapsed_time(e1) / 3
    rays = prim + shad
    # the inverse albedo fit on frame 0 (water legs traced for the G-buffer)
    m.batch_set(frames[0])
    m.batch_run(secondary=True)
    k = S.consts()
    gb = S.gbuffer(m, k, torch)
    p0 = S.default_params()
    target, _ = S.forward(gb, torch.from_numpy(p0).cuda(), k, torch)
    p = torch.from_numpy(S.perturbed(p0)).cuda().requires_grad_(True)
    opt = torch.optim.Adam([p], lr=2e-3)
    losses, ms_bwd, ms_step = [], [], []
    for _ in range(fit_steps):
        e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        e0.record(stream)
        g, loss = S.backward(gb, p.detach(), k, torch, target=target, with_loss=True)
        e1.record(stream)
        p.grad = g.float()
        opt.step()
        e2.record(stream)
        torch.cuda.synchronize()
        losses.append(loss.item())
        ms_bwd.append(e0.elapsed_time(e1))
        ms_step.append(e0.elapsed_time(e2))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(10):
        S.forward(gb, p.detach(), k, torch)
    e1.record(stream)
    torch.cuda.synchronize()
    fwd = e0.elapsed_time(e1) / 10
    m.close()
    return {"workload": f"{n_views} views of 256^2..1024^2 ({px} pixels per frame) over the 4096x256x4096 sparse "
                        f"world ({int(w.pool_stats().n_chunks)} chunks), soft shadows (4 rays per hit), "
                        f"8 Halton-jittered frames", "unit": UNIT,
            "value": rays / (total_ms * 1e-3) / 1e9, "ms_per_frame": total_ms / 8,
            "rays_per_frame": {"primary": prim // 8, "soft_shadow": shad // 8}, "tuning": best,
            "fit": {"steps": fit_steps, "loss_first": losses[0], "loss_last": losses[-1],
                    "fused_loss_grad_ms_per_view": float(np.mean(ms_bwd[5:])) / n_views,
                    "adam_step_ms": float(np.mean(ms_step[5:])), "fwd_ms_per_view": fwd / n_views,
                    "grad_check": "FP64 oracle gradient on sparse-world views: tests/test_sparse_soft.py"}}


def bench_filter(m, vb, pools, stream, flush, steps, warmup, cpu=True):
    """The bilateral soft-shadow reconstruction (vm_soften_shadows) over the
    timed 1080p frame's visibility and blocker distances, at the engine's two
    radius limits (4 with SOFT_PENUMBRA 1.5, 8 with 3.0).  Algorithmic bytes
    per launch: 16 per pixel (8 key + 4 distance read, 4 mask written)."""
    import torch
    peak, peak_kind = peaks()
    npix = int(vb.frame.res[0]) * int(vb.frame.res[1])
    m.upload_view(vb)
    m.render()                       # the filter's input: frame B's keys and blocker distances
    out = {"workload": "1920x1080 timed frame of the 1024x256x1024 terrain: its keys and blocker distances",
           "l2": "flushed between timed steps (256 MB write)"}
    for limit, pen in ((4, 1.5), (8, 3.0)):
        for _ in range(warmup):
            m.soften_shadows(limit, pen)
        ms = []
        for _ in range(steps):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            m.soften_shadows(limit, pen)
            e1.record(stream)
            torch.cuda.synchronize()
            ms.append(e0.elapsed_time(e1))
        t = float(np.mean(ms))
        mask = m.read_shadow_mask()
        gbs = 16 * npix / (t * 1e-3) / 1e9
        rec = {"us": t * 1e3, "mpx_per_s": npix / (t * 1e-3) / 1e6, "soft_pixels": int(((mask > 0) & (mask < 1)).sum()),
               "roofline": {"bound": "hbm", "achieved": gbs, "peak": peak, "unit": "GB/s", "frac": gbs / peak,
                            "peak_kind": peak_kind, "algorithmic_bytes_per_launch": 16 * npix,
                            "traffic": profile_traffic("soften") if limit == 4 else None}}
        if cpu:
            from oracle.oracle import Oracle
            vis, dist = m.read_vis(), m.read_shadow()
            o = Oracle(vb, *pools)
            t0 = time.perf_counter()
            _, ref = o.soften(vis, dist, limit, pen)
            rec["cpu_oracle_ms"] = (time.perf_counter() - t0) * 1e3
            rec["cpu_cores"] = os.cpu_count()
            rec["max_abs_diff_vs_oracle"] = float(np.abs(ref - mask).max())
        out[f"limit{limit}_penumbra{pen}"] = rec
    return out


def bench_reflect(m, w, stream, flush, steps, warmup):
    """The timed 1080p frame with FLAG_WATER_REFLECT: every water hit also
    traces its reflect leg (reflect(rd, n), 768 voxels) on the secondary
    lanes.  Frame time (CUDA events around vm_render) and reflect rays."""
    import torch
    from voxelcraft_menu_b200 import world as W
    rec = W.recipe_large_terrain()
    flags = W.FLAG_SHADOWS | W.FLAG_WATER_REFRACT | W.FLAG_HIZ | W.FLAG_WATER_REFLECT
    m.upload_view(w.view(W.large_terrain_camera(rec, flags=flags, dx=0.5)))
    for _ in range(warmup):
        m.render()
    ms = []
    for _ in range(steps):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        m.render()
        e1.record(stream)
        torch.cuda.synchronize()
        ms.append(e0.elapsed_time(e1))
    k, _ = m.read_reflection()
    sk, _ = m.read_secondary()
    return {"workload": "the timed 1920x1080 frame with FLAG_WATER_REFLECT (reflect leg per water hit)",
            "ms_per_frame": float(np.mean(ms)),
            "reflect_rays": int(((k >> np.uint64(63)) & np.uint64(1)).sum()),
            "refract_and_glass_rays": int(((sk >> np.uint64(63)) & np.uint64(1)).sum()),
            "l2": "flushed between timed steps (256 MB write)"}


def bench_resolve(m, w, pools, stream, flush, steps, warmup, cpu=True):
    """The resolve (vm_resolve: sky, opaque surfaces, water with its shared
    legs and glass, with the engine's default look, probe field and shaft
    envelope) over the timed 1080p frame.  Algorithmic bytes per call: 28 per
    pixel (8 key + 4 shadow read, 16 RGBA written); the material gathers
    (chunk records, light, tree nodes, atlas, probes, shaft) are L2-resident.
    The oracle is timed on a bounded sample of rows and compared there."""
    import torch
    from oracle.oracle import Oracle
    from voxelcraft_menu_b200 import look as LK
    from voxelcraft_menu_b200 import world as W
    rec = W.recipe_large_terrain()
    flags = W.FLAG_SHADOWS | W.FLAG_WATER_REFRACT | W.FLAG_HIZ | LK.LOOK_FLAGS
    v = w.view(W.large_terrain_camera(rec, flags=flags, dx=0.5))
    LK.apply_defaults(v.frame, rec.seed)
    look = (LK.atlas(rec.seed), LK.block_faces(), LK.probe_field(rec.seed),
            LK.shaft_envelope(rec, v.frame.sun_dir, v.frame.shaft_origin, 4.0))
    m.upload_view(v)
    m.upload_look(*look)
    m.render()
    for _ in range(warmup):
        m.resolve(LK.HI_DEFAULT)
    ms = []
    for _ in range(steps):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        m.resolve(LK.HI_DEFAULT)
        e1.record(stream)
        torch.cuda.synchronize()
        ms.append(e0.elapsed_time(e1))
    t = float(np.mean(ms))
    npix = v.n_pixels
    peak, peak_kind = peaks()
    gbs = 28 * npix / (t * 1e-3) / 1e9
    out = {"workload": "the timed 1920x1080 frame of the 1024x256x1024 terrain, the engine's default look "
                       "(fog, clouds, god rays, biome tint, probes, shaft envelope)",
           "l2": "flushed between timed steps (256 MB write)", "us": t * 1e3, "gpx_per_s": npix / (t * 1e-3) / 1e9,
           "roofline": {"bound": "hbm", "achieved": gbs, "peak": peak, "unit": "GB/s", "frac": gbs / peak,
                        "peak_kind": peak_kind, "algorithmic_bytes_per_launch": 28 * npix,
                        "traffic": profile_traffic("resolve"),
                        "note": "issue-bound: per pixel the transcendental-heavy look (sky, clouds, shafts, "
                                "noise) and a 9-sample light gather over L2-resident tables"}}
    if cpu:
        color = m.read_color()
        vis, sh = m.read_vis(), m.read_shadow()
        o = Oracle(v, *pools)
        rows = 68                                  # a band of 68 rows through the frame's centre
        p0, p1 = 506 * 1920, (506 + rows) * 1920
        t0 = time.perf_counter()
        ref = o.resolve(vis, LK.sun_visibility(sh), *look, spec_hi=LK.HI_DEFAULT, pix=(p0, p1))
        dt = time.perf_counter() - t0
        out["cpu_oracle"] = {"sample": f"{rows} rows ({p1 - p0} pixels) of the frame", "s": dt,
                             "mpx_per_s": (p1 - p0) / dt / 1e6, "cores": os.cpu_count(),
                             "max_abs_diff": float(np.abs(ref - color[p0:p1]).max())}
    return out


def bench_encoder(local, steps, warmup, cpu=True):
    """The dense -> 64-tree encoder (vm_encode_trees) over every chunk of the
    1024x256x1024 terrain (1024 dense 64^3 chunks, 512 MB of block ids
    resident on the device); the engine's own measurement of its CPU encoder
    is 1325.9 us per chunk (its --bench-terrain "tree build")."""
    import torch
    from voxelcraft_menu_b200 import encode as E
    from voxelcraft_menu_b200 import world as W
    dense = W.recipe_dense_chunks(W.recipe_large_terrain())
    n = len(dense)
    d = torch.from_numpy(dense.view(np.int16)).to(f"cuda:{local}")
    cap = 16384
    out = E.DeviceTrees(n, cap, torch, d.device)
    stream = torch.cuda.current_stream(d.device)
    for _ in range(warmup):
        E.gpu_encode(d, n, cap, torch, out)
    ms = []
    for _ in range(steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        E.gpu_encode(d, n, cap, torch, out)
        e1.record(stream)
        torch.cuda.synchronize()
        ms.append(e0.elapsed_time(e1))
    t = float(np.mean(ms))
    host = out.to_host()
    out_bytes = int(n * (64 + 8 + 4) + 24 * host.info["n_l1"].sum() + 8 * host.info["n_leaves"].sum() +
                    4 * host.info["n_attrs"].sum() + 4 * host.info["n_palette"].sum())
    algo = n * 64 ** 3 * 2 + out_bytes
    peak, peak_kind = peaks()
    rec = {"workload": "1024 dense 64^3 chunks of the 1024x256x1024 terrain (512 MB of u16 block ids on the device)",
           "ms": t, "us_per_chunk": t * 1e3 / n, "chunks_per_s": n / (t * 1e-3),
           "roofline": {"bound": "hbm", "achieved": algo / (t * 1e-3) / 1e9, "peak": peak, "unit": "GB/s",
                        "frac": algo / (t * 1e-3) / 1e9 / peak, "peak_kind": peak_kind,
                        "algorithmic_bytes_per_launch": algo,
                        "traffic": profile_traffic("encode", "1024_chunks")},
           "reference_cpu_us_per_chunk": 1325.9,
           "l2": "not flushed: the 512 MB input is larger than L2"}
    if cpu:
        sample = dense[::16]
        t0 = time.perf_counter()
        E.cpu_build(sample, cap)
        rec["cpu_restatement_us_per_chunk"] = (time.perf_counter() - t0) * 1e6 / len(sample)
        rec["cpu_sample"] = f"{len(sample)} of the chunks, one host thread (vmw_build_tree)"
    return rec


def profile_row(kernel, row, workload="1080p"):
    """A value of the committed ncu summary's table (e.g. "issue active"), if any."""
    f = ROOT / "profiles" / f"k_{kernel}_{workload}.md"
    if not f.exists():
        return None
    for line in f.read_text().splitlines():
        cells = [c.strip() for c in line.strip().strip("|").split("|")]
        if len(cells) == 2 and cells[0] == row:
            return cells[1]
    return None


def profile_traffic(kernel, workload="1080p"):
    """dram bytes per launch of kernel from the committed ncu summary, if any."""
    f = ROOT / "profiles" / f"k_{kernel}_{workload}.md"
    if not f.exists():
        return None
    for line in f.read_text().splitlines():
        if line.startswith("traffic_bytes_per_launch:"):
            return float(line.split(":", 1)[1])
    return None


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--warps", type=int, default=0, help="primary kernel warps per block (0: autotune)")
    ap.add_argument("--reg-level", type=int, default=0, help="primary kernel register level with --warps")
    ap.add_argument("--packet", type=int, default=1, help="primary kernel pixels per lane with --warps")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched probe views")
    ap.add_argument("--no-shade", action="store_true", help="skip the shading forward / adjoint")
    ap.add_argument("--no-sparse", action="store_true", help="skip the sparse-world views and the fit")
    ap.add_argument("--no-filter", action="store_true", help="skip the shadow filter, reflect frame and encoder")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return reference_arm(args)

    import torch
    import torch.distributed as dist
    rank, world, local = dist_env()
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)

    from voxelcraft_menu_b200.march import Marcher
    from voxelcraft_menu_b200 import tuning
    from voxelcraft_menu_b200 import world as W

    rec = W.recipe_large_terrain()
    w, pools, va, vb = build_workload()
    m = Marcher(1920, 1080, device=local)
    # the library enqueues on torch's (non-default) current stream, so torch's
    # CUDA events bracket exactly the march's launches
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    m._ck(m._L.vm_set_stream(m._h, __import__("ctypes").c_void_p(stream.cuda_stream)))
    m.upload_world(*pools)

    # warps per block / register budget of the primary kernel: autotuned on this frame unless fixed
    if args.warps > 0:
        best = {"warps": args.warps, "reg_level": args.reg_level, "ctas_per_sm": 0, "packet": args.packet}
    else:
        best = tuning.autotune_single(m, vb, warm=va)
    m.set_tuning(best["warps"], best["reg_level"], best["ctas_per_sm"], best["packet"])

    # A moving camera: frame A at the centre, then one view per step, each 0.5
    # voxel further along x (the first is frame B), so every timed frame's
    # Hi-Z and primary cost order come from the frame before it, as in a
    # renderer.  Each view's chunk list, grid and frame are uploaded from
    # page-locked memory on the stream before the step's first event.
    import ctypes as C
    L = m._L
    path = [vb] + [w.view(W.large_terrain_camera(rec, flags=FLAGS, dx=0.5 * (k + 2)))
                   for k in range(args.warmup + args.steps - 1)]
    pinned = [(torch.from_numpy(v.chunks.view(np.uint8).copy()).pin_memory(),
               torch.from_numpy(v.grid.view(np.int32).copy()).pin_memory()) for v in path]

    def put(c, k):
        v, (ch, gr) = path[k], pinned[k]
        c._ck(L.vm_upload_chunks(c._h, C.c_void_p(ch.data_ptr()), len(v.chunks), C.c_void_p(gr.data_ptr()),
                                 v.grid.size))
        c._ck(L.vm_set_frame(c._h, C.byref(v.frame)))

    timed_views = range(args.warmup, args.warmup + args.steps)
    counted = []
    for k in timed_views:
        put(m, k - 1)
        m.render()
        put(m, k)
        counted.append(m.render_counted())
    traffic = mean_traffic(counted)
    m.upload_view(va)
    m.render()
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)   # > 126 MB L2

    for k in range(args.warmup):
        put(m, k)
        m.render()
    torch.cuda.synchronize(dev)
    # five events per step, recorded by the library between its stages (STAGES)
    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(5)] for _ in range(args.steps)]
    for row in evs:
        for e in row:
            e.record(stream)   # creates the underlying CUDA event
    torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
    sampler = ClockSampler(local)
    sampler.start()
    torch.cuda.synchronize(dev)
    for i in range(args.steps):
        flush.zero_()
        put(m, args.warmup + i)
        m.render_events([e.cuda_event for e in evs[i]])
    torch.cuda.synchronize(dev)
    clocks = sampler.stop()
    m.upload_view(vb)
    ms = [row[0].elapsed_time(row[4]) for row in evs]
    stage_ms = {name: float(np.mean([row[i].elapsed_time(row[j]) for row in evs]))
                for name, (i, j) in STAGES.items()}
    ms_step = max_over_ranks(float(np.mean(ms)), world, dev)
    if world > 1:
        dist.barrier()

    filt = bench_filter(m, vb, pools, stream, flush, max(5, min(args.steps, 20)), 3,
                        cpu=not args.no_cpu and rank == 0) if not args.no_filter else None
    refl = bench_reflect(m, w, stream, flush, max(5, min(args.steps, 20)), 3) if not args.no_filter else None
    resolve = bench_resolve(m, w, pools, stream, flush, max(5, min(args.steps, 20)), 3,
                            cpu=not args.no_cpu and rank == 0) if not args.no_filter else None

    npix = 1920 * 1080
    rays = traffic["rays_primary"] + traffic["rays_shadow"]
    value = job_value(world, rays, ms_step)

    # e2e through the C ABI with host buffers (pinned), per step: frame + chunk
    # list + grid up, render, vis + shadow down
    vis_h = torch.empty(npix, dtype=torch.int64).pin_memory()
    sh_h = torch.empty(npix, dtype=torch.float32).pin_memory()
    ch_h = torch.from_numpy(vb.chunks.view(np.uint8).copy()).pin_memory()
    gr_h = torch.from_numpy(vb.grid.view(np.int32).copy()).pin_memory()

    def e2e_step():
        m._ck(L.vm_upload_chunks(m._h, C.c_void_p(ch_h.data_ptr()), len(vb.chunks), C.c_void_p(gr_h.data_ptr()),
                                 vb.grid.size))
        m._ck(L.vm_set_frame(m._h, C.byref(vb.frame)))
        m._ck(L.vm_render(m._h))
        m._ck(L.vm_read_vis(m._h, C.c_void_p(vis_h.data_ptr())))
        m._ck(L.vm_read_shadow(m._h, C.c_void_p(sh_h.data_ptr())))

    for _ in range(3):
        e2e_step()
    e_ms = []
    for i in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize(dev)
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        e2e_step()
        ev1.record(stream)
        torch.cuda.synchronize(dev)
        e_ms.append(ev0.elapsed_time(ev1))
    e2e_serial_ms = max_over_ranks(float(np.mean(e_ms)), world, dev)

    # e2e as a renderer runs consecutive frames: two contexts alternate; each
    # step renders its frame after the other context's last render
    # (vm_wait_render), uploads the next frame's chunk list, grid and frame
    # from page-locked host memory to the other context, and enqueues its own
    # visibility + shadow read-back into page-locked host memory
    # (vm_read_async_r16f: the shadow in the engine's R16F target format; and
    # vm_read_async: as float); a step's read-back overlaps the next step's
    # kernels.  Device time from an event before the first step to the later
    # of the two streams' ends, over the steps.
    m2 = Marcher(1920, 1080, device=local)
    m2.upload_world(*pools)
    m2.set_tuning(best["warps"], best["reg_level"], best["ctas_per_sm"], best["packet"])
    m2.upload_view(va)
    m2.render()
    ctxs = (m, m2)
    m._ck(L.vm_set_stream(m._h, None))   # both contexts on their own streams
    streams = [torch.cuda.ExternalStream(c.device_buffers().stream, device=dev) for c in ctxs]

    def e2e_two_contexts(r16f):
        """ms per step; r16f: the shadow read back in the engine's R16F
        target format (vm_read_async_r16f), else as float (vm_read_async)."""
        sh_dtype = torch.int16 if r16f else torch.float32
        host = [(torch.empty(npix, dtype=torch.int64).pin_memory(), torch.empty(npix, dtype=sh_dtype).pin_memory())
                for _ in ctxs]
        read = L.vm_read_async_r16f if r16f else L.vm_read_async

        def step(i):
            # frame i (view i of the camera path) on context i % 2, its inputs
            # uploaded by the step before
            c, other = ctxs[i % 2], ctxs[(i + 1) % 2]
            vh, shh = host[i % 2]
            # this frame's kernels start once the previous frame's are done
            # (not its read-back): each frame has the whole GPU while the
            # previous one's result crosses the host link
            c._ck(L.vm_wait_render(c._h, other._h))
            c._ck(L.vm_render(c._h))
            # the next frame's inputs, enqueued ahead of this frame's
            # read-back so that the small upload does not queue behind it
            put(other, (i + 1) % len(path))
            c._ck(read(c._h, C.c_void_p(vh.data_ptr()), C.c_void_p(shh.data_ptr())))

        put(ctxs[0], 0)
        for i in range(4):
            step(i)
        torch.cuda.synchronize(dev)
        start = torch.cuda.Event(enable_timing=True)
        start.record(streams[0])
        streams[1].wait_event(start)
        for i in range(4, 4 + args.steps):
            step(i)
        ends = [torch.cuda.Event(enable_timing=True) for _ in ctxs]
        for e, st in zip(ends, streams):
            e.record(st)
        torch.cuda.synchronize(dev)
        ms_ = max(start.elapsed_time(e) for e in ends) / args.steps
        # the last two frames read back equal those views rendered alone
        last = 4 + args.steps - 1
        for i in (last - 1, last):
            m2.upload_view(path[i % len(path)])
            m2.render()
            vh, shh = host[i % 2]
            assert np.array_equal(vh.numpy().view(np.uint64), m2.read_vis())
            want = m2.read_shadow()
            want = want.astype(np.float16).view(np.int16) if r16f else want
            assert np.array_equal(shh.numpy(), want)
        return max_over_ranks(ms_, world, dev)

    e2e_ms = e2e_two_contexts(True)
    e2e_f32_ms = e2e_two_contexts(False)
    m2.close()
    h2d = int(np.mean([v.chunks.nbytes + v.grid.nbytes for v in path])) + 352
    d2h = npix * (8 + 2)       # vis keys + binary16 blocker distances
    d2h_f32 = npix * (8 + 4)

    # roofline of the dominant kernel: its algorithmic bytes per launch over
    # its own event-timed duration
    sbytes = stage_bytes(traffic, npix)
    top = max(sbytes, key=lambda k: stage_ms[k])
    peak, peak_kind = peaks()
    achieved = sbytes[top] / (stage_ms[top] * 1e-3) / 1e9
    l2_peak = l2_copy_gbs(dev)
    stats = m.stats()
    m.close()
    extra = {}
    if rank == 0 and not args.no_batch:
        extra["batched"] = bench_batched(local, max(3, min(args.steps, 5)), 3)
    if rank == 0 and not args.no_shade:
        extra["shading"] = bench_shading(local, max(5, min(args.steps, 20)), 5)
    if rank == 0 and not args.no_sparse:
        extra["sparse"] = bench_sparse(local)
    if rank == 0 and not args.no_filter:
        extra["encoder"] = bench_encoder(local, max(5, min(args.steps, 20)), 3, cpu=not args.no_cpu)
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "resolution": [1920, 1080], "chunks": int(len(vb.chunks)),
                       "l2": "flushed between timed steps (256 MB write)", "parallelism": f"replicas x{world}"},
            "tuning": best,
            "stage_ms": stage_ms,
            "work_per_step": traffic,
            "rays_per_step": {"primary": traffic["rays_primary"], "shadow": traffic["rays_shadow"],
                              "secondary_uncounted": traffic["rays_secondary"]},
            "roofline": {"bound": "hbm", "kernel": STAGE_KERNELS[top],
                         "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": profile_traffic(top), "peak_kind": peak_kind,
                         "note": "the tree pools are L2-resident: the kernel is bound by instruction issue, "
                                 "not HBM (ncu issue active and threads per instruction below)",
                         "issue_active_ncu": profile_row(top, "issue active"),
                         "threads_per_instruction_ncu": profile_row(top, "threads per executed instruction (of 32)"),
                         "algorithmic_bytes_per_launch": sbytes[top], "launch_ms": stage_ms[top],
                         "dda_steps_per_launch": stage_iters(traffic, top),
                         "bytes_per_dda_step": sbytes[top] / max(stage_iters(traffic, top), 1),
                         "l2": {"achieved": achieved, "peak": l2_peak, "unit": "GB/s", "frac": achieved / l2_peak,
                                "peak_kind": "measured here: device copy between two 24 MB buffers resident in L2",
                                "note": "the bound the tree pools (L2-resident) would set"}},
            "e2e": {"value": job_value(world, rays, e2e_ms), "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "ms_per_step": e2e_ms,
                    "method": "two contexts alternate; every step renders once the other context's last render is "
                              "done (vm_wait_render), uploads the next step's inputs from pinned host memory ahead "
                              "of its own read-back, and reads vis (u64 keys) + shadow back in the engine's own "
                              "formats (the shadow target is r16float, shadow.wgsl:1; vm_read_async_r16f), "
                              "overlapping the next step's kernels"},
            "e2e_f32": {"value": job_value(world, rays, e2e_f32_ms), "unit": UNIT, "h2d_bytes_per_step": h2d,
                        "d2h_bytes_per_step": d2h_f32, "ms_per_step": e2e_f32_ms,
                        "method": "as e2e, the shadow read back as float (vm_read_async)"},
            "e2e_serial": {"value": job_value(world, rays, e2e_serial_ms), "unit": UNIT,
                           "ms_per_step": e2e_serial_ms,
                           "method": "one context, synchronous read-back, L2 flushed before each step"},
            # per frame: k_prepass, k_cull, k_order, k_primary, k_shadow, k_secondary_q
            "gpu_launches": 6 * args.steps,
            "clocks": clocks,
            "device_error": int(stats.device_error),
        }
        if filt is not None:
            line["shadow_filter"] = filt
        if refl is not None:
            line["reflect"] = refl
        if resolve is not None:
            line["resolve"] = resolve
        line.update(extra)
        if not args.no_cpu:
            _, o_pools, o_va, o_vb = oracle_workload()
            line["cpu_baseline"] = cpu_sample(o_pools, o_va, o_vb)
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
