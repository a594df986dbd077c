"""The march behind the engine's renderer interface.

`Renderer` mirrors the engine's `Renderer` for this path
(src/render/mod.rs:747-2060): `sync_world`, `build_chunk_list`, `render` and
the `march_stats` / `pair_demand` read-backs, each a thin call into the C ABI
of include/voxmarch.h.  Every call raises `MarchError` when the library
reports an error; there is no CPU path.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import native
from .native import VmCaps, VmDevicePtrs, VmFrame, VmStats, VmTraffic, lib, ptr
from .world import FLAG_HIZ, View, World

VM_OK = 0
STATUS = {0: "VM_OK", 1: "VM_E_INVALID", 2: "VM_E_CAPACITY", 3: "VM_E_TILE_OVERFLOW", 4: "VM_E_ITER_CAP",
          5: "VM_E_TIMEOUT", 6: "VM_E_CUDA", 7: "VM_E_NOT_READY", 8: "VM_E_TOO_LARGE"}

# warps per block and register levels of the persistent primary-ray kernel (vm_set_tuning)
PRIMARY_WARPS = (4, 8)
REG_LEVELS = (0, 1, 2, 3, 4)
PACKETS = (1, 2)
# pipeline specialisations (VM_SPEC_* of vm_types.h)
SPEC_FULL_MARCH, SPEC_WATER_REPAIR, SPEC_LEAF_CUTOUT, SPEC_GLASS = 1, 2, 4, 8
SPEC_EMITTER_GATHER, SPEC_FOLIAGE, SPEC_SNELL_BEND, SPEC_LEAF_THIN = 16, 32, 64, 128
SPEC_DEFAULT = SPEC_FULL_MARCH | SPEC_WATER_REPAIR | SPEC_LEAF_CUTOUT | SPEC_GLASS | SPEC_EMITTER_GATHER | \
    SPEC_FOLIAGE | SPEC_LEAF_THIN
SPEC_SOFT_RAYS = 256      # extension: VM_SOFT_SAMPLES jittered sun rays per hit, blocked fraction


class MarchError(RuntimeError):
    def __init__(self, code: int, text: str):
        super().__init__(f"{STATUS.get(code, code)}: {text}")
        self.code = code


@dataclass
class PairDemand:
    """src/render/mod.rs:41-60"""
    select: int
    deferred: int
    recover: int
    cap: int

    def overflowed(self) -> bool:
        return self.select > self.cap or self.deferred > self.cap or self.recover > self.cap


class Marcher:
    """One vm_ctx: the device state of one renderer."""

    def __init__(self, max_width: int, max_height: int, device: int = 0, max_chunks: int = 8191, max_views: int = 0,
                 max_batch_pixels: int = 0):
        self._L = lib()
        caps = VmCaps(max_width, max_height, max_chunks, max_views, max_batch_pixels)
        h = C.c_void_p()
        rc = self._L.vm_create(device, C.byref(caps), C.byref(h))
        if rc:
            raise MarchError(rc, "vm_create failed (no CUDA device?)")
        self._h = h
        self.view: View | None = None

    def close(self):
        if self._h:
            self._L.vm_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ck(self, rc: int):
        if rc != VM_OK:
            raise MarchError(rc, self._L.vm_last_error(self._h).decode())

    # -- inputs -------------------------------------------------------------
    def upload_world(self, inners: np.ndarray, leaves: np.ndarray, bricks: np.ndarray):
        i = np.ascontiguousarray(inners, np.uint32)
        l = np.ascontiguousarray(leaves, np.uint32)
        b = np.ascontiguousarray(bricks, np.uint32)
        self._ck(self._L.vm_upload_world(self._h, ptr(i), i.size // 4, ptr(l), l.size // 2, ptr(b), b.size))

    def update_pool(self, pool: int, offset: int, data: np.ndarray):
        d = np.ascontiguousarray(data, np.uint32)
        per = (4, 2, 1)[pool]
        self._ck(self._L.vm_update_pool(self._h, pool, offset, ptr(d), d.size // per))

    def upload_view(self, v: View):
        ch = np.ascontiguousarray(v.chunks)
        g = np.ascontiguousarray(v.grid, np.uint32)
        self._ck(self._L.vm_upload_chunks(self._h, ptr(ch), len(ch), ptr(g), g.size))
        self._ck(self._L.vm_set_frame(self._h, C.byref(v.frame)))
        self.view = v

    def set_frame(self, frame: VmFrame):
        self._ck(self._L.vm_set_frame(self._h, C.byref(frame)))

    def set_tuning(self, warps: int = 4, reg_level: int = 0, ctas_per_sm: int = 0, packet: int = 1):
        """Warps per block (4, 8), register budget (resident warps per SM the
        allocation must allow: 0 unconstrained, 1 24, 2 32, 3 20, 4 16),
        resident blocks per SM (0 = occupancy maximum) and pixels per lane
        (1: 8x4-pixel items, 2: 8x8) of the persistent primary-ray kernel."""
        self._ck(self._L.vm_set_tuning(self._h, warps, reg_level, ctas_per_sm))
        self._ck(self._L.vm_set_packet(self._h, packet))

    def set_spec(self, spec: int = None):
        """The pipeline specialisations (VM_SPEC_* bits, the engine's make_spec
        override constants); None restores the engine's defaults."""
        self._ck(self._L.vm_set_spec(self._h, SPEC_DEFAULT if spec is None else spec))

    def set_stream(self, stream: int = 0):
        """The CUDA stream (a cudaStream_t as an int, e.g. a torch stream's
        cuda_stream) the context's work is issued on; 0: its own stream."""
        self._ck(self._L.vm_set_stream(self._h, C.c_void_p(stream or None)))

    # -- the engine's passes ------------------------------------------------------
    def select(self):
        self._ck(self._L.vm_select(self._h))

    def march(self):
        self._ck(self._L.vm_march(self._h))

    def primary_shadow(self):
        self._ck(self._L.vm_primary_shadow(self._h))

    def secondary(self):
        self._ck(self._L.vm_secondary(self._h))

    def soften_shadows(self, radius_limit: int = 4, penumbra: float = 1.5):
        """shadow_horizontal + shadow_vertical (shadow.wgsl:62-116) over the
        frame's blocker distances: the bilateral soft-shadow reconstruction
        (read it with read_shadow_mask)."""
        self._ck(self._L.vm_soften_shadows(self._h, radius_limit, penumbra))

    def render_passes(self):
        """tile_select .. march (+Hi-Z / recover) .. primary_shadow .. secondary"""
        self.select()
        self.march()
        self.primary_shadow()
        self.secondary()

    def render(self):
        """The wavefront pipeline (cull, primary, shadow, secondary kernels):
        same outputs as render_passes()."""
        self._ck(self._L.vm_render(self._h))

    def render_counted(self) -> dict:
        t = VmTraffic()
        self._ck(self._L.vm_render_counted(self._h, C.byref(t)))
        return self._traffic(t)

    def batch_counted(self, secondary: bool = False) -> dict:
        t = VmTraffic()
        self._ck(self._L.vm_batch_counted(self._h, 1 if secondary else 0, C.byref(t)))
        return self._traffic(t)

    @staticmethod
    def _traffic(t) -> dict:
        out = {n: int(getattr(t, n)) for n, _ in VmTraffic._fields_[:11]}
        out["stage_iters"] = [int(x) for x in t.stage_iters]
        out["stage_chunks"] = [int(x) for x in t.stage_chunks]
        out["stage_bytes"] = [int(x) for x in t.stage_bytes]
        return out

    def render_events(self, events):
        """render() recording five CUDA events (start, after the cull, after
        the primary, shadow and secondary kernels); events are raw
        cudaEvent_t handles (e.g. torch.cuda.Event().cuda_event after a
        first record)."""
        arr = (C.c_void_p * 5)(*events)
        self._ck(self._L.vm_render_events(self._h, arr))

    def sync(self):
        self._ck(self._L.vm_sync(self._h))

    # -- outputs --------------------------------------------------------------
    def _npix(self):
        f = self.view.frame
        return int(f.res[0]) * int(f.res[1])

    def read_vis(self, out: np.ndarray | None = None) -> np.ndarray:
        out = np.empty(self._npix(), np.uint64) if out is None else out
        self._ck(self._L.vm_read_vis(self._h, ptr(out)))
        return out

    def read_shadow(self, out: np.ndarray | None = None) -> np.ndarray:
        out = np.empty(self._npix(), np.float32) if out is None else out
        self._ck(self._L.vm_read_shadow(self._h, ptr(out)))
        return out

    def wait_render(self, other: "Marcher"):
        """vm_wait_render: later work of this context waits for other's last
        render (its kernels, not its read-back)."""
        self._ck(self._L.vm_wait_render(self._h, other._h))

    def read_shadow_r16f(self) -> np.ndarray:
        """The blocker distances as the engine's R16F shadow target
        (vm_read_async_r16f): binary16 bit patterns, rounded to nearest even."""
        out = np.empty(self._npix(), np.uint16)
        self._ck(self._L.vm_read_async_r16f(self._h, None, ptr(out)))
        self.sync()
        return out

    def read_reflection(self):
        """Reflect legs of the water hits of the last FLAG_WATER_REFLECT frame: (key, t)."""
        k = np.empty(self._npix(), np.uint64)
        t = np.empty(self._npix(), np.float32)
        self._ck(self._L.vm_read_reflection(self._h, ptr(k), ptr(t)))
        return k, t

    def water_sec(self, shift: int = 1):
        """The engine's water-leg schedule (water_sec, resolve.wgsl:1468-1535)
        over the last frame's visibility, one leg pair per 2^shift square."""
        self._ck(self._L.vm_water_sec(self._h, shift))
        self._ws_shift = shift

    def read_water_sec(self):
        """(refract key, refract t, reflect key, reflect t) per water_sec cell,
        shaped (ceil(h / 2^shift), ceil(w / 2^shift))."""
        w, h = int(self.view.frame.res[0]), int(self.view.frame.res[1])
        sp = 1 << self._ws_shift
        shape = ((h + sp - 1) // sp, (w + sp - 1) // sp)
        out = [np.empty(shape, np.uint64), np.empty(shape, np.float32), np.empty(shape, np.uint64),
               np.empty(shape, np.float32)]
        self._ck(self._L.vm_read_water_sec(self._h, *(ptr(a) for a in out)))
        return tuple(out)

    def upload_look(self, atlas: np.ndarray, faces: np.ndarray, probes: np.ndarray | None = None,
                    shaft: np.ndarray | None = None):
        """The resolve's material inputs (vm_upload_atlas, vm_upload_block_faces,
        vm_upload_probes, vm_upload_shaft); None for the probe field or the
        shaft envelope keeps the engine's neutral default."""
        a = np.ascontiguousarray(atlas, np.uint8)
        self._ck(self._L.vm_upload_atlas(self._h, ptr(a), a.size // (4 * 340), 16, 4))
        fc = np.ascontiguousarray(faces, np.uint32)
        self._ck(self._L.vm_upload_block_faces(self._h, ptr(fc), fc.size))
        if probes is None:
            self._ck(self._L.vm_upload_probes(self._h, None, 0, 0, 0))
        else:
            pr = np.ascontiguousarray(probes, np.uint16)
            self._ck(self._L.vm_upload_probes(self._h, ptr(pr), 128, 768, 128))
        if shaft is None:
            self._ck(self._L.vm_upload_shaft(self._h, None, 0))
        else:
            sh = np.ascontiguousarray(shaft, np.float32)
            self._ck(self._L.vm_upload_shaft(self._h, ptr(sh), 512))
        self._look = (a, fc, probes, shaft)

    def resolve(self, spec_hi: int):
        """The engine's resolve (sky, opaque surfaces, water, glass) over the
        last frame: vm_resolve with the engine's FLAG_HI_* word."""
        self._ck(self._L.vm_resolve(self._h, spec_hi))

    def read_color(self) -> np.ndarray:
        """RGBA float per pixel of the last vm_resolve (alpha 1)."""
        out = np.empty((self._npix(), 4), np.float32)
        self._ck(self._L.vm_read_color(self._h, ptr(out)))
        return out

    def read_shadow_mask(self, out: np.ndarray | None = None) -> np.ndarray:
        """clamp(1 - occlusion, 0, 1) per pixel after soften_shadows; 1 = lit."""
        out = np.empty(self._npix(), np.float32) if out is None else out
        self._ck(self._L.vm_read_shadow_mask(self._h, ptr(out)))
        return out

    def read_secondary(self):
        k = np.empty(self._npix(), np.uint64)
        t = np.empty(self._npix(), np.float32)
        self._ck(self._L.vm_read_secondary(self._h, ptr(k), ptr(t)))
        return k, t

    def read_hiz(self) -> np.ndarray:
        f = self.view.frame
        out = np.empty(int(f.tiles[0]) * int(f.tiles[1]), np.uint32)
        self._ck(self._L.vm_read_hiz(self._h, ptr(out)))
        return out

    def write_hiz(self, hiz: np.ndarray):
        h = np.ascontiguousarray(hiz, np.uint32)
        self._ck(self._L.vm_write_hiz(self._h, ptr(h)))

    def read_heatmap(self) -> np.ndarray:
        out = np.empty(self._npix(), np.uint32)
        self._ck(self._L.vm_read_heatmap(self._h, ptr(out)))
        return out

    def read_expanded(self, origin, dims):
        n = self._npix()
        vox = np.empty(n, np.uint32)
        face = np.empty(n, np.uint8)
        t = np.empty(n, np.float32)
        o = np.asarray(origin, np.int32)
        d = np.asarray(dims, np.uint32)
        self._ck(self._L.vm_read_expanded(self._h, ptr(o), ptr(d), ptr(vox), ptr(face), ptr(t)))
        return vox, face, t

    def stats(self) -> VmStats:
        s = VmStats()
        self._ck(self._L.vm_stats_read(self._h, C.byref(s)))
        return s

    def pair_demand(self) -> PairDemand:
        s = self.stats()
        return PairDemand(s.pairs_selected, s.pairs_deferred, s.pairs_recovered, s.max_pairs)

    def device_buffers(self) -> VmDevicePtrs:
        p = VmDevicePtrs()
        self._ck(self._L.vm_device_buffers(self._h, C.byref(p)))
        return p

    # -- batches -------------------------------------------------------------
    def batch_set(self, views: list[View]):
        frames = (VmFrame * len(views))(*[v.frame for v in views])
        chunks = np.ascontiguousarray(np.concatenate([v.chunks for v in views]))
        counts = np.array([len(v.chunks) for v in views], np.uint32)
        grids = np.ascontiguousarray(np.concatenate([v.grid for v in views]).astype(np.uint32))
        glens = np.array([v.grid.size for v in views], np.uint32)
        self._ck(self._L.vm_batch_set(self._h, len(views), C.cast(frames, C.c_void_p), ptr(chunks), ptr(counts),
                                      ptr(grids), ptr(glens)))
        self.batch_views = views

    def batch_run(self, per_view: bool = False, secondary: bool = False):
        """All views in one graph-replayed pipeline, or (per_view) one launch
        sequence per view; secondary also traces the water / glass rays."""
        self._ck(self._L.vm_batch_run(self._h, (1 if per_view else 0) | (2 if secondary else 0)))

    def batch_pixels(self) -> int:
        return int(self._L.vm_batch_pixels(self._h))

    def batch_read(self):
        n = self.batch_pixels()
        vis = np.empty(n, np.uint64)
        sh = np.empty(n, np.float32)
        self._ck(self._L.vm_batch_read(self._h, ptr(vis), ptr(sh)))
        return vis, sh

    def batch_read_secondary(self):
        n = self.batch_pixels()
        k = np.empty(n, np.uint64)
        t = np.empty(n, np.float32)
        self._ck(self._L.vm_batch_read_secondary(self._h, ptr(k), ptr(t)))
        return k, t


class Renderer:
    """The engine's Renderer, reduced to this path (src/render/mod.rs:747)."""

    def __init__(self, width: int, height: int, device: int = 0):
        self.size = (width, height)
        self.marcher = Marcher(width, height, device)
        self.world = None
        self._view = None

    def sync_world(self, world: World):
        """src/render/mod.rs:1355-1396"""
        self.world = world
        self.marcher.upload_world(*world.pools())

    def build_chunk_list(self, cam) -> View:
        """src/render/mod.rs:1447-1564"""
        cam.width, cam.height = self.size
        self._view = self.world.view(cam)
        self.marcher.upload_view(self._view)
        return self._view

    def render(self, fused: bool = True):
        """src/render/mod.rs:1593-1919 (march, Hi-Z, shadow and secondary passes)"""
        if fused:
            self.marcher.render()
        else:
            self.marcher.render_passes()

    def pair_demand(self) -> PairDemand:
        return self.marcher.pair_demand()

    def march_stats(self) -> dict:
        """src/render/mod.rs:1977-2045 over the FLAG_HEATMAP iteration buffer."""
        it = self.marcher.read_heatmap().astype(np.int64)
        touched = it[it > 0]
        s = np.sort(touched)
        pct = (lambda q: int(s[min(len(s) - 1, int(q * len(s)))]) if len(s) else 0)
        return {"pixels": int(it.size), "iters": int(it.sum()), "worst": int(it.max(initial=0)),
                "touched": int(touched.size), "p50": pct(0.5), "p90": pct(0.9), "p99": pct(0.99)}
