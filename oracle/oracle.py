"""ctypes binding of the oracle (oracle/liboracle.so) -- test infrastructure.

Only tests/, __graft_entry__.smoke() and bench.py's CPU baseline leg import
this module, and only as the checker / the timed CPU restatement; the product
never calls it.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"

vp = C.c_void_p


class OrWorld(C.Structure):
    _fields_ = [("frame", vp), ("chunks", vp), ("n_chunks", C.c_uint32), ("inners", vp), ("n_inners", C.c_uint64),
                ("leaves", vp), ("n_leaves", C.c_uint64), ("bricks", vp), ("n_bricks", C.c_uint64), ("grid", vp),
                ("n_grid", C.c_uint64), ("spec", C.c_uint32), ("atlas", vp), ("atlas_layers", C.c_uint32),
                ("faces", vp), ("n_faces", C.c_uint32)]


# pipeline specialisations (VM_SPEC_* of vm_types.h; the engine's make_spec, src/render/mod.rs:2355-2689)
SPEC_FULL_MARCH, SPEC_WATER_REPAIR, SPEC_LEAF_CUTOUT, SPEC_GLASS = 1, 2, 4, 8
SPEC_EMITTER_GATHER, SPEC_FOLIAGE, SPEC_SNELL_BEND, SPEC_LEAF_THIN = 16, 32, 64, 128
SPEC_DEFAULT = SPEC_FULL_MARCH | SPEC_WATER_REPAIR | SPEC_LEAF_CUTOUT | SPEC_GLASS | SPEC_EMITTER_GATHER | \
    SPEC_FOLIAGE | SPEC_LEAF_THIN
SPEC_SOFT_RAYS = 256      # extension: jittered sun rays per hit, the shadow buffer holds the blocked fraction


class OrLook(C.Structure):
    """The resolve's material inputs as the engine uploads them."""
    _fields_ = [("atlas_srgb", vp), ("layers", C.c_uint32), ("faces", vp), ("n_faces", C.c_uint32), ("probes", vp),
                ("shaft", vp), ("spec_hi", C.c_uint32)]


class OrHit(C.Structure):
    _fields_ = [("hit", C.c_uint32), ("t", C.c_float), ("normal", C.c_uint32), ("voxel", C.c_uint32 * 3),
                ("micro", C.c_uint32 * 3), ("iters", C.c_uint32)]


class OrCounters(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in ("chunk_records", "l1_fetches", "leaf_fetches", "attr_fetches",
                                          "palette_decodes", "grid_lookups", "iters", "march_calls", "rays")]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not LIB.exists():
            from . import build as _b
            _b.build()
        L = C.CDLL(str(LIB))
        sig = {
            "or_last_error": (C.c_int, [C.c_char_p, C.c_int]),
            "or_clear_error": (None, []),
            "or_ray_dir": (None, [vp, C.c_float, C.c_float, vp]),
            "or_soft_sun_dir": (None, [vp, C.c_uint32, C.c_uint32, C.c_uint32, vp]),
            "or_march_chunk": (C.c_int, [vp, C.c_uint32, vp, vp, C.c_float, C.c_uint32, C.c_uint32, C.c_uint32,
                                         C.c_uint32, C.POINTER(OrHit)]),
            "or_shadow_ray_t": (C.c_float, [vp, vp, vp, C.c_float]),
            "or_trace_world": (C.c_int, [vp, vp, vp, C.c_float, C.c_uint32, vp, vp, vp, vp, vp]),
            "or_block_at": (C.c_uint32, [vp, C.c_uint32, vp]),
            "or_world_block_at": (C.c_uint32, [vp, vp]),
            "or_make_key": (C.c_uint64, [vp, C.c_float, C.c_uint32, C.c_uint32, vp, vp]),
            "or_depth_key": (C.c_uint32, [vp, C.c_float]),
            "or_leaf_solid": (C.c_uint32, [vp, vp]),
            "or_frame": (C.c_int, [vp, vp, vp, vp, vp, vp, C.c_uint32, C.c_uint32, C.c_int, vp]),
            "or_tile_pairs": (C.c_uint32, [vp, C.c_uint32, vp, vp, C.c_uint32, vp, C.c_uint32, vp]),
            "or_primary_shadow": (C.c_int, [vp, vp, vp, C.c_uint64, C.c_uint64, C.c_int, vp]),
            "or_secondary": (C.c_int, [vp, vp, vp, vp, C.c_uint64, C.c_uint64, C.c_int]),
            "or_expand": (C.c_int, [vp, vp, vp, vp, vp, vp, vp, C.c_int]),
            "or_grid_block": (C.c_uint32, [vp, C.c_int32, C.c_int32, C.c_int32]),
            "or_pick": (C.c_int, [vp, vp, vp, C.c_uint32, C.c_float, vp, vp, vp]),
            "or_soften_shadows": (C.c_int, [vp, vp, vp, C.c_uint32, C.c_float, vp, vp, C.c_int]),
            "or_reflect": (C.c_int, [vp, vp, vp, vp, C.c_uint64, C.c_uint64, C.c_int]),
            "or_water_sec": (C.c_int, [vp, vp, C.c_uint32, vp, vp, vp, vp, C.c_int]),
            "or_resolve": (C.c_int, [vp, vp, vp, vp, vp, C.c_uint64, C.c_uint64, C.c_int]),
            "or_resolve_heat": (C.c_int, [vp, vp, vp, C.c_uint64, C.c_uint64]),
            "or_build_atlas": (None, [C.c_float, C.c_int, vp]),
            "or_pick_rows": (C.c_uint64, [vp, C.c_uint32, C.c_uint32, C.c_uint32, C.c_int, vp]),
            "or_f16_round": (None, [vp, vp, C.c_uint64]),
        }
        for n, (r, a) in sig.items():
            f = getattr(L, n)
            f.restype, f.argtypes = r, a
        _lib = L
    return _lib


def _p(a):
    return C.c_void_p(a.ctypes.data)


def engine_atlas(water_mottle: float = 0.0, tint_balance: bool = False) -> np.ndarray:
    """The engine's block atlas (src/textures.rs build_atlas + downsample, as
    make_atlas uploads it): uint8 sRGB RGBA, 27 layers, mips 16, 8, 4, 2."""
    out = np.zeros(27 * 340 * 4, np.uint8)
    lib().or_build_atlas(water_mottle, 1 if tint_balance else 0, _p(out))
    return out


class Oracle:
    """The oracle bound to one view (frame + chunk list + grid) and the pools."""

    def __init__(self, view, inners, leaves, bricks, threads: int = 0, spec: int = SPEC_DEFAULT, atlas=None,
                 faces=None):
        """atlas / faces: the engine's atlas bytes and face table, for the
        tuft cross-quads (without them tufts are transparent)."""
        self.L = lib()
        self.view = view
        self.frame = view.frame
        self._keep = [np.ascontiguousarray(view.chunks), np.ascontiguousarray(inners, np.uint32),
                      np.ascontiguousarray(leaves, np.uint32), np.ascontiguousarray(bricks, np.uint32),
                      np.ascontiguousarray(view.grid, np.uint32)]
        ch, i, l, b, g = self._keep
        self.w = OrWorld(C.cast(C.pointer(self.frame), vp), _p(ch), len(ch), _p(i), i.size // 4, _p(l), l.size // 2,
                         _p(b), b.size, _p(g), g.size, spec)
        if atlas is not None and faces is not None:
            a, fc = np.ascontiguousarray(atlas, np.uint8), np.ascontiguousarray(faces, np.uint32)
            self._keep += [a, fc]
            self.w.atlas, self.w.atlas_layers = _p(a), a.size // (4 * 340)
            self.w.faces, self.w.n_faces = _p(fc), fc.size
        self.spec = spec
        self.threads = threads
        self.L.or_clear_error()

    @property
    def npix(self):
        return int(self.frame.res[0]) * int(self.frame.res[1])

    @property
    def ntiles(self):
        return int(self.frame.tiles[0]) * int(self.frame.tiles[1])

    def _check(self, rc):
        if rc:
            buf = C.create_string_buffer(256)
            self.L.or_last_error(buf, 256)
            raise RuntimeError(f"oracle read out of bounds: {buf.value.decode()}")

    def frame_vis(self, hiz_in=None, tiles=None, heat=False, traffic=False):
        """Visibility keys by the engine's pass sequence; returns (vis, hiz, counters[, dbg][, traffic])."""
        vis = np.zeros(self.npix, np.uint64)
        hiz = np.zeros(self.ntiles, np.uint32)
        ctr = np.zeros(8, np.uint32)
        dbg = np.zeros(self.npix, np.uint32) if heat else None
        hz_in = None if hiz_in is None else np.ascontiguousarray(hiz_in, np.uint32)
        t0, t1 = (0, self.ntiles) if tiles is None else tiles
        tc = OrCounters() if traffic else None
        rc = self.L.or_frame(C.byref(self.w), None if hz_in is None else _p(hz_in), _p(vis), _p(hiz), _p(ctr),
                             None if dbg is None else _p(dbg), t0, t1, self.threads,
                             C.byref(tc) if tc is not None else None)
        self._check(rc)
        out = [vis, hiz, ctr]
        if heat:
            out.append(dbg)
        if traffic:
            out.append({n: int(getattr(tc, n)) for n, _ in OrCounters._fields_})
        return tuple(out)

    def shadow(self, vis, pix=None, traffic=False):
        out = np.zeros(self.npix, np.float32)
        p0, p1 = (0, self.npix) if pix is None else pix
        tc = OrCounters() if traffic else None
        v = np.ascontiguousarray(vis, np.uint64)
        self._check(self.L.or_primary_shadow(C.byref(self.w), _p(v), _p(out), p0, p1, self.threads,
                                             C.byref(tc) if tc is not None else None))
        if traffic:
            return out, {n: int(getattr(tc, n)) for n, _ in OrCounters._fields_}
        return out

    def reflection(self, vis, pix=None):
        """The reflect leg of every water hit: (key, t) per pixel, key 0 where none."""
        k = np.zeros(self.npix, np.uint64)
        t = np.zeros(self.npix, np.float32)
        p0, p1 = (0, self.npix) if pix is None else pix
        v = np.ascontiguousarray(vis, np.uint64)
        self._check(self.L.or_reflect(C.byref(self.w), _p(v), _p(k), _p(t), p0, p1, self.threads))
        return k, t

    def water_sec(self, vis, shift: int = 1):
        """water_sec (resolve.wgsl:1468-1535): (refract key, refract t,
        reflect key, reflect t) per (2^shift)^2 block, shaped (rows, cols)."""
        w, h = int(self.frame.res[0]), int(self.frame.res[1])
        sp = 1 << shift
        shape = ((h + sp - 1) // sp, (w + sp - 1) // sp)
        out = [np.zeros(shape, np.uint64), np.zeros(shape, np.float32), np.zeros(shape, np.uint64),
               np.zeros(shape, np.float32)]
        v = np.ascontiguousarray(vis, np.uint64)
        self._check(self.L.or_water_sec(C.byref(self.w), _p(v), shift, *(_p(a) for a in out), self.threads))
        return tuple(out)

    def resolve_heat(self, dbg, pix=None):
        """The heat-map view of a FLAG_HEATMAP frame (resolve.wgsl:36-44,
        1389-1394): RGBA per pixel from the summed march iterations dbg."""
        b, e = (0, self.npix) if pix is None else pix
        d = np.ascontiguousarray(dbg, np.uint32)
        out = np.zeros((e - b, 4), np.float32)
        self._check(self.L.or_resolve_heat(C.byref(self.w), _p(d), _p(out), b, e))
        return out

    def resolve(self, vis, sun_vis, atlas, faces, probes=None, shaft=None, spec_hi: int = 0, pix=None):
        """The resolve (resolve.wgsl:1378-1466), every lane: RGBA float per
        pixel of [pix[0], pix[1]) (default: all), alpha 1.  sun_vis: the
        per-pixel sun visibility (the engine's primary_sun)."""
        b, e = (0, self.npix) if pix is None else pix
        keep = [np.ascontiguousarray(atlas, np.uint8), np.ascontiguousarray(faces, np.uint32)]
        pr = None if probes is None else np.ascontiguousarray(probes, np.uint16)
        sh = None if shaft is None else np.ascontiguousarray(shaft, np.float32)
        look = OrLook(_p(keep[0]), keep[0].size // (4 * 340), _p(keep[1]), keep[1].size,
                      None if pr is None else _p(pr), None if sh is None else _p(sh), spec_hi)
        v = np.ascontiguousarray(vis, np.uint64)
        sv = np.ascontiguousarray(sun_vis, np.float32)
        out = np.zeros((e - b, 4), np.float32)
        self._check(self.L.or_resolve(C.byref(self.w), C.byref(look), _p(v), _p(sv), _p(out), b, e, self.threads))
        return out

    def soften(self, vis, dist, limit: int = 4, penumbra: float = 1.5):
        """shadow_horizontal + shadow_vertical over the frame's blocker
        distances: returns (h, mask), h the horizontal pass (npix, 2) as stored
        in rg16float, mask clamp(1 - occlusion, 0, 1) before r8unorm."""
        h = np.zeros((self.npix, 2), np.float32)
        mask = np.zeros(self.npix, np.float32)
        v = np.ascontiguousarray(vis, np.uint64)
        d = np.ascontiguousarray(dist, np.float32)
        self._check(self.L.or_soften_shadows(C.byref(self.w), _p(v), _p(d), limit, penumbra, _p(h), _p(mask),
                                             self.threads))
        return h, mask

    def secondary(self, vis, pix=None):
        k = np.zeros(self.npix, np.uint64)
        t = np.zeros(self.npix, np.float32)
        p0, p1 = (0, self.npix) if pix is None else pix
        v = np.ascontiguousarray(vis, np.uint64)
        self._check(self.L.or_secondary(C.byref(self.w), _p(v), _p(k), _p(t), p0, p1, self.threads))
        return k, t

    def expand(self, vis, origin, dims):
        n = self.npix
        vox = np.zeros(n, np.uint32)
        face = np.zeros(n, np.uint8)
        t = np.zeros(n, np.float32)
        o = np.asarray(origin, np.int32)
        d = np.asarray(dims, np.uint32)
        v = np.ascontiguousarray(vis, np.uint64)
        self._check(self.L.or_expand(C.byref(self.w), _p(v), _p(o), _p(d), _p(vox), _p(face), _p(t), self.threads))
        return vox, face, t

    def tile_pairs(self, tile_id, hiz_in=None):
        cap = 8192
        out = np.zeros(cap, np.uint32)
        dfr = np.zeros(cap, np.uint32)
        nd = C.c_uint32(0)
        hz = None if hiz_in is None else np.ascontiguousarray(hiz_in, np.uint32)
        n = self.L.or_tile_pairs(C.byref(self.w), tile_id, None if hz is None else _p(hz), _p(out), cap, _p(dfr), cap,
                                 C.byref(nd))
        return out[:n].copy(), dfr[: nd.value].copy()

    def march_chunk(self, ci, ro, rd, t_limit, skip_water=False, skip_foliage=False, skip_glass=False, sun_ray=False):
        h = OrHit()
        ro = np.asarray(ro, np.float32)
        rd = np.asarray(rd, np.float32)
        self._check(self.L.or_march_chunk(C.byref(self.w), ci, _p(ro), _p(rd), t_limit, skip_water, skip_foliage,
                                          skip_glass, sun_ray, C.byref(h)))
        return h

    def shadow_ray_t(self, ro, rd, max_dist):
        ro = np.asarray(ro, np.float32)
        rd = np.asarray(rd, np.float32)
        return float(self.L.or_shadow_ray_t(C.byref(self.w), _p(ro), _p(rd), max_dist))

    def trace_world(self, ro, rd, max_dist, skip_water):
        ro = np.asarray(ro, np.float32)
        rd = np.asarray(rd, np.float32)
        hit, normal, ci = C.c_uint32(), C.c_uint32(), C.c_uint32()
        t = C.c_float()
        vox = np.zeros(3, np.uint32)
        self._check(self.L.or_trace_world(C.byref(self.w), _p(ro), _p(rd), max_dist, skip_water, C.byref(hit),
                                          C.byref(t), C.byref(normal), _p(vox), C.byref(ci)))
        return bool(hit.value), t.value, normal.value, tuple(vox.tolist()), ci.value

    def ray_dir(self, px, py):
        out = np.zeros(3, np.float32)
        self.L.or_ray_dir(C.byref(self.frame), px, py, _p(out))
        return out

    def soft_sun_dir(self, px, py, s):
        out = np.zeros(3, np.float32)
        self.L.or_soft_sun_dir(C.byref(self.frame), px, py, s, _p(out))
        return out

    def depth_key(self, t):
        return int(self.L.or_depth_key(C.byref(self.frame), t))

    def make_key(self, t, normal, ci, v, micro):
        v = np.asarray(v, np.uint32)
        m = np.asarray(micro, np.uint32)
        return int(self.L.or_make_key(C.byref(self.frame), t, normal, ci, _p(v), _p(m)))

    def block_at(self, ci, v):
        v = np.asarray(v, np.uint32)
        return int(self.L.or_block_at(C.byref(self.w), ci, _p(v)))

    def world_block_at(self, p):
        p = np.asarray(p, np.float32)
        return int(self.L.or_world_block_at(C.byref(self.w), _p(p)))

    def grid_block(self, x, y, z):
        return int(self.L.or_grid_block(C.byref(self.w), x, y, z))

    def pick_rows(self, row0, rows, max_steps=4096):
        """Player::pick per pixel of pixel rows [row0, row0 + rows): (pixels, hits)."""
        hits = C.c_uint64()
        n = self.L.or_pick_rows(C.byref(self.w), row0, rows, max_steps, self.threads, C.byref(hits))
        return int(n), int(hits.value)

    def pick(self, origin, direction, max_steps=64, reach=1e9):
        o = np.asarray(origin, np.float32)
        d = np.asarray(direction, np.float32)
        blk = np.zeros(3, np.int32)
        nrm = np.zeros(3, np.int32)
        dist = C.c_float()
        hit = self.L.or_pick(C.byref(self.w), _p(o), _p(d), max_steps, reach, _p(blk), _p(nrm), C.byref(dist))
        if not hit:
            return None
        return tuple(blk.tolist()), tuple(nrm.tolist()), dist.value


def leaf_solid(wv, m):
    wv = np.asarray(wv, np.int32)
    m = np.asarray(m, np.uint32)
    return bool(lib().or_leaf_solid(_p(wv), _p(m)))


def f16_round(x):
    """The oracle's binary16 storage rounding of float32 values."""
    x = np.ascontiguousarray(x, np.float32)
    out = np.empty_like(x)
    lib().or_f16_round(_p(x), _p(out), x.size)
    return out

