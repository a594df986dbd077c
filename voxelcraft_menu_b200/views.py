"""View sets of the batched workloads: cube-face probe captures and player
views over one world, marched together by vm_batch_run.

The engine captures such views one render at a time (its probe and lookbook
captures, src/headless.rs); here they are packed into one batch of ragged
resolutions.
"""
from __future__ import annotations

import math

import numpy as np

from .world import AIR, Camera, World

PROBE_RES = (32, 64, 128, 256)

# cube faces: forward axis and an up vector orthogonal to it
_FACES = (((1, 0, 0), (0, 1, 0)), ((-1, 0, 0), (0, 1, 0)), ((0, 1, 0), (0, 0, 1)),
          ((0, -1, 0), (0, 0, -1)), ((0, 0, 1), (0, 1, 0)), ((0, 0, -1), (0, 1, 0)))


def face_basis(face: int):
    f = np.array(_FACES[face][0], np.float32)
    up = np.array(_FACES[face][1], np.float32)
    r = np.cross(f, up).astype(np.float32)
    u = np.cross(r, f).astype(np.float32)
    return tuple(f.tolist()), tuple(r.tolist()), tuple(u.tolist())


def probe_centres(world: World, n: int, rng: np.random.Generator):
    """n points uniform in the world's air volume (rejection sampling)."""
    sx, sy, sz = world.recipe.size
    out = []
    while len(out) < n:
        p = rng.uniform((0.0, 0.0, 0.0), (sx, sy, sz))
        if world.get_block(int(p[0]), int(p[1]), int(p[2])) == AIR:
            out.append(tuple(float(v) for v in p))
    return out


def probe_views(world: World, n_probes: int = 512, seed: int = 3, res=PROBE_RES, **cam):
    """n_probes cube captures: 6 faces of fov 90 deg, aspect 1, each face's
    resolution drawn uniformly from res (seed 3)."""
    rng = np.random.default_rng(seed)
    views = []
    for c in probe_centres(world, n_probes, rng):
        for face in range(6):
            r = int(rng.choice(res))
            views.append(world.view(Camera(pos=c, basis=face_basis(face), fov_y=math.radians(90.0), width=r,
                                           height=r, **cam)))
    return views


def player_views(world: World, pos=(128.0, 110.0, 20.0), n: int = 4, seed: int = 3, width: int = 1920,
                 height: int = 1080, pitch_deg: float = -10.0, **cam):
    """n views at width x height from pos with random yaw (seed 3) and fixed pitch."""
    rng = np.random.default_rng(seed + 1000)
    return [world.view(Camera(pos=pos, yaw=float(rng.uniform(0.0, 2.0 * math.pi)), pitch=math.radians(pitch_deg),
                              width=width, height=height, **cam)) for _ in range(n)]


def ragged_views(world: World, n: int = 64, seed: int = 21, sizes=tuple(range(256, 1025, 64)), height_above=40.0,
                 pitch_deg: float = -10.0, **cam):
    """n square views of sides drawn uniformly from sizes (seed), at uniform
    positions over the world (height_above its surface, or the sea level),
    random yaw, fixed pitch."""
    from .world import surface_height
    rng = np.random.default_rng(seed)
    sx, _, sz = world.recipe.size
    views = []
    for _ in range(n):
        x, z = rng.uniform(0.07 * sx, 0.93 * sx), rng.uniform(0.07 * sz, 0.93 * sz)
        h = max(surface_height(world.recipe, int(x), int(z)), world.recipe.water_level)
        side = int(rng.choice(sizes))
        views.append(world.view(Camera(pos=(float(x), float(h) + height_above, float(z)),
                                       yaw=float(rng.uniform(0.0, 2.0 * math.pi)), pitch=math.radians(pitch_deg),
                                       width=side, height=side, **cam)))
    return views
