"""The product's world store against the oracle's producer (CPU).

The oracle producer (oracle/producer.cpp) restates the engine's encoder, run
pools and chunk list; the product store (csrc/store.cpp) is its own design
(staged encoder, pools packed from encoded chunks).  They must agree on:
  * the encoder's flat output, byte for byte, for recipe chunks of every
    level of detail and for hand-made palettes of every width;
  * every chunk record of a view (the pool offsets in root[2] and attr_base
    excepted), the frame and the grid, including LOD cross-fades;
  * the march: the oracle marched over the product's pools and view gives
    the same keys, shadow distances and water / glass rays as over its own.
"""
import math

import numpy as np
import pytest

from oracle import producer as OP
from oracle.oracle import Oracle
from voxelcraft_menu_b200 import encode as E
from voxelcraft_menu_b200 import world as W
from voxelcraft_menu_b200.world import Camera, World


def _flat(trees, i):
    info, l1, leaves, attrs, pal = (np.ascontiguousarray(a) for a in trees.chunk(i))
    return info, l1, leaves, attrs, pal


def _same_tree(got, want, what):
    for a, b, name in zip(got, want, ("info", "l1", "leaves", "attrs", "palette")):
        a = a.view(np.uint8) if a.dtype.names else a
        b = b.view(np.uint8) if b.dtype.names else b
        assert np.array_equal(a, b), f"{what}: {name} differs"


def _palette_chunk(seed, n_ids):
    rng = np.random.default_rng(seed)
    d = rng.integers(1, n_ids + 1, 64 ** 3).astype(np.uint16)
    d[rng.random(64 ** 3) < 0.3] = W.AIR
    return d


@pytest.mark.parametrize("case", ["recipe", "lod1", "lod2", "palettes", "empty", "full", "water"])
def test_host_encoder_equals_the_oracle_encoder(case):
    rec = W.recipe_small_terrain()
    if case == "recipe":
        dense = W.recipe_dense_chunks(rec)[::3]
    elif case == "lod1":
        dense = np.stack([W.recipe_dense_lod(W.recipe_mixed_lod(), 1, k) for k in [(0, 0, 0), (3, 0, 1), (2, 1, 2)]])
    elif case == "lod2":
        dense = np.stack([W.recipe_dense_lod(W.recipe_mixed_lod(), 2, k) for k in [(0, 0, 0), (1, 0, 1)]])
    elif case == "palettes":
        dense = np.stack([_palette_chunk(s, n) for s, n in enumerate((2, 3, 4, 5, 16, 17, 40, 64))])
    elif case == "empty":
        dense = np.zeros((1, 64 ** 3), np.uint16)
    elif case == "full":
        dense = np.full((1, 64 ** 3), W.STONE, np.uint16)
    else:
        d = np.full(64 ** 3, W.WATER, np.uint16)
        d[: 64 * 64 * 20] = W.STONE        # y < 20 (index x | z<<6 | y<<12)
        dense = d[None]
    got = E.cpu_build(dense)
    for i in range(len(dense)):
        want = OP.build_tree(dense[i])
        _same_tree(_flat(got, i), want, f"{case} chunk {i}")


def _record_fields(ch):
    """A chunk list without the pool offsets (root run pointer, attribute base)."""
    c = ch.copy()
    full = (c["root"][:, 2] & 0x80000000) != 0
    c["root"][~full, 2] = 0
    uniform = (c["attr_flags"] & 1) != 0
    c["attr_base"][~uniform] = 0
    return c


def _same_view(a, b):
    assert bytes(a.frame) == bytes(b.frame), "frame differs"
    assert len(a.chunks) == len(b.chunks)
    assert np.array_equal(_record_fields(a.chunks).view(np.uint8), _record_fields(b.chunks).view(np.uint8)), \
        "chunk records differ"
    assert np.array_equal(a.grid, b.grid), "grid differs"


@pytest.fixture(scope="module")
def small_pair():
    rec = W.recipe_small_terrain()
    return World.generate(rec), OP.OracleWorld.generate(rec)


@pytest.fixture(scope="module")
def lod_pair():
    rec, lay = W.recipe_mixed_lod(), W.mixed_lod_layout()
    pw = World()
    W.build_layout(pw, rec, lay)
    return pw, OP.build_layout(rec, lay)


def test_generated_worlds_have_the_same_blocks(small_pair):
    pw, ow = small_pair
    rng = np.random.default_rng(5)
    for x, y, z in rng.integers((0, 0, 0), (256, 128, 256), (4000, 3)):
        assert pw.get_block(int(x), int(y), int(z)) == ow.get_block(int(x), int(y), int(z))
    for key in [(0, 0, 0), (1, 1, 2), (3, 0, 3)]:
        a, b = pw.chunk_info(key), ow.chunk_info(key)
        for f in ("aabb_min", "aabb_max", "solid_count", "leaf_count", "dry_mask", "has_water", "has_cutout",
                  "attr_uniform"):
            assert np.array_equal(np.asarray(getattr(a, f)), np.asarray(getattr(b, f))), f
    sp, so = pw.pool_stats(), ow.pool_stats()
    assert sp.n_chunks == so.n_chunks
    assert sp.n_inners <= so.n_inners + 64 and sp.n_leaves <= so.n_leaves, "run sharing as tight as the engine's"


@pytest.mark.parametrize("cam", [dict(), dict(yaw=math.radians(200.0), pitch=math.radians(-40.0)),
                                 dict(pos=(40.0, 70.0, 200.0), yaw=0.3, grid_dim=(4, 2, 4)),
                                 dict(offscreen_shadows=False, max_chunks=12)])
def test_views_agree(small_pair, cam):
    pw, ow = small_pair
    kw = dict(pos=(128.0, 110.0, 20.0), width=320, height=180)
    kw.update(cam)
    _same_view(pw.view(Camera(**kw)), ow.view(Camera(**kw)))


def test_mixed_lod_views_agree(lod_pair):
    pw, ow = lod_pair
    for cam in (Camera(pos=(128.0, 110.0, 20.0), width=320, height=180),
                Camera(pos=(300.0, 90.0, 150.0), yaw=math.radians(135.0), width=200, height=200)):
        a, b = pw.view(cam), ow.view(cam)
        _same_view(a, b)
        lods = set(int(x) for x in a.chunks["lod"])
        assert lods == {0, 1, 2}, lods
        fades = set(round(float(x), 3) for x in a.chunks["fade"])
        assert {0.6, -0.6, 1.0} <= fades


def _march_all(view, pools):
    o = Oracle(view, *pools)
    vis, hiz, _ = o.frame_vis()
    sh = o.shadow(vis)
    sk, st = o.secondary(vis)
    return vis, sh, sk, st


@pytest.mark.parametrize("which", ["small", "lod"])
def test_oracle_march_over_either_producer_agrees(small_pair, lod_pair, which):
    pw, ow = small_pair if which == "small" else lod_pair
    cam = Camera(pos=(128.0, 110.0, 20.0), width=240, height=135)
    got = _march_all(pw.view(cam), pw.pools())
    want = _march_all(ow.view(cam), ow.pools())
    for g, w_, name in zip(got, want, ("vis", "shadow", "secondary key", "secondary t")):
        assert np.array_equal(g, w_), name
    assert (got[0] != 0).mean() > 0.3


def test_store_edits_repack(small_pair):
    """Replacing and removing chunks: the packed pools always describe the
    current chunks (blocks and views equal the oracle producer's after the
    same edits)."""
    rec = W.recipe_small_terrain()
    pw, ow = World.generate(rec), OP.OracleWorld.generate(rec)
    d = np.zeros(64 ** 3, np.uint16)
    d[: 64 * 64 * 10] = W.GLOWSTONE
    for w in (pw, ow):
        w.insert_dense((1, 0, 1), d)
        w.remove((2, 1, 2))
        w.insert_dense((9, 0, 9), d)
    cam = Camera(pos=(128.0, 110.0, 20.0), width=160, height=90)
    _same_view(pw.view(cam), ow.view(cam))
    assert pw.get_block(64 + 5, 3, 64 + 7) == W.GLOWSTONE == ow.get_block(64 + 5, 3, 64 + 7)
    assert pw.get_block(64 + 5, 30, 64 + 7) == W.AIR


def test_set_fade_rejects_bad_values():
    w = World()
    w.insert_dense((0, 0, 0), np.full(64 ** 3, W.STONE, np.uint16))
    with pytest.raises(KeyError):
        w.set_fade((5, 5, 5), 0.5)
    with pytest.raises(ValueError):
        w.set_fade((0, 0, 0), 1.5)
    w.set_fade((0, 0, 0), -0.25)
