"""The dense -> 64-tree chunk encoder (build_local, src/voxel/tree.rs:89-204).

The checker is the oracle's restatement of build_local (oracle/producer.cpp,
orw_build_tree).  CPU: the product's host encoder (vmw_build_tree) equals it
on hand-made chunks covering the encoder's cases (empty, one id everywhere,
full L1 nodes of mixed ids, water-only nodes and water lines, 64 distinct ids
in a leaf, emitters, foliage, glass, palette overflow), and its flat export
inserted chunk by chunk (vmw_insert_tree) gives the same pools as
World.generate.  GPU: vm_encode_trees equals the oracle field for field on
those chunks and on every chunk of the 256x128x256 and 1024x256x1024
terrains, and a world built from its output has World.generate's pools."""
import numpy as np
import pytest

from oracle import producer as OP
from voxelcraft_menu_b200 import encode as E
from voxelcraft_menu_b200 import world as W


def oracle_trees(dense, palette_cap):
    """orw_build_tree of every chunk, in the Trees layout."""
    out = E.empty(len(dense), palette_cap)
    for i, d in enumerate(dense):
        info, l1, leaves, attrs, pal = OP.build_tree(d, max(palette_cap, 1))
        out.info[i] = info[0]
        out.l1[i, :len(l1)] = l1
        out.leaves[i, :len(leaves)] = leaves
        out.attrs[i, :len(attrs)] = attrs
        out.palette[i, :len(pal)] = pal
    return out


def dense_index(x, y, z):
    return x | (z << 6) | (y << 12)


def special_chunks():
    rng = np.random.default_rng(4)
    n = 10
    d = np.zeros((n, 64, 64, 64), np.uint16)           # [chunk, y, z, x]: index x | z<<6 | y<<12
    # 0: empty
    d[1] = W.STONE                                       # 1: one id everywhere (uniform)
    d[2, :32] = W.STONE                                  # 2: full L1 nodes of two ids, grass top, water above
    d[2, 31] = W.GRASS
    d[2, 32:40] = W.WATER
    d[3] = rng.integers(0, 64, (64, 64, 64))             # 3: up to 64 distinct ids per leaf (8-bit indices)
    d[4, :, :, :] = W.WATER                              # 4: water, a sand corner (water lines, dry mask)
    d[4, :5, :, :20] = W.SAND
    d[5, 10:50, 10:50, 10:50] = rng.choice([W.GLOWSTONE, 20, W.LEAVES, W.GLASS, W.TALL_GRASS, W.DIRT],
                                           (40, 40, 40))  # 5: emitters (20: amber lamp), cutout, glass, foliage
    d[6] = np.where(rng.random((64, 64, 64)) < 0.5, W.STONE, W.AIR)   # 6: half-full leaves, 1-bit palettes
    d[7, 3, 7, 9] = W.LOG                                # 7: a single voxel
    d[8] = rng.integers(0, 3, (64, 64, 64))              # 8: 2-3 ids per leaf (1 and 2-bit indices)
    d[9, :, :, :] = rng.integers(1, 17, (64, 64, 64))    # 9: full chunk of 16 ids (4-bit indices, full L1s)
    return d.reshape(n, -1)


@pytest.fixture(scope="module")
def small_dense():
    return W.recipe_dense_chunks(W.recipe_small_terrain())


def test_cpu_flat_round_trip_equals_generate(small_dense):
    rec = W.recipe_small_terrain()
    trees = E.cpu_build(small_dense)
    w = W.World()
    nx, ny = rec.size[0] // 64, rec.size[1] // 64
    for i in range(len(trees)):
        E.insert(w, (i % nx, i // nx % ny, i // (nx * ny)), trees, i)
    ref = W.World.generate(rec)
    for a, b in zip(w.pools(), ref.pools()):
        assert np.array_equal(a, b)


def test_cpu_special_chunks():
    d = special_chunks()
    t = E.cpu_build(d, palette_cap=1 << 18)
    info = t.info
    assert info[0]["n_l1"] == 0 and info[0]["uniform"] == -1 and info[0]["solid_count"] == 0
    assert info[1]["uniform"] == W.STONE and info[1]["n_attrs"] == 0 and info[1]["solid_count"] == 64 ** 3
    assert (t.l1[1]["full"] == 1).all() and info[1]["n_leaves"] == 0
    assert info[3]["n_palette"] > 4096 * 30                       # ~40 ids per leaf: 8-bit indices
    assert info[4]["dry_mask"] != 0 and (info[4]["flags"] & 1)
    assert info[5]["emitters"] > 0 and (info[5]["flags"] & 0x1E) == 0x1E
    assert tuple(info[7]["aabb_min"]) == (9, 3, 7) and tuple(info[7]["aabb_max"]) == (10, 4, 8)
    # palette overflow: flagged, n_palette = the words needed
    small = E.cpu_build(d[3:4], palette_cap=100)
    assert small.info[0]["flags"] & E.PALETTE_OVERFLOW and small.info[0]["n_palette"] == info[3]["n_palette"]
    assert np.array_equal(small.palette[0, :100], t.palette[3, :100])
    # the comparison used by the GPU tests: equal to itself, not to a neighbour
    assert all(E.same_chunk(t, i, t, i) for i in range(len(t)))
    assert not E.same_chunk(t, 2, t, 6)
    # and the host encoder is the oracle's build_local
    for cap in (1 << 18, 100):
        assert_same_trees(E.cpu_build(d, cap), oracle_trees(d, cap))


def gpu_trees(dense, palette_cap):
    import torch
    d = torch.from_numpy(np.ascontiguousarray(dense).view(np.int16)).cuda()
    out = E.gpu_encode(d, len(dense), palette_cap, torch)
    torch.cuda.synchronize()
    return out.to_host()


def assert_same_trees(g, c):
    bad = [i for i in range(len(c)) if not E.same_chunk(g, i, c, i)]
    assert not bad, f"{len(bad)} of {len(c)} chunks differ, first {bad[:5]}"


@pytest.mark.gpu
def test_gpu_special_chunks():
    d = special_chunks()
    for cap in (1 << 18, 100):
        assert_same_trees(gpu_trees(d, cap), oracle_trees(d, cap))


@pytest.mark.gpu
def test_gpu_lod_chunks():
    rec = W.recipe_mixed_lod()
    d = np.stack([W.recipe_dense_lod(rec, lod, key) for lod, key, _ in W.mixed_lod_layout() if lod > 0])
    assert_same_trees(gpu_trees(d, 16384), oracle_trees(d, 16384))


@pytest.mark.gpu
def test_gpu_terrains_and_world(small_dense):
    rec = W.recipe_small_terrain()
    g = gpu_trees(small_dense, 16384)
    assert_same_trees(g, oracle_trees(small_dense, 16384))
    w = W.World()
    nx, ny = rec.size[0] // 64, rec.size[1] // 64
    for i in range(len(g)):
        E.insert(w, (i % nx, i // nx % ny, i // (nx * ny)), g, i)
    for a, b in zip(w.pools(), W.World.generate(rec).pools()):
        assert np.array_equal(a, b)
    large = W.recipe_dense_chunks(W.recipe_large_terrain())
    assert_same_trees(gpu_trees(large, 16384), oracle_trees(large, 16384))
