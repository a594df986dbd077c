"""The dense -> 64-tree chunk encoder (build_local, src/voxel/tree.rs:89-204).

`gpu_encode` runs vm_encode_trees over a batch of dense chunks already on the
device (one CTA per chunk); `cpu_build` is the CPU restatement
(vmw_build_tree) with the same flat output; `insert` puts one encoded chunk
into a World (World::insert_local, src/voxel/world.rs:63-175).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from .native import lib, ptr

CHUNK_VOXELS = 64 ** 3
TREE_L1, TREE_LEAVES = 64, 4096
PALETTE_OVERFLOW = 0x80000000

INFO_DTYPE = np.dtype([("root_mask", "<u8"), ("dry_mask", "<u8"), ("uniform", "<i4"), ("flags", "<u4"),
                       ("emitters", "<u4"), ("solid_count", "<u4"), ("leaf_count", "<u4"), ("n_l1", "<u4"),
                       ("n_leaves", "<u4"), ("n_attrs", "<u4"), ("n_palette", "<u4"), ("aabb_min", "u1", 3),
                       ("aabb_max", "u1", 3), ("pad", "u1", 6)])
L1_DTYPE = np.dtype([("mask", "<u8"), ("leaf_start", "<u4"), ("leaf_prefix", "<u4"), ("full", "u1"),
                     ("water_line", "u1"), ("pad", "u1", 6)])
assert INFO_DTYPE.itemsize == 64 and L1_DTYPE.itemsize == 24


@dataclass
class Trees:
    """n encoded chunks: info (n,), l1 (n, 64), leaves (n, 4096) u64,
    attrs (n, 4096) u32, palette (n, palette_cap) u32; only the first
    n_l1 / n_leaves / n_attrs / n_palette entries of a chunk are defined."""
    info: np.ndarray
    l1: np.ndarray
    leaves: np.ndarray
    attrs: np.ndarray
    palette: np.ndarray

    def __len__(self):
        return len(self.info)

    def chunk(self, i):
        n = self.info[i]
        return (self.info[i:i + 1], self.l1[i, :n["n_l1"]], self.leaves[i, :n["n_leaves"]], self.attrs[i, :n["n_attrs"]],
                self.palette[i, :min(int(n["n_palette"]), self.palette.shape[1])])


def empty(n: int, palette_cap: int) -> Trees:
    return Trees(np.zeros(n, INFO_DTYPE), np.zeros((n, TREE_L1), L1_DTYPE), np.zeros((n, TREE_LEAVES), np.uint64),
                 np.zeros((n, TREE_LEAVES), np.uint32), np.zeros((n, max(palette_cap, 1)), np.uint32))


def cpu_build(dense: np.ndarray, palette_cap: int = 16384) -> Trees:
    """vmw_build_tree of every chunk of dense (n x 64^3 u16)."""
    d = np.ascontiguousarray(dense, np.uint16).reshape(-1, CHUNK_VOXELS)
    out = empty(len(d), palette_cap)
    L = lib()
    for i in range(len(d)):
        rc = L.vmw_build_tree(ptr(d[i]), palette_cap, ptr(out.info[i:i + 1]), ptr(out.l1[i]), ptr(out.leaves[i]),
                              ptr(out.attrs[i]), ptr(out.palette[i]))
        if rc:
            raise RuntimeError("vmw_build_tree failed")
    return out


class DeviceTrees:
    """vm_encode_trees outputs as torch device tensors."""

    def __init__(self, n: int, palette_cap: int, torch, device="cuda"):
        u8 = torch.uint8
        self.n, self.palette_cap = n, palette_cap
        self.info = torch.empty(n * INFO_DTYPE.itemsize, dtype=u8, device=device)
        self.l1 = torch.empty(n * TREE_L1 * L1_DTYPE.itemsize, dtype=u8, device=device)
        self.leaves = torch.empty(n * TREE_LEAVES * 8, dtype=u8, device=device)
        self.attrs = torch.empty(n * TREE_LEAVES * 4, dtype=u8, device=device)
        self.palette = torch.empty(max(n * palette_cap, 1) * 4, dtype=u8, device=device)

    def to_host(self) -> Trees:
        n, cap = self.n, self.palette_cap
        return Trees(self.info.cpu().numpy().view(INFO_DTYPE).copy(),
                     self.l1.cpu().numpy().view(L1_DTYPE).reshape(n, TREE_L1).copy(),
                     self.leaves.cpu().numpy().view(np.uint64).reshape(n, TREE_LEAVES).copy(),
                     self.attrs.cpu().numpy().view(np.uint32).reshape(n, TREE_LEAVES).copy(),
                     self.palette.cpu().numpy().view(np.uint32)[:n * cap].reshape(n, max(cap, 1) if cap else 0)
                     if cap else np.zeros((n, 1), np.uint32))


def gpu_encode(d_dense, n: int, palette_cap: int, torch, out: DeviceTrees | None = None) -> DeviceTrees:
    """vm_encode_trees over n chunks of the device tensor d_dense (u16 / int16,
    n x 64^3), on torch's current stream."""
    out = out or DeviceTrees(n, palette_cap, torch, d_dense.device)
    s = C.c_void_p(torch.cuda.current_stream(d_dense.device).cuda_stream)
    rc = lib().vm_encode_trees(C.c_void_p(d_dense.data_ptr()), n, palette_cap, C.c_void_p(out.info.data_ptr()),
                               C.c_void_p(out.l1.data_ptr()), C.c_void_p(out.leaves.data_ptr()),
                               C.c_void_p(out.attrs.data_ptr()), C.c_void_p(out.palette.data_ptr()), s)
    if rc:
        raise RuntimeError(f"vm_encode_trees failed ({rc})")
    return out


def insert(world, key: tuple, trees: Trees, i: int, lod: int = 0):
    """World::insert_local of chunk i of trees at key (vmw_insert_tree)."""
    info, l1, leaves, attrs, pal = (np.ascontiguousarray(a) for a in trees.chunk(i))
    rc = lib().vmw_insert_tree(world._h, lod, key[0], key[1], key[2], ptr(info), ptr(l1) if l1.size else None,
                               ptr(leaves) if leaves.size else None, ptr(attrs) if attrs.size else None,
                               ptr(pal) if pal.size else None)
    if rc:
        raise RuntimeError("vmw_insert_tree rejected the chunk")


def same_chunk(a: Trees, i: int, b: Trees, j: int) -> bool:
    ca, cb = a.chunk(i), b.chunk(j)
    return all(np.array_equal(x.view(np.uint8) if x.dtype.names else x, y.view(np.uint8) if y.dtype.names else y)
               for x, y in zip(ca, cb))
