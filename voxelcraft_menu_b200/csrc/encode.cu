// GPU tree encoder: build_local (src/voxel/tree.rs:89-204, encode_leaf
// src/voxel/attributes.rs:90-139) for a batch of dense 64^3 chunks, one CTA
// per chunk, written in the flat layout of vm_tree_info (vm_types.h).
//
// The CPU encoder walks L1 nodes (l1z, l1y, l1x), their leaves (lz, ly, lx)
// and each leaf's voxels (vz, vy, vx), appending leaf masks, attribute
// entries and palette words as it goes.  Those orders are the ascending
// cell_bit orders, so here:
//   pass 1  a warp per L1 node takes its 64 leaves one by one, 2 voxels per
//           lane: the occupancy mask by two ballots, the palette (ids in order
//           of first appearance) by electing the lowest unassigned voxel per
//           round, and the leaf's palette word count; the L1 node's dry flag
//           and water line and the chunk's flags, emitter count and bounds;
//   scan    a block scan over the 4096 leaves in that order gives every leaf
//           its attribute index, kept-leaf index and palette offset;
//   pass 2  the warps write the L1 nodes, leaf masks, attribute entries and
//           palette words at those offsets (palettes recomputed, voxels
//           re-read from L2), which is the CPU encoder's output bit for bit.
#include <cub/block/block_scan.cuh>
#include "../../include/voxmarch.h"
#include "kernels.cuh"

namespace vmk {

constexpr uint32_t ENC_THREADS = 256, ENC_WARPS = ENC_THREADS / 32;
constexpr uint64_t CHUNK_VOXELS = 64ull * 64ull * 64ull;
constexpr uint32_t ENC_FULL = 0xFFFFFFFFu;

__device__ __forceinline__ bool enc_foliage(uint32_t id) { return id == VM_TALL_GRASS || id == VM_GRASS_TALL || id == VM_REEDS; }
__device__ __forceinline__ bool enc_cutout(uint32_t id) { return id == VM_LEAVES || id == VM_PINE_LEAVES; }
__device__ __forceinline__ bool enc_emitter(uint32_t id) {
  return id == VM_GLOWSTONE || id == VM_AMBER_LAMP || id == VM_AZURE_LAMP || id == VM_VERDANT_LAMP;
}
__device__ __forceinline__ uint32_t enc_bits(uint32_t n) { return n <= 2u ? 1u : (n <= 4u ? 2u : (n <= 16u ? 4u : 8u)); }
// palette words of a leaf with n distinct ids: none when uniform, else the
// header, the packed ids and 64 * bits index bits
__device__ __forceinline__ uint32_t enc_words(uint32_t n) { return n <= 1u ? 0u : 1u + (n + 1u) / 2u + 2u * enc_bits(n); }

struct EncShared {
  unsigned long long mask[4096];     // per leaf (L1 index * 64 + leaf index): occupancy
  uint16_t pal0[4096];               // first id of the leaf
  uint8_t words[4096];               // palette words of the leaf
  uint16_t pal[ENC_WARPS][64];       // pass 2: the palette a warp is encoding
  uint8_t l1_full[64], l1_dry[64], l1_wl[64];
  uint32_t l1_attr[64], l1_kept[64], l1_word[64], l1_slot[64];
  uint32_t flags, emitters, amin[3], amax[3], first;
  uint32_t n_attrs, n_kept, n_words, solid;
};

// The two voxels of lane `lane` in leaf (bx, by, bz): cell bits lane and lane + 32.
__device__ __forceinline__ void enc_load(const uint16_t* __restrict__ dense, uint32_t bx, uint32_t by, uint32_t bz,
                                         uint32_t lane, uint32_t* id0, uint32_t* id1) {
  const uint32_t vx = lane & 3u, vy = (lane >> 2) & 3u, vz = lane >> 4;
  const uint32_t x = bx + vx, y = by + vy;
  *id0 = __ldg(dense + (x | ((bz + vz) << 6) | (y << 12)));
  *id1 = __ldg(dense + (x | ((bz + vz + 2u) << 6) | (y << 12)));
}

// The palette of a leaf: *p0 / *p1 the palette index of the lane's voxels,
// returns the number of distinct ids (first appearance order); pal (if not
// null) receives them.
__device__ __forceinline__ uint32_t enc_palette(uint32_t id0, uint32_t id1, bool in0, bool in1, uint32_t* p0,
                                                uint32_t* p1, uint32_t* first, uint16_t* pal) {
  uint32_t n = 0;
  *p0 = *p1 = 0xFFu;
  for (;;) {
    const uint32_t u0 = __ballot_sync(ENC_FULL, in0 && *p0 == 0xFFu);
    const uint32_t u1 = __ballot_sync(ENC_FULL, in1 && *p1 == 0xFFu);
    if ((u0 | u1) == 0u) break;
    const bool hi = u0 == 0u;
    const uint32_t src = (uint32_t)__ffs(hi ? u1 : u0) - 1u;
    const uint32_t id = __shfl_sync(ENC_FULL, hi ? id1 : id0, (int)src);
    if (n == 0u) *first = id;
    if (pal) pal[n] = (uint16_t)id;
    if (in0 && id0 == id) *p0 = n;
    if (in1 && id1 == id) *p1 = n;
    ++n;
  }
  return n;
}

__global__ void __launch_bounds__(ENC_THREADS) k_encode(const uint16_t* __restrict__ dense_all, uint32_t palette_cap,
                                                        vm_tree_info* __restrict__ info_all,
                                                        vm_tree_l1* __restrict__ l1_all,
                                                        unsigned long long* __restrict__ leaves_all,
                                                        uint32_t* __restrict__ attrs_all,
                                                        uint32_t* __restrict__ palette_all) {
  typedef cub::BlockScan<uint32_t, ENC_THREADS> Scan;
  __shared__ EncShared s;
  __shared__ typename Scan::TempStorage scan_tmp;
  const uint32_t c = blockIdx.x, lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  const uint16_t* dense = dense_all + (uint64_t)c * CHUNK_VOXELS;
  if (threadIdx.x == 0) {
    s.flags = 0u; s.emitters = 0u; s.first = ENC_FULL; s.solid = 0u;
    for (int i = 0; i < 3; ++i) { s.amin[i] = 64u; s.amax[i] = 0u; }
  }
  __syncthreads();

  // ---- pass 1 ----------------------------------------------------------------
  // Statistics are kept per lane (its two voxels of every leaf) and reduced
  // once per L1 node (dry flag, water line) or once per warp (flags, emitter
  // count, bounds); the next leaf's voxels are loaded while one is encoded.
  uint32_t flags = 0u, emitters = 0u, mn[3] = {64u, 64u, 64u}, mx[3] = {0u, 0u, 0u};
  const uint32_t vx = lane & 3u, vy = (lane >> 2) & 3u, vz = lane >> 4;
  for (uint32_t li = warp; li < 64u; li += ENC_WARPS) {
    const uint32_t l1x = li & 3u, l1y = (li >> 2) & 3u, l1z = li >> 4;
    bool all_full = true, dry = false;
    uint32_t top = 0u;   // 1 + highest non-water y of the lane's voxels in the node, 0: none
    uint32_t nx0, nx1;
    enc_load(dense, l1x * 16u, l1y * 16u, l1z * 16u, lane, &nx0, &nx1);
    for (uint32_t j = 0; j < 64u; ++j) {
      const uint32_t lx = j & 3u, ly = (j >> 2) & 3u, lz = j >> 4;
      const uint32_t bx = l1x * 16u + lx * 4u, by = l1y * 16u + ly * 4u, bz = l1z * 16u + lz * 4u;
      const uint32_t id0 = nx0, id1 = nx1;
      if (j + 1u < 64u) {
        const uint32_t k = j + 1u;
        enc_load(dense, l1x * 16u + (k & 3u) * 4u, l1y * 16u + ((k >> 2) & 3u) * 4u, l1z * 16u + (k >> 4) * 4u,
                 lane, &nx0, &nx1);
      }
      const bool in0 = id0 != VM_AIR, in1 = id1 != VM_AIR;
      const uint32_t mlo = __ballot_sync(ENC_FULL, in0), mhi = __ballot_sync(ENC_FULL, in1);
      const unsigned long long m = ((unsigned long long)mhi << 32) | mlo;
      const uint32_t g = li * 64u + j;
      if (m == 0ull) {
        all_full = false;
        if (lane == 0) { s.mask[g] = 0ull; s.words[g] = 0; s.pal0[g] = 0; }
        continue;
      }
      if (m != ~0ull) all_full = false;
      // the first present voxel's id; a leaf of that id alone (the common
      // case) needs no palette rounds and its statistics are the id's
      const uint32_t fv = (uint32_t)__ffsll((long long)m) - 1u;
      uint32_t first = __shfl_sync(ENC_FULL, fv >= 32u ? id1 : id0, (int)(fv & 31u));
      const bool one = __all_sync(ENC_FULL, (!in0 || id0 == first) && (!in1 || id1 == first));
      uint32_t n = 1u;
      if (!one) {
        uint32_t p0, p1;
        n = enc_palette(id0, id1, in0, in1, &p0, &p1, &first, nullptr);
      }
      if (lane == 0) { s.mask[g] = m; s.words[g] = (uint8_t)enc_words(n); s.pal0[g] = (uint16_t)first; }
      if (one) {
        if (first == VM_WATER) flags |= VM_TREE_WATER;
        else if (in0 || in1) { dry = true; top = max(top, ly * 4u + vy + 1u); }
        if (enc_foliage(first)) flags |= VM_TREE_FOLIAGE;
        if (enc_cutout(first)) flags |= VM_TREE_CUTOUT;
        if (first == VM_GLASS) flags |= VM_TREE_GLASS;
        if (enc_emitter(first) && lane == 0) emitters += (uint32_t)__popcll(m);
      } else {
        // the lane's statistics
        const bool w0 = in0 && id0 == VM_WATER, w1 = in1 && id1 == VM_WATER;
        const bool d0 = in0 && !w0, d1 = in1 && !w1;
        if (w0 || w1) flags |= VM_TREE_WATER;
        if (d0 || d1) { dry = true; top = max(top, ly * 4u + vy + 1u); }
        if ((in0 && enc_foliage(id0)) || (in1 && enc_foliage(id1))) flags |= VM_TREE_FOLIAGE;
        if ((in0 && enc_cutout(id0)) || (in1 && enc_cutout(id1))) flags |= VM_TREE_CUTOUT;
        if ((in0 && id0 == VM_GLASS) || (in1 && id1 == VM_GLASS)) flags |= VM_TREE_GLASS;
        emitters += (in0 && enc_emitter(id0) ? 1u : 0u) + (in1 && enc_emitter(id1) ? 1u : 0u);
      }
      if (in0 || in1) {
        const uint32_t x = bx + vx, y = by + vy;
        mn[0] = min(mn[0], x); mx[0] = max(mx[0], x + 1u);
        mn[1] = min(mn[1], y); mx[1] = max(mx[1], y + 1u);
        mn[2] = min(mn[2], in0 ? bz + vz : bz + vz + 2u);
        mx[2] = max(mx[2], (in1 ? bz + vz + 2u : bz + vz) + 1u);
      }
    }
    const bool node_dry = __any_sync(ENC_FULL, dry);
    const uint32_t node_top = __reduce_max_sync(ENC_FULL, top);
    if (lane == 0) {
      s.l1_full[li] = all_full ? 1 : 0;
      s.l1_dry[li] = node_dry ? 1 : 0;
      s.l1_wl[li] = node_dry ? (uint8_t)(node_top - 1u) : 15;
    }
  }
  if (emitters) flags |= VM_TREE_EMITTER;
  flags = __reduce_or_sync(ENC_FULL, flags);
  emitters = __reduce_add_sync(ENC_FULL, emitters);
  for (int i = 0; i < 3; ++i) { mn[i] = __reduce_min_sync(ENC_FULL, mn[i]); mx[i] = __reduce_max_sync(ENC_FULL, mx[i]); }
  if (lane == 0) {
    atomicOr(&s.flags, flags);
    atomicAdd(&s.emitters, emitters);
    for (int i = 0; i < 3; ++i) { atomicMin(&s.amin[i], mn[i]); atomicMax(&s.amax[i], mx[i]); }
  }
  __syncthreads();

  // ---- scan: thread t owns leaves [16 t, 16 t + 16) ---------------------------
  const uint32_t g0 = threadIdx.x * 16u;
  uint32_t n_present = 0, n_kept = 0, n_words = 0, solid = 0, first_leaf = ENC_FULL;
#pragma unroll 4
  for (uint32_t k = 0; k < 16u; ++k) {
    const uint32_t g = g0 + k;
    const unsigned long long m = s.mask[g];
    if (m == 0ull) continue;
    first_leaf = min(first_leaf, g);
    ++n_present;
    if (!s.l1_full[g >> 6]) ++n_kept;
    n_words += s.words[g];
    solid += (uint32_t)__popcll(m);
  }
  uint32_t attr_base, kept_base, word_base, tot;
  Scan(scan_tmp).ExclusiveSum(n_present, attr_base, tot);
  if (threadIdx.x == 0) s.n_attrs = tot;
  __syncthreads();
  Scan(scan_tmp).ExclusiveSum(n_kept, kept_base, tot);
  if (threadIdx.x == 0) s.n_kept = tot;
  __syncthreads();
  Scan(scan_tmp).ExclusiveSum(n_words, word_base, tot);
  if (threadIdx.x == 0) s.n_words = tot;
  if ((g0 & 63u) == 0u) {          // the first thread of each L1 node
    s.l1_attr[g0 >> 6] = attr_base;
    s.l1_kept[g0 >> 6] = kept_base;
    s.l1_word[g0 >> 6] = word_base;
  }
  atomicAdd(&s.solid, solid);
  if (first_leaf != ENC_FULL) atomicMin(&s.first, first_leaf);
  __syncthreads();
  // uniform: every present voxel has the chunk's first id (each leaf a single
  // id, all the same)
  const uint32_t first_id = s.first != ENC_FULL ? s.pal0[s.first] : 0u;
  int mixed = 0;
  for (uint32_t k = 0; k < 16u; ++k) {
    const uint32_t g = g0 + k;
    if (s.mask[g] != 0ull && (s.words[g] != 0 || s.pal0[g] != first_id)) mixed = 1;
  }
  const int any_mixed = __syncthreads_or(mixed);
  const bool uniform = s.first != ENC_FULL && !any_mixed;
  if (warp == 0) {                 // compacted L1 slots
    const bool ne0 = s.l1_attr[lane] != (lane < 63u ? s.l1_attr[lane + 1u] : s.n_attrs);
    const bool ne1 = s.l1_attr[lane + 32u] != (lane + 32u < 63u ? s.l1_attr[lane + 33u] : s.n_attrs);
    const uint32_t b0 = __ballot_sync(ENC_FULL, ne0), b1 = __ballot_sync(ENC_FULL, ne1);
    s.l1_slot[lane] = ne0 ? (uint32_t)__popc(b0 & ((1u << lane) - 1u)) : ENC_FULL;
    s.l1_slot[lane + 32u] = ne1 ? (uint32_t)__popc(b0) + (uint32_t)__popc(b1 & ((1u << lane) - 1u)) : ENC_FULL;
  }
  __syncthreads();

  // ---- pass 2 ----------------------------------------------------------------
  vm_tree_l1* l1_out = l1_all + (uint64_t)c * VM_TREE_L1;
  unsigned long long* leaves = leaves_all + (uint64_t)c * VM_TREE_LEAVES;
  uint32_t* attrs = attrs_all + (uint64_t)c * VM_TREE_LEAVES;
  uint32_t* palette = palette_all + (uint64_t)c * palette_cap;
  uint16_t* pal = s.pal[warp];
  for (uint32_t li = warp; li < 64u; li += ENC_WARPS) {
    const uint32_t slot = s.l1_slot[li];
    if (slot == ENC_FULL) continue;
    const bool full = s.l1_full[li] != 0;
    const unsigned long long lm = ((unsigned long long)__ballot_sync(ENC_FULL, s.mask[li * 64u + 32u + lane] != 0ull) << 32) |
                                  __ballot_sync(ENC_FULL, s.mask[li * 64u + lane] != 0ull);
    if (lane == 0) {
      vm_tree_l1 o;
      memset(&o, 0, sizeof o);
      o.mask = lm;
      o.leaf_start = s.l1_kept[li];
      o.leaf_prefix = s.l1_attr[li];
      o.full = full ? 1 : 0;
      o.water_line = s.l1_wl[li];
      l1_out[slot] = o;
    }
    uint32_t a_run = s.l1_attr[li], k_run = s.l1_kept[li], w_run = s.l1_word[li];
    const uint32_t l1x = li & 3u, l1y = (li >> 2) & 3u, l1z = li >> 4;
    for (uint32_t j = 0; j < 64u; ++j) {
      const uint32_t g = li * 64u + j;
      const unsigned long long m = s.mask[g];
      if (m == 0ull) continue;
      const uint32_t words = s.words[g];
      if (!full && lane == 0) leaves[k_run] = m;
      if (!uniform) {
        if (words == 0u) {
          if (lane == 0) attrs[a_run] = VM_UNIFORM_BIT | s.pal0[g];
        } else {
          if (lane == 0) attrs[a_run] = w_run;
          const uint32_t lx = j & 3u, ly = (j >> 2) & 3u, lz = j >> 4;
          uint32_t id0, id1;
          enc_load(dense, l1x * 16u + lx * 4u, l1y * 16u + ly * 4u, l1z * 16u + lz * 4u, lane, &id0, &id1);
          const bool in0 = id0 != VM_AIR, in1 = id1 != VM_AIR;
          uint32_t p0, p1, first;
          const uint32_t n = enc_palette(id0, id1, in0, in1, &p0, &p1, &first, lane == 0 ? pal : nullptr);
          __syncwarp();
          const uint32_t bits = enc_bits(n), npw = (n + 1u) / 2u, niw = 2u * bits;
          // every word below palette_cap is written (a leaf may straddle it)
          const auto put = [&](uint32_t at, uint32_t v) { if (at < palette_cap) palette[at] = v; };
          // index words: voxel v at bit v * bits
          const uint32_t b0 = lane * bits, b1 = (lane + 32u) * bits;
          const uint32_t c0 = in0 ? p0 << (b0 & 31u) : 0u, c1 = in1 ? p1 << (b1 & 31u) : 0u;
          uint32_t mine = 0u;
          for (uint32_t wi = 0; wi < niw; ++wi) {
            const uint32_t v = __reduce_or_sync(ENC_FULL, ((b0 >> 5) == wi ? c0 : 0u) | ((b1 >> 5) == wi ? c1 : 0u));
            if (lane == wi) mine = v;
          }
          if (lane == 0) put(w_run, n | (bits << 8));
          if (lane < npw)
            put(w_run + 1u + lane,
                (uint32_t)pal[2u * lane] | ((2u * lane + 1u < n ? (uint32_t)pal[2u * lane + 1u] : 0u) << 16));
          if (lane < niw) put(w_run + 1u + npw + lane, mine);
          __syncwarp();
        }
      }
      ++a_run;
      w_run += words;
      if (!full) ++k_run;
    }
  }

  if (threadIdx.x == 0) {
    vm_tree_info in;
    memset(&in, 0, sizeof in);
    unsigned long long root = 0ull, drym = 0ull;
    uint32_t n_l1 = 0;
    for (uint32_t li = 0; li < 64u; ++li) {
      if (s.l1_slot[li] == ENC_FULL) continue;
      root |= 1ull << li;
      ++n_l1;
      if (s.l1_dry[li]) drym |= 1ull << li;
    }
    in.root_mask = root;
    in.dry_mask = drym;
    in.uniform = uniform ? (int32_t)first_id : -1;
    in.flags = s.flags;
    in.emitters = s.emitters;
    in.solid_count = s.solid;
    in.leaf_count = s.n_attrs;
    in.n_l1 = n_l1;
    in.n_leaves = s.n_kept;
    in.n_attrs = uniform ? 0u : s.n_attrs;
    in.n_palette = uniform ? 0u : s.n_words;
    if (in.n_palette > palette_cap) in.flags |= VM_TREE_PALETTE_OVERFLOW;
    if (s.solid > 0u)
      for (int i = 0; i < 3; ++i) { in.aabb_min[i] = (uint8_t)s.amin[i]; in.aabb_max[i] = (uint8_t)s.amax[i]; }
    info_all[c] = in;
  }
}

}  // namespace vmk

extern "C" int vm_encode_trees(const uint16_t* d_dense, uint32_t n_chunks, uint32_t palette_cap, vm_tree_info* d_info,
                               vm_tree_l1* d_l1, uint64_t* d_leaves, uint32_t* d_attrs, uint32_t* d_palette,
                               void* stream) {
  if (n_chunks == 0) return VM_OK;
  if (!d_dense || !d_info || !d_l1 || !d_leaves || !d_attrs || (palette_cap && !d_palette)) return VM_E_INVALID;
  vmk::k_encode<<<n_chunks, vmk::ENC_THREADS, 0, (cudaStream_t)stream>>>(
      d_dense, palette_cap, d_info, d_l1, reinterpret_cast<unsigned long long*>(d_leaves), d_attrs, d_palette);
  return cudaGetLastError() == cudaSuccess ? VM_OK : VM_E_CUDA;
}
