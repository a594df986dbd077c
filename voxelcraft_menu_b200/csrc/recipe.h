// Synthetic terrain of the benchmark worlds: a value-noise heightfield with
// grass / dirt / stone layers, a water level, trees, scattered glass and, for
// sparse worlds, islands.  This is the workload's own definition (the engine's
// worlds come from its worldgen, which these recipes replace), so both the
// product's world store and the oracle's producer include this header and
// see the same dense blocks.  Header-only: every includer gets its own copy.
//
// Chunks of level-of-detail `lod` have voxels of 1 << lod blocks: a coarse
// voxel takes the block of its column's height sample at its top block (the
// way the engine samples coarse chunks, src/worldgen.rs:534-561), with no
// trees and no glass.
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "vm_types.h"
#include "../../include/voxmarch_world.h"

namespace vmr {

inline uint32_t mix32(uint32_t h) {
  h ^= h >> 16; h *= 0x7feb352du; h ^= h >> 15; h *= 0x846ca68bu; h ^= h >> 16;
  return h;
}
inline uint32_t hash3(int32_t x, int32_t y, int32_t z, uint32_t seed) {
  return mix32((uint32_t)x * 0x8da6b343u ^ mix32((uint32_t)y * 0xd8163841u ^ mix32((uint32_t)z * 0xcb1ab31fu ^ seed)));
}
inline float unit(uint32_t h) { return (float)(h >> 8) * (1.0f / 16777216.0f); }

// Value noise: lattice values from hash3, smoothstep-weighted bilinear blend.
inline float value_noise(float x, float z, uint32_t octave, uint32_t seed) {
  float fx = floorf(x), fz = floorf(z);
  int32_t ix = (int32_t)fx, iz = (int32_t)fz;
  float tx = x - fx, tz = z - fz;
  tx = tx * tx * (3.0f - 2.0f * tx);
  tz = tz * tz * (3.0f - 2.0f * tz);
  uint32_t s = seed * 0x9e3779b9u + octave * 0x632be5abu;
  float a = unit(hash3(ix, 0, iz, s)), b = unit(hash3(ix + 1, 0, iz, s));
  float c = unit(hash3(ix, 0, iz + 1, s)), d = unit(hash3(ix + 1, 0, iz + 1, s));
  float ab = a + (b - a) * tx, cd = c + (d - c) * tx;
  return ab + (cd - ab) * tz;
}

// fbm in [0, 1): octaves at base_freq * 2^o with gain 0.5, normalised.
inline float fbm(float x, float z, const vmw_recipe& r) {
  float sum = 0.0f, norm = 0.0f, amp = 1.0f, freq = r.base_freq;
  for (uint32_t o = 0; o < r.octaves; ++o) {
    sum += amp * value_noise(x * freq, z * freq, o, r.seed);
    norm += amp;
    amp *= 0.5f;
    freq *= 2.0f;
  }
  return sum / norm;
}

// Surface height of column (x, z): the first air block above the terrain.
inline int32_t column_height(const vmw_recipe& r, int32_t x, int32_t z) {
  float hf = r.base + r.amplitude * fbm((float)x, (float)z, r);
  int32_t h = (int32_t)floorf(hf);
  if (r.island_permille > 0) {
    // sparse worlds: terrain only where a coarse mask noise is high
    float m = value_noise((float)x * r.base_freq * 0.5f, (float)z * r.base_freq * 0.5f, 97u, r.seed ^ 0xA5A5u);
    if (m * 1000.0f >= (float)r.island_permille) h = 0;
  }
  return std::max(0, std::min(h, (int32_t)r.size[1] - 8));
}

inline bool column_tree(const vmw_recipe& r, int32_t x, int32_t z, int32_t h) {
  bool dry = r.water_level < 0 || h - 1 >= r.water_level;
  return h > 0 && dry && r.tree_permille > 0 && hash3(x, 7, z, r.seed ^ 0x7777u) % 1000u < r.tree_permille;
}

// A foliage tuft on the first air block of a dry grass column without a tree:
// TALL_GRASS, GRASS_TALL or REEDS by the column's hash.
inline uint16_t column_tuft(const vmw_recipe& r, int32_t x, int32_t z, int32_t h, bool tree) {
  if (tree || h <= 0 || r.tuft_permille == 0) return VM_AIR;
  if (r.water_level >= 0 && h - 1 < r.water_level) return VM_AIR;
  const uint32_t k = hash3(x, 11, z, r.seed ^ 0x3131u);
  if (k % 1000u >= r.tuft_permille) return VM_AIR;
  const uint16_t ids[3] = {VM_TALL_GRASS, VM_GRASS_TALL, VM_REEDS};
  return ids[(k >> 10) % 3u];
}

struct Heights {
  uint32_t sx = 0, sz = 0;
  std::vector<int32_t> h;
  std::vector<uint8_t> tree;
  int32_t at(int32_t x, int32_t z) const { return h[(size_t)z * sx + x]; }
};

inline Heights make_heights(const vmw_recipe& r) {
  Heights hs;
  hs.sx = r.size[0]; hs.sz = r.size[2];
  hs.h.resize((size_t)hs.sx * hs.sz);
  hs.tree.assign((size_t)hs.sx * hs.sz, 0);
#pragma omp parallel for schedule(static)
  for (int64_t z = 0; z < (int64_t)hs.sz; ++z)
    for (uint32_t x = 0; x < hs.sx; ++x) {
      const int32_t h = column_height(r, (int32_t)x, (int32_t)z);
      hs.h[(size_t)z * hs.sx + x] = h;
      hs.tree[(size_t)z * hs.sx + x] = column_tree(r, (int32_t)x, (int32_t)z, h) ? 1 : 0;
    }
  return hs;
}

// The block of the surface layers for a block at height y of a column whose
// first air block is h (y < h).
inline uint16_t layer_block(int32_t y, int32_t h) {
  if (y == h - 1) return VM_GRASS;
  if (y >= h - 4) return VM_DIRT;
  return VM_STONE;
}

// One lod-0 chunk's dense block grid (chunk cell cx, cy, cz), dense index
// x | z<<6 | y<<12.
inline void fill_chunk(const vmw_recipe& r, const Heights& hs, int32_t cx, int32_t cy, int32_t cz, uint16_t* dense) {
  memset(dense, 0, sizeof(uint16_t) * 64 * 64 * 64);
  int32_t ox = cx * 64, oy = cy * 64, oz = cz * 64;
  for (int32_t lz = 0; lz < 64; ++lz)
    for (int32_t lx = 0; lx < 64; ++lx) {
      int32_t x = ox + lx, z = oz + lz;
      int32_t h = hs.at(x, z);
      for (int32_t ly = 0; ly < 64; ++ly) {
        int32_t y = oy + ly;
        uint16_t id = VM_AIR;
        if (y < h) {
          id = layer_block(y, h);
          if (r.glass_permille > 0 && y >= h - 2 && hash3(x, y, z, r.seed ^ 0x5151u) % 1000u < r.glass_permille)
            id = VM_GLASS;
        } else if (r.water_level >= 0 && y < r.water_level && (r.island_permille == 0 || y >= r.water_level - r.water_depth)) {
          id = VM_WATER;
        } else if (y == h) {
          id = column_tuft(r, x, z, h, hs.tree[(size_t)z * hs.sx + x] != 0);
        }
        dense[lx | (lz << 6) | (ly << 12)] = id;
      }
    }
  // trees whose trunk or 5x5x3 leaf blob reaches this chunk
  for (int32_t z = std::max(0, oz - 2); z < std::min<int32_t>(hs.sz, oz + 66); ++z)
    for (int32_t x = std::max(0, ox - 2); x < std::min<int32_t>(hs.sx, ox + 66); ++x) {
      if (!hs.tree[(size_t)z * hs.sx + x]) continue;
      int32_t h = hs.at(x, z);
      auto put = [&](int32_t bx, int32_t by, int32_t bz, uint16_t id, bool only_air) {
        int32_t lx = bx - ox, ly = by - oy, lz = bz - oz;
        if (lx < 0 || ly < 0 || lz < 0 || lx >= 64 || ly >= 64 || lz >= 64) return;
        uint16_t& d = dense[lx | (lz << 6) | (ly << 12)];
        if (!only_air || d == VM_AIR) d = id;
      };
      for (int32_t dy = 0; dy < 5; ++dy) put(x, h + dy, z, VM_LOG, false);
      for (int32_t dy = 3; dy < 6; ++dy)
        for (int32_t dz = -2; dz <= 2; ++dz)
          for (int32_t dx = -2; dx <= 2; ++dx) put(x + dx, h + dy, z + dz, VM_LEAVES, true);
    }
}

// One chunk of level `lod` (voxels of s = 1 << lod blocks) at chunk cell
// (cx, cy, cz) of that level: column (x, z) samples the heightfield at block
// (o.x + x s, o.z + z s); a voxel whose bottom block is below the surface
// takes the layer block of its top block inside the terrain, else water below
// the water level.  Columns outside the recipe's extent are empty.
inline void fill_chunk_lod(const vmw_recipe& r, uint32_t lod, int32_t cx, int32_t cy, int32_t cz, uint16_t* dense) {
  memset(dense, 0, sizeof(uint16_t) * 64 * 64 * 64);
  const int32_t s = 1 << lod, ox = cx * 64 * s, oy = cy * 64 * s, oz = cz * 64 * s;
  for (int32_t lz = 0; lz < 64; ++lz)
    for (int32_t lx = 0; lx < 64; ++lx) {
      const int32_t x = ox + lx * s, z = oz + lz * s;
      if (x < 0 || z < 0 || x >= (int32_t)r.size[0] || z >= (int32_t)r.size[2]) continue;
      const int32_t h = column_height(r, x, z);
      for (int32_t ly = 0; ly < 64; ++ly) {
        const int32_t y = oy + ly * s;
        uint16_t id = VM_AIR;
        if (y < h) {
          id = layer_block(std::min(y + s - 1, h - 1), h);
        } else if (r.water_level >= 0 && y < r.water_level &&
                   (r.island_permille == 0 || y + s > r.water_level - r.water_depth)) {
          id = VM_WATER;
        }
        dense[lx | (lz << 6) | (ly << 12)] = id;
      }
    }
}

}  // namespace vmr
