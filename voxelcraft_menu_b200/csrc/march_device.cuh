// Device-side traversal of the engine's 64-tree chunks, sm_100a.
//
// Numerical contract (shared with the CPU oracle so that results are
// bit-identical): this translation unit is compiled with --fmad=false and IEEE
// division / sqrt, floor/ceil are exact, float->int conversions saturate
// (cvt.rzi), and min/max are IEEE minNum/maxNum.  Every function cites the
// WGSL it re-implements (src/render/shaders/*.wgsl in the reference).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "vm_types.h"

namespace vmd {

// Device view of the world pools.  Every index computed from the data is
// checked against the pool size; a bad index records an error code in *err
// and reads element 0 instead, so malformed pools never fault.
struct DevWorld {
  const vm_chunk* chunks; uint32_t n_chunks;
  const uint4* inners; uint64_t n_inners;
  const uint2* leaves; uint64_t n_leaves;
  const uint32_t* bricks; uint64_t n_bricks;
  const uint32_t* grid; uint64_t n_grid;
  uint32_t* err;
  uint32_t spec;     // VM_SPEC_* pipeline specialisations
  // the atlas alpha the tuft cross-quads test (the engine's atlas, sampled at
  // an explicit level), [mip][layer][y][x] for mips 16, 8, 4, 2; null: no
  // atlas uploaded, tufts stay transparent
  const float* atlas_alpha; uint32_t atlas_layers;
  uint32_t tuft_layer[3];   // block_faces[id * 8 + NORMAL_CROSS_A] of TALL_GRASS, GRASS_TALL, REEDS
};

enum : uint32_t { ERR_CHUNK = 1u, ERR_INNER = 2u, ERR_LEAF = 4u, ERR_BRICK = 8u, ERR_GRID = 16u, ERR_LIST = 32u };

__device__ __forceinline__ void flag(const DevWorld& w, uint32_t e) { atomicOr(w.err, e); }

__device__ __forceinline__ uint4 ld_inner(const DevWorld& w, uint64_t i) {
  if (i >= w.n_inners) { flag(w, ERR_INNER); i = 0; }
  return __ldg(w.inners + i);
}
__device__ __forceinline__ uint2 ld_leaf(const DevWorld& w, uint64_t i) {
  if (i >= w.n_leaves) { flag(w, ERR_LEAF); i = 0; }
  return __ldg(w.leaves + i);
}
__device__ __forceinline__ uint32_t ld_brick(const DevWorld& w, uint64_t i) {
  if (i >= w.n_bricks) { flag(w, ERR_BRICK); i = 0; }
  return __ldg(w.bricks + i);
}
__device__ __forceinline__ uint32_t ld_grid(const DevWorld& w, uint64_t i) {
  if (i >= w.n_grid) { flag(w, ERR_GRID); return VM_NO_CHUNK; }
  return __ldg(w.grid + i);
}

// The march-relevant part of a GpuChunk, loaded with six 128-bit loads.
struct Chunk {
  float aabb_min[3]; float vs;
  float aabb_max[3]; uint32_t lod;
  float origin[3]; float fade;
  uint32_t root[4];
  uint32_t attr_base, attr_flags, light_base, light_flags;
  uint32_t dry[2], res[2];
};
static_assert(sizeof(Chunk) == 96, "Chunk mirrors vm_chunk");

__device__ __forceinline__ Chunk ld_chunk(const DevWorld& w, uint32_t ci) {
  if (ci >= w.n_chunks) { flag(w, ERR_CHUNK); ci = 0; }
  const uint4* p = reinterpret_cast<const uint4*>(w.chunks + ci);
  Chunk c;
  uint4* d = reinterpret_cast<uint4*>(&c);
#pragma unroll
  for (int i = 0; i < 6; ++i) d[i] = __ldg(p + i);
  return c;
}

struct F3 { float x, y, z; };
__device__ __forceinline__ F3 f3(float x, float y, float z) { return {x, y, z}; }
__device__ __forceinline__ F3 operator+(F3 a, F3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ F3 operator-(F3 a, F3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ F3 operator*(F3 a, F3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
__device__ __forceinline__ F3 operator*(F3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ F3 operator/(F3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }
__device__ __forceinline__ F3 neg(F3 a) { return {-a.x, -a.y, -a.z}; }
__device__ __forceinline__ float dot(F3 a, F3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ F3 cross(F3 a, F3 b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ F3 ld3(const float* p) { return {p[0], p[1], p[2]}; }
__device__ __forceinline__ float comp(F3 a, uint32_t i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }
__device__ __forceinline__ float signf(float x) { return x > 0.0f ? 1.0f : (x < 0.0f ? -1.0f : 0.0f); }
__device__ __forceinline__ float tiny_fix(float d) { return fabsf(d) < 1e-6f ? 1e-6f * signf(d + 1e-9f) : d; }
__device__ __forceinline__ int32_t ffloor_i(float x) { return __float2int_rd(x); }
__device__ __forceinline__ int32_t fceil_i(float x) { return __float2int_ru(x); }
__device__ __forceinline__ uint32_t popc(uint32_t x) { return __popc(x); }

// x / d for the scales the march divides by.  Voxel sizes (1 << lod) and the
// 64-voxel chunk edge are powers of two; for those, IEEE division and
// multiplication by the exact reciprocal round the same real number x * 2^-k
// and give identical results (subnormals included, as -ftz=false keeps them),
// so the multiply replaces a multi-instruction correctly rounded divide.
// Other divisors keep the division.
struct Scale { float d, inv; bool pow2; };
__device__ __forceinline__ Scale make_scale(float d) {
  const uint32_t b = __float_as_uint(d);
  const uint32_t e = (b >> 23) & 0xFFu;
  Scale s;
  s.d = d;
  s.pow2 = (b & 0x807FFFFFu) == 0u && e >= 27u && e <= 227u;
  s.inv = s.pow2 ? __uint_as_float((254u - e) << 23) : 0.0f;
  return s;
}
__device__ __forceinline__ float sdiv(float x, const Scale& s) { return s.pow2 ? x * s.inv : x / s.d; }
constexpr float INV64 = 1.0f / 64.0f;   // exact: dividing by 64 == multiplying by 2^-6

__device__ __forceinline__ uint32_t cell_bit(uint32_t x, uint32_t y, uint32_t z) { return x | (y << 2) | (z << 4); }
__device__ __forceinline__ bool mask_has(uint32_t lo, uint32_t hi, uint32_t bit) {
  return bit < 32u ? ((lo >> bit) & 1u) != 0u : ((hi >> (bit - 32u)) & 1u) != 0u;
}
__device__ __forceinline__ uint32_t mask_below(uint32_t lo, uint32_t hi, uint32_t bit) {
  // popcount of the mask bits strictly below `bit` (common.wgsl:306-314)
  uint64_t m = ((uint64_t)hi << 32) | lo;
  return (uint32_t)__popcll(m & ((1ull << bit) - 1ull));
}
// 2x2x2 sub-block occupancy test below base bit `sh` (common.wgsl:764-773,781-790)
__device__ __forceinline__ bool block2_empty(uint32_t lo, uint32_t hi, uint32_t sh) {
  uint64_t m = ((uint64_t)hi << 32) | lo;
  return ((uint32_t)(m >> sh) & 0x00330033u) == 0u;
}

// ray_dir: common.wgsl:358-368
__device__ __forceinline__ F3 ray_dir(const vm_frame& f, float px, float py) {
  float ndc_x = ((px + f.jitter[0]) / (float)f.res[0]) * 2.0f - 1.0f;
  float ndc_y = 1.0f - ((py + f.jitter[1]) / (float)f.res[1]) * 2.0f;
  F3 v = (ld3(f.cam_fwd) + ld3(f.cam_right) * (ndc_x * f.tan_half_fov * f.aspect)) +
         ld3(f.cam_up) * (ndc_y * f.tan_half_fov);
  float l = sqrtf(dot(v, v));
  F3 d = {v.x / l, v.y / l, v.z / l};
  return {tiny_fix(d.x), tiny_fix(d.y), tiny_fix(d.z)};
}

// dither / ray_skips: common.wgsl:370-385
__device__ __forceinline__ bool ray_skips(const vm_frame& f, float fade, uint32_t px, uint32_t py) {
  if (fade >= 1.0f) return false;
  float p0 = (float)px + 5.588238f * (float)f.frame_index;
  float p1 = (float)py;
  float x = p0 * 0.06711056f + p1 * 0.00583715f;
  x = x - floorf(x);
  float d = 52.9829189f * x;
  d = d - floorf(d);
  if (fade >= 0.0f) return d >= fade;
  return d < -fade;
}

// normal_of: common.wgsl:387-398
__device__ __forceinline__ F3 normal_of(uint32_t id) {
  if (id >= VM_NORMAL_CROSS_A) {
    float s = id == VM_NORMAL_CROSS_B ? 1.0f : -1.0f;
    return {0.70710678f, 0.0f, s * 0.70710678f};
  }
  uint32_t axis = id >> 1u;
  float s = (id & 1u) == 1u ? 1.0f : -1.0f;
  if (axis == 0u) return {s, 0.0f, 0.0f};
  if (axis == 1u) return {0.0f, s, 0.0f};
  return {0.0f, 0.0f, s};
}

// hash_u32 / leaf_solid: common.wgsl:1422-1430, 514-518
__device__ __forceinline__ uint32_t hash_u32(uint32_t h) {
  h ^= h >> 16u; h *= 0x7feb352du; h ^= h >> 15u; h *= 0x846ca68bu; h ^= h >> 16u;
  return h;
}
__device__ __forceinline__ float leaf_fill(uint32_t spec) {   // SPEC_LEAF_FILL
  return (spec & VM_SPEC_LEAF_THIN) ? VM_LEAF_FILL : VM_LEAF_FILL_PRE43;
}
__device__ __forceinline__ bool leaf_solid(int32_t wx, int32_t wy, int32_t wz, uint32_t mx, uint32_t my, uint32_t mz,
                                           float fill = VM_LEAF_FILL) {
  uint32_t qx = (uint32_t)wx * 4u + mx, qy = (uint32_t)wy * 4u + my, qz = (uint32_t)wz * 4u + mz;
  uint32_t h = hash_u32((qx * 73856093u) ^ (qy * 19349663u) ^ (qz * 83492791u));
  return (float)(h >> 8u) * (1.0f / 16777216.0f) < fill;
}

// leaf_block: common.wgsl:320-334
__device__ __forceinline__ uint32_t leaf_block(const DevWorld& w, uint32_t entry, uint32_t vx, uint32_t vy, uint32_t vz) {
  if ((entry & VM_UNIFORM_BIT) != 0u) return entry & 0xFFFFu;
  uint32_t hdr = ld_brick(w, entry);
  uint32_t n = hdr & 0xFFu;
  uint32_t bits = (hdr >> 8u) & 0xFFu;
  uint32_t pal_words = (n + 1u) / 2u;
  uint32_t vb = cell_bit(vx & 3u, vy & 3u, vz & 3u);
  uint32_t bitpos = vb * bits;
  uint32_t wd = ld_brick(w, (uint64_t)entry + 1u + pal_words + (bitpos >> 5u));
  uint32_t idx = (wd >> (bitpos & 31u)) & ((bits >= 32u ? 0u : (1u << bits)) - 1u);
  uint32_t pw = ld_brick(w, (uint64_t)entry + 1u + idx / 2u);
  return (pw >> ((idx & 1u) * 16u)) & 0xFFFFu;
}

// leaf_attr + block_at: common.wgsl:336-356
__device__ __forceinline__ uint32_t block_at(const DevWorld& w, const Chunk& c, uint32_t vx, uint32_t vy, uint32_t vz) {
  if ((c.attr_flags & VM_ATTR_UNIFORM) != 0u) return c.attr_base;
  uint32_t l1b = cell_bit(vx >> 4, vy >> 4, vz >> 4);
  uint4 l1;
  if ((c.root[2] & VM_FULL_BIT) != 0u) {
    l1 = make_uint4(0xFFFFFFFFu, 0xFFFFFFFFu, VM_FULL_BIT, l1b * 64u);
  } else {
    l1 = ld_inner(w, (uint64_t)(c.root[2] & VM_PTR_MASK) + mask_below(c.root[0], c.root[1], l1b));
  }
  uint32_t lfb = cell_bit((vx >> 2) & 3u, (vy >> 2) & 3u, (vz >> 2) & 3u);
  uint32_t entry = ld_brick(w, (uint64_t)c.attr_base + (l1.w & 0x0FFFFFFFu) + mask_below(l1.x, l1.y, lfb));
  return leaf_block(w, entry, vx, vy, vz);
}

// voxel_occupied: common.wgsl:912-940
__device__ __forceinline__ bool voxel_occupied(const DevWorld& w, const Chunk& c, int32_t x, int32_t y, int32_t z) {
  if (x < 0 || y < 0 || z < 0 || x > 63 || y > 63 || z > 63) return false;
  uint32_t ux = x, uy = y, uz = z;
  uint32_t l1b = cell_bit(ux >> 4, uy >> 4, uz >> 4);
  if (!mask_has(c.root[0], c.root[1], l1b)) return false;
  if ((c.root[2] & VM_FULL_BIT) != 0u) return true;
  uint4 l1 = ld_inner(w, (uint64_t)(c.root[2] & VM_PTR_MASK) + mask_below(c.root[0], c.root[1], l1b));
  if ((l1.z & VM_FULL_BIT) != 0u) return true;
  uint32_t lfb = cell_bit((ux >> 2) & 3u, (uy >> 2) & 3u, (uz >> 2) & 3u);
  if (!mask_has(l1.x, l1.y, lfb)) return false;
  uint2 leaf = ld_leaf(w, (uint64_t)(l1.z & VM_PTR_MASK) + mask_below(l1.x, l1.y, lfb));
  return mask_has(leaf.x, leaf.y, cell_bit(ux & 3u, uy & 3u, uz & 3u));
}

// i32 subtraction with WGSL's wrapping semantics (a cell from the floor of an
// infinite coordinate saturates to INT32_MAX / INT32_MIN and may overflow)
__device__ __forceinline__ int32_t wsub(int32_t a, int32_t b) { return (int32_t)((uint32_t)a - (uint32_t)b); }

__device__ __forceinline__ bool grid_rel(const vm_frame& f, int32_t cx, int32_t cy, int32_t cz, uint64_t* idx) {
  int32_t rx = wsub(cx, f.grid_min[0]), ry = wsub(cy, f.grid_min[1]), rz = wsub(cz, f.grid_min[2]);
  if (rx < 0 || ry < 0 || rz < 0 || rx >= (int32_t)f.grid_dim[0] || ry >= (int32_t)f.grid_dim[1] ||
      rz >= (int32_t)f.grid_dim[2])
    return false;
  *idx = (uint64_t)(uint32_t)rx + (uint64_t)(uint32_t)ry * f.grid_dim[0] +
         (uint64_t)(uint32_t)rz * f.grid_dim[0] * f.grid_dim[1];
  return true;
}

// world_block_at: common.wgsl:266-277.  Inlined (as is cutout_march): an
// out-of-line call made the march kernels save and restore their live
// registers around it (a stack frame and spills), which cost more than the
// larger body.
static __device__ __forceinline__ uint32_t world_block_at(const DevWorld& w, const vm_frame& f, F3 p) {
  uint64_t gi;
  if (!grid_rel(f, ffloor_i(p.x * INV64), ffloor_i(p.y * INV64), ffloor_i(p.z * INV64), &gi)) return 0u;
  uint32_t ci = ld_grid(w, gi);
  if (ci == VM_NO_CHUNK) return 0u;
  Chunk c = ld_chunk(w, ci);
  const Scale s = make_scale(c.vs);
  int32_t vx = ffloor_i(sdiv(p.x - c.origin[0], s));
  int32_t vy = ffloor_i(sdiv(p.y - c.origin[1], s));
  int32_t vz = ffloor_i(sdiv(p.z - c.origin[2], s));
  if (vx < 0 || vy < 0 || vz < 0 || vx >= 64 || vy >= 64 || vz >= 64) return 0u;
  if (!voxel_occupied(w, c, vx, vy, vz)) return 0u;
  return block_at(w, c, vx, vy, vz);
}

struct Hit {
  bool hit; float t; uint32_t normal;
  uint32_t vx, vy, vz;
  uint32_t mx, my, mz;
  uint32_t iters;
  uint32_t id;    // block id of the hit voxel (march_chunk<..., WANT_ID = true> only)
};

__device__ __forceinline__ bool is_tuft(uint32_t b) { return b == VM_TALL_GRASS || b == VM_GRASS_TALL || b == VM_REEDS; }
__device__ __forceinline__ bool is_cutout_id(uint32_t b) { return b == VM_LEAVES || b == VM_PINE_LEAVES; }

// micro_entry: common.wgsl:520-528
__device__ __forceinline__ void micro_entry(uint32_t ux, uint32_t uy, uint32_t uz, F3 ro, F3 rd, float t, uint32_t axis,
                                            bool px_, bool py_, bool pz_, bool snap, uint32_t* m) {
  F3 p = ((ro + rd * t) - f3((float)ux, (float)uy, (float)uz)) * 4.0f;
  int32_t a = min(max(ffloor_i(p.x), 0), 3), b = min(max(ffloor_i(p.y), 0), 3), c = min(max(ffloor_i(p.z), 0), 3);
  if (snap) {
    if (axis == 0) a = px_ ? 0 : 3;
    else if (axis == 1) b = py_ ? 0 : 3;
    else c = pz_ ? 0 : 3;
  }
  m[0] = a; m[1] = b; m[2] = c;
}

// cutout_march: common.wgsl:537-577
static __device__ __forceinline__ bool cutout_march(int32_t wx, int32_t wy, int32_t wz, uint32_t ux, uint32_t uy, uint32_t uz,
                                          F3 ro, F3 rd, F3 inv, float t_in, uint32_t axis_in, bool pdx, bool pdy,
                                          bool pdz, bool snap, float fill, float* t_out, uint32_t* n_out,
                                          uint32_t* m_out) {
  // inv is the ray's 1 / rd, the value the WGSL recomputes here
  const float ms = 1.0f / 4.0f;
  uint32_t me[3];
  micro_entry(ux, uy, uz, ro, rd, t_in, axis_in, pdx, pdy, pdz, snap, me);
  int32_t m0 = me[0], m1 = me[1], m2 = me[2];
  float t = t_in;
  uint32_t axis = axis_in;
  for (uint32_t i = 0; i < 12u; ++i) {
    if (m0 < 0 || m1 < 0 || m2 < 0 || m0 >= 4 || m1 >= 4 || m2 >= 4) return false;
    if (leaf_solid(wx, wy, wz, m0, m1, m2, fill)) {
      *t_out = t;
      bool pd = axis == 0 ? pdx : (axis == 1 ? pdy : pdz);
      *n_out = axis * 2u + (pd ? 0u : 1u);
      m_out[0] = m0; m_out[1] = m1; m_out[2] = m2;
      return true;
    }
    F3 bound = {(float)(pdx ? m0 + 1 : m0), (float)(pdy ? m1 + 1 : m1), (float)(pdz ? m2 + 1 : m2)};
    F3 tn = ((f3((float)ux, (float)uy, (float)uz) + bound * ms) - ro) * inv;
    if (tn.x <= tn.y && tn.x <= tn.z) { t = tn.x; axis = 0u; m0 += pdx ? 1 : -1; }
    else if (tn.y <= tn.z) { t = tn.y; axis = 1u; m1 += pdy ? 1 : -1; }
    else { t = tn.z; axis = 2u; m2 += pdz ? 1 : -1; }
  }
  return false;
}

__device__ __forceinline__ F3 refract(F3 e1, F3 e2, float e3);

// Ray state shared by a sequence of march_chunk calls on one ray.  A zero
// direction component (a sun exactly on the horizon) gives an infinite
// reciprocal, as the WGSL's 1.0 / rd does; every later step is IEEE
// arithmetic, which the oracle repeats operation for operation.
struct Ray {
  F3 o, d, inv;
  bool pdx, pdy, pdz;
};
__device__ __forceinline__ Ray make_ray(F3 o, F3 d) {
  Ray r;
  r.o = o; r.d = d;
  r.inv = {1.0f / d.x, 1.0f / d.y, 1.0f / d.z};
  r.pdx = d.x > 0.0f; r.pdy = d.y > 0.0f; r.pdz = d.z > 0.0f;
  return r;
}

// The atlas alpha at (u, v) of a layer at an explicit level, through the
// engine's atlas sampler (mag nearest, min / mipmap linear, clamp to edge):
// level <= 0 magnifies (nearest texel of mip 0), otherwise the two mips
// around it are sampled bilinearly and blended.
__device__ __forceinline__ float atlas_alpha_at(const DevWorld& w, uint32_t mip, uint32_t layer, int32_t x, int32_t y) {
  const uint32_t size = 16u >> mip;
  uint64_t base = 0;
  for (uint32_t m = 0; m < mip; ++m) base += (uint64_t)w.atlas_layers * (16u >> m) * (16u >> m);
  x = min(max(x, 0), (int32_t)size - 1);
  y = min(max(y, 0), (int32_t)size - 1);
  return __ldg(w.atlas_alpha + base + ((uint64_t)layer * size + (uint32_t)y) * size + (uint32_t)x);
}
__device__ __forceinline__ float atlas_alpha_bilinear(const DevWorld& w, uint32_t mip, uint32_t layer, float u, float v) {
  const float size = (float)(16u >> mip);
  const float x = u * size - 0.5f, y = v * size - 0.5f;
  const float x0 = floorf(x), y0 = floorf(y);
  const float ax = x - x0, ay = y - y0;
  const int32_t ix = ffloor_i(x0), iy = ffloor_i(y0);
  const int32_t ix1 = (int32_t)((uint32_t)ix + 1u), iy1 = (int32_t)((uint32_t)iy + 1u);
  const float a0 = atlas_alpha_at(w, mip, layer, ix, iy) * (1.0f - ax) + atlas_alpha_at(w, mip, layer, ix1, iy) * ax;
  const float a1 = atlas_alpha_at(w, mip, layer, ix, iy1) * (1.0f - ax) + atlas_alpha_at(w, mip, layer, ix1, iy1) * ax;
  return a0 * (1.0f - ay) + a1 * ay;
}
__device__ __forceinline__ float atlas_alpha(const DevWorld& w, uint32_t layer, float u, float v, float lod) {
  layer = min(layer, w.atlas_layers - 1u);
  if (!(lod > 0.0f)) return atlas_alpha_at(w, 0, layer, ffloor_i(u * 16.0f), ffloor_i(v * 16.0f));
  const float d = fminf(lod, 3.0f);
  const float dl = floorf(d);
  const float delta = d - dl;
  const uint32_t m0 = __float2uint_rz(dl);
  const float a = atlas_alpha_bilinear(w, m0, layer, u, v);
  if (!(delta > 0.0f) || m0 + 1u >= 4u) return a;
  return a * (1.0f - delta) + atlas_alpha_bilinear(w, m0 + 1u, layer, u, v) * delta;
}

// hash_alpha: common.wgsl:400-406
__device__ __forceinline__ float hash_alpha3(float x, float y, float z) {
  const int32_t qx = ffloor_i(x * 64.0f), qy = ffloor_i(y * 64.0f), qz = ffloor_i(z * 64.0f);
  uint32_t h = ((uint32_t)qx * 73856093u) ^ ((uint32_t)qy * 19349663u) ^ ((uint32_t)qz * 83492791u);
  h = h ^ (h >> 13u);
  h = h * 1274126177u;
  return (float)((h >> 8u) & 0xFFFFFFu) / 16777216.0f;
}

// wind_shear: common.wgsl:419-423 (SPEC_WIND_SWAY)
__device__ __forceinline__ void wind_shear(float wx, float wz, float time, float* sx, float* sz) {
  const float g = 0.65f * sinf(time * 1.9f + wx * 0.11f + wz * 0.07f) +
                  0.35f * sinf(time * 3.1f + wx * 0.173f + wz * 0.129f + 1.7f);
  *sx = g * 0.8f * 0.09f;
  *sz = g * 0.6f * 0.09f;
}

// cross_quad: common.wgsl:425-487.  The two diagonal quads of a tuft voxel
// (x - z = const: NORMAL_CROSS_A, x + z = const: NORMAL_CROSS_B), nearest
// first; a quad hit counts where the atlas alpha at its texel exceeds the
// voxel's hash threshold.  ro, rd and t are chunk-local (voxel units).
// Out of line: only tuft voxels reach it, and inlined it cost the march
// kernels registers (more spills) on every path.
static __device__ __noinline__ bool cross_quad(const DevWorld& w, const vm_frame& f, uint32_t ux, uint32_t uy, uint32_t uz,
                                           F3 ro, F3 rd, uint32_t layer, float vs, float shx, float shz, bool sway,
                                           float* qt, uint32_t* qn) {
  const float bx = (float)ux, by = (float)uy, bz = (float)uz;
  float tsx = -1.0f, tsy = -1.0f;
  if (sway) {
    const float dy = ro.y - by;
    const float ka = shx - shz, kb = shx + shz;
    const float da = rd.x - rd.z - ka * rd.y;
    if (fabsf(da) > 1e-6f) tsx = ((bx - bz) + ka * dy - (ro.x - ro.z)) / da;
    const float db = rd.x + rd.z - kb * rd.y;
    if (fabsf(db) > 1e-6f) tsy = ((bx + bz + 1.0f) + kb * dy - (ro.x + ro.z)) / db;
  } else {
    const float da = rd.x - rd.z;
    if (fabsf(da) > 1e-6f) tsx = ((bx - bz) - (ro.x - ro.z)) / da;
    const float db = rd.x + rd.z;
    if (fabsf(db) > 1e-6f) tsy = ((bx + bz + 1.0f) - (ro.x + ro.z)) / db;
  }
  uint32_t o0 = VM_NORMAL_CROSS_A, o1 = VM_NORMAL_CROSS_B;
  if (tsy < tsx) {
    const float tt = tsx; tsx = tsy; tsy = tt;
    o0 = VM_NORMAL_CROSS_B; o1 = VM_NORMAL_CROSS_A;
  }
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    const float tq = i == 0 ? tsx : tsy;
    if (tq < 0.0f) continue;
    const F3 p = ro + rd * tq;
    const F3 local = {p.x - bx, p.y - by, p.z - bz};
    if (local.x < -1e-4f || local.y < -1e-4f || local.z < -1e-4f || local.x > 1.0f + 1e-4f ||
        local.y > 1.0f + 1e-4f || local.z > 1.0f + 1e-4f)
      continue;
    const float footprint = fmaxf(tq * vs, 1e-3f) * 2.0f * f.tan_half_fov / (float)f.res[1] * 16.0f / vs;
    const float lod = fminf(fmaxf(log2f(fmaxf(footprint, 1e-4f)) + f.mip_bias, 0.0f), 3.0f);
    const float a = atlas_alpha(w, layer, local.x, 1.0f - local.y, lod);
    if (a <= hash_alpha3(p.x, p.y, p.z)) continue;
    *qt = tq;
    *qn = i == 0 ? o0 : o1;
    return true;
  }
  return false;
}

// march_chunk: common.wgsl:579-910.
//   SKIP_WATER / SKIP_GLASS / SUN_RAY are the WGSL arguments of the same name;
//   skip_foliage, which gates the tuft cross-quad trace, equals sun_ray at
//   every call site of the engine (march.wgsl:21,32; common.wgsl:1125,1172,1237).
//   COUNT enables the per-ray traffic counters used by the roofline.
struct Traffic { uint32_t chunk, l1, leaf, attr, pal, grid, iters, entries; };

//   WANT_ID also returns the hit voxel's block id (block_at, common.wgsl:350),
//   decoded from the L1 node and leaf slot the march already holds.
//   TUFTS compiles the tuft cross-quad trace in (the host selects such
//   kernels only for frames whose chunks hold tufts and whose context has the
//   atlas): the code costs the march registers on every path.
template <bool SKIP_WATER, bool SKIP_GLASS, bool SUN_RAY, bool COUNT, bool WANT_ID = false, bool TUFTS = false>
__device__ __forceinline__ Hit march_chunk(const DevWorld& w, const vm_frame& f, const Chunk& c, const Ray& r,
                                           float t_limit, Traffic* tr) {
  Hit h;
  h.hit = false; h.t = 0.0f; h.normal = 0u; h.vx = h.vy = h.vz = 0u; h.mx = h.my = h.mz = 0u; h.iters = 0u;
  h.id = 0u;
  if (COUNT) tr->chunk++;
  const float vs = c.vs;
  const Scale sv = make_scale(vs);
  const F3 origin = ld3(c.origin);
  const F3 ro = {sdiv(r.o.x - origin.x, sv), sdiv(r.o.y - origin.y, sv), sdiv(r.o.z - origin.z, sv)};
  const F3 rd = r.d;
  const F3 inv = r.inv;
  const F3 bmin = {sdiv(c.aabb_min[0] - origin.x, sv), sdiv(c.aabb_min[1] - origin.y, sv),
                   sdiv(c.aabb_min[2] - origin.z, sv)};
  const F3 bmax = {sdiv(c.aabb_max[0] - origin.x, sv), sdiv(c.aabb_max[1] - origin.y, sv),
                   sdiv(c.aabb_max[2] - origin.z, sv)};
  const F3 t0 = (bmin - ro) * inv;
  const F3 t1 = (bmax - ro) * inv;
  const F3 tmin3 = {fminf(t0.x, t1.x), fminf(t0.y, t1.y), fminf(t0.z, t1.z)};
  const F3 tmax3 = {fmaxf(t0.x, t1.x), fmaxf(t0.y, t1.y), fmaxf(t0.z, t1.z)};
  const float t_enter = fmaxf(fmaxf(tmin3.x, tmin3.y), tmin3.z);
  const float t_exit = fminf(fminf(tmax3.x, tmax3.y), tmax3.z);
  const float t_end = fminf(t_exit, sdiv(t_limit, sv));
  float t = fmaxf(t_enter, 0.0f);
  if (t >= t_end) return h;
  uint32_t axis;
  if (tmin3.x >= tmin3.y && tmin3.x >= tmin3.z) axis = 0u;
  else if (tmin3.y >= tmin3.z) axis = 1u;
  else axis = 2u;
  const bool pdx = r.pdx, pdy = r.pdy, pdz = r.pdz;
  F3 pos = ro + rd * t;
  int32_t cx = ffloor_i(pos.x), cy = ffloor_i(pos.y), cz = ffloor_i(pos.z);
  if (t_enter > 0.0f) {
    if (axis == 0) cx = pdx ? ffloor_i(bmin.x) : fceil_i(bmax.x) - 1;
    else if (axis == 1) cy = pdy ? ffloor_i(bmin.y) : fceil_i(bmax.y) - 1;
    else cz = pdz ? ffloor_i(bmin.z) : fceil_i(bmax.z) - 1;
  }
  cx = min(max(cx, 0), 63); cy = min(max(cy, 0), 63); cz = min(max(cz, 0), 63);
  const uint32_t root_lo = c.root[0], root_hi = c.root[1];
  const uint32_t root_ptr = c.root[2] & VM_PTR_MASK;
  const bool attr_uniform = (c.attr_flags & VM_ATTR_UNIFORM) != 0u;

  bool water_aware = SKIP_WATER && (c.attr_flags & VM_ATTR_HAS_WATER) != 0u;
  if (water_aware && attr_uniform) {
    if (c.attr_base == VM_WATER) return h;
    water_aware = false;
  }
  const uint32_t spec = w.spec;
  bool foliage_aware = (spec & VM_SPEC_FOLIAGE) != 0u && (c.attr_flags & VM_ATTR_HAS_FOLIAGE) != 0u;
  if (foliage_aware && attr_uniform && !is_tuft(c.attr_base)) foliage_aware = false;
  bool cutout_aware = (spec & VM_SPEC_LEAF_CUTOUT) != 0u && (c.attr_flags & VM_ATTR_HAS_CUTOUT) != 0u && vs == 1.0f;
  if (cutout_aware && attr_uniform && c.attr_base != VM_LEAVES && c.attr_base != VM_PINE_LEAVES) cutout_aware = false;
  bool glass_aware = SKIP_GLASS && (spec & VM_SPEC_GLASS) != 0u && (c.attr_flags & VM_ATTR_HAS_GLASS) != 0u;
  if (glass_aware && attr_uniform) {
    if (c.attr_base == VM_GLASS) return h;
    glass_aware = false;
  }
  const bool noncaster_aware = SUN_RAY && (spec & VM_SPEC_EMITTER_GATHER) != 0u &&
                               (c.attr_flags & VM_ATTR_HAS_EMITTER) != 0u;
  if (noncaster_aware && attr_uniform && c.attr_base == VM_GLOWSTONE) return h;
  const bool water_interface = !SKIP_WATER && (spec & VM_SPEC_WATER_REPAIR) != 0u &&
                               (c.attr_flags & VM_ATTR_HAS_WATER) != 0u;
  const bool attr_needed = (noncaster_aware && !attr_uniform) || (water_interface && !attr_uniform) || water_aware ||
                           glass_aware || ((foliage_aware || cutout_aware) && !attr_uniform);
  const bool any_filter = noncaster_aware || water_interface || water_aware || glass_aware || foliage_aware || cutout_aware;

  uint32_t trav_lo = root_lo, trav_hi = root_hi;
  if (water_aware) { trav_lo = c.dry[0]; trav_hi = c.dry[1]; }
  const bool root_full = (c.root[2] & VM_FULL_BIT) != 0u;
  if (root_full && (spec & VM_SPEC_FULL_MARCH) == 0u && !noncaster_aware && !water_interface) {
    // the full-root shortcut (common.wgsl:677-686): the entry cell is the hit
    h.hit = true;
    h.t = t * vs;
    const bool pd = axis == 0 ? pdx : (axis == 1 ? pdy : pdz);
    h.normal = axis * 2u + (pd ? 0u : 1u);
    h.vx = cx; h.vy = cy; h.vz = cz;
    uint32_t m[3];
    micro_entry(cx, cy, cz, ro, rd, t, axis, pdx, pdy, pdz, t > 0.0f, m);
    h.mx = m[0]; h.my = m[1]; h.mz = m[2];
    if (WANT_ID) h.id = attr_uniform ? c.attr_base : block_at(w, c, cx, cy, cz);
    return h;
  }
  if (trav_lo == 0u && trav_hi == 0u) return h;

  uint32_t l1_cached = 0xFFFFFFFFu;
  uint4 l1 = make_uint4(0u, 0u, 0u, 0u);
  uint32_t leaf_cached = 0xFFFFFFFFu;
  uint2 leaf = make_uint2(0u, 0u);
  uint32_t attr = 0u;
  // The leaf's attribute word is read the first time a solid voxel of the
  // leaf needs its block id, not when the leaf is entered: most leaves a ray
  // crosses yield no hit, and the read was a dependent load on every new
  // leaf's critical path.  A pure read, so the results are unchanged.
  uint32_t attr_slot = 0xFFFFFFFFu;   // attribute index of the leaf in hand
  bool attr_have = false;
  // A cell a march has already left without a hit, reached again: the step
  // out of a cell that yields no hit depends on the cell alone (its masks
  // decide the skip, its box the next t and axis; the water-repair and
  // cutout tests either hit or skip 1), so the walk is then a cycle through
  // the same cells with the same entry t and axis, no hit and no exit, until
  // the 512-step cap ends it with no hit.  Marches that run past 64 steps
  // (float rounding sends grazing rays back into a cell they left) keep a
  // cell at steps 64, 128, 256 and stop with the cap's result when they come
  // back to it: h.iters = MAX_ITERS + 1, hit false, as the cap gives.
  int32_t kx = -1, ky = -1, kz = -1;
  for (;;) {
    h.iters += 1u;
    if (COUNT) tr->iters++;
    if (h.iters > VM_MAX_ITERS) break;
    if ((uint32_t)cx > 63u || (uint32_t)cy > 63u || (uint32_t)cz > 63u) break;
    const uint32_t ux = cx, uy = cy, uz = cz;
    int32_t skip = 16;
    bool solid = false;
    const uint32_t l1b = cell_bit(ux >> 4, uy >> 4, uz >> 4);
    if (mask_has(trav_lo, trav_hi, l1b)) {
      if (l1b != l1_cached) {
        l1_cached = l1b;
        if (root_full) {
          l1 = make_uint4(0xFFFFFFFFu, 0xFFFFFFFFu, VM_FULL_BIT, (l1b * 64u) | 0xF0000000u);
        } else {
          if (COUNT) tr->l1++;
          l1 = ld_inner(w, (uint64_t)root_ptr + mask_below(root_lo, root_hi, l1b));
        }
        leaf_cached = 0xFFFFFFFFu;
      }
      bool line_skip = false;
      if (water_aware) {
        const uint32_t wl = l1.w >> 28u;
        const float ly = (float)(uy & 15u);
        if (wl < 15u && ly > (float)wl) {
          line_skip = rd.y >= 0.0f;
          if (!line_skip) {
            const float hh = fmaxf(fabsf(rd.x), fabsf(rd.z));
            if (hh > 1e-6f && (ly - (float)wl) > 16.0f * (fabsf(rd.y) / hh)) line_skip = true;
          }
        }
      }
      const uint32_t lfb = cell_bit((ux >> 2) & 3u, (uy >> 2) & 3u, (uz >> 2) & 3u);
      if (line_skip) {
        skip = 16;
      } else if ((l1.z & VM_FULL_BIT) != 0u) {
        solid = true;
        if (attr_needed && lfb != leaf_cached) {
          leaf_cached = lfb;
          attr_slot = (l1.w & 0x0FFFFFFFu) + lfb;
          attr_have = false;
        }
      } else if (mask_has(l1.x, l1.y, lfb)) {
        if (lfb != leaf_cached) {
          leaf_cached = lfb;
          const uint32_t li = mask_below(l1.x, l1.y, lfb);
          if (COUNT) tr->leaf++;
          leaf = ld_leaf(w, (uint64_t)(l1.z & VM_PTR_MASK) + li);
          attr_slot = (l1.w & 0x0FFFFFFFu) + li;
          attr_have = false;
        }
        const uint32_t vb = cell_bit(ux & 3u, uy & 3u, uz & 3u);
        if (mask_has(leaf.x, leaf.y, vb)) solid = true;
        else skip = block2_empty(leaf.x, leaf.y, vb & 42u) ? 2 : 1;
      } else {
        skip = 4;
      }
    } else {
      skip = block2_empty(trav_lo, trav_hi, l1b & 42u) ? 32 : 16;
    }
    // block id of a solid voxel: the chunk's id when uniform, else decoded once
    uint32_t id = c.attr_base;
    bool id_known = attr_uniform;
    if (solid && any_filter) {
      const bool need_id = !attr_uniform && (noncaster_aware || water_interface || water_aware || glass_aware ||
                                             foliage_aware || cutout_aware);
      if (attr_needed && !attr_have) {
        if (COUNT) tr->attr++;
        attr = ld_brick(w, (uint64_t)c.attr_base + attr_slot);
        attr_have = true;
      }
      if (need_id) {
        if (COUNT && (attr & VM_UNIFORM_BIT) == 0u) tr->pal++;
        id = leaf_block(w, attr, ux, uy, uz);
        id_known = true;
      }
      if (noncaster_aware && id == VM_GLOWSTONE) { solid = false; skip = 1; }
      if (solid && water_interface && id == VM_WATER) {
        const uint32_t nid = axis * 2u + ((axis == 0 ? pdx : (axis == 1 ? pdy : pdz)) ? 0u : 1u);
        const F3 outward = normal_of(nid);
        const F3 boundary = r.o + rd * (t * vs);
        if (COUNT) tr->grid++;
        if (world_block_at(w, f, boundary + outward * (0.002f * vs)) == VM_WATER) { solid = false; skip = 1; }
      }
      if (solid && water_aware && id == VM_WATER) { solid = false; skip = (attr & VM_UNIFORM_BIT) != 0u ? 4 : 1; }
      if (solid && glass_aware && id == VM_GLASS) { solid = false; skip = (attr & VM_UNIFORM_BIT) != 0u ? 4 : 1; }
      if (solid && foliage_aware && is_tuft(id)) {
        solid = false;
        skip = 1;
        if (TUFTS && !SUN_RAY && w.atlas_alpha != nullptr) {
          float shx = 0.0f, shz = 0.0f;
          const bool sway = (spec & VM_SPEC_WIND_SWAY) != 0u;
          if (sway)
            wind_shear(c.origin[0] + (float)ux * vs, c.origin[2] + (float)uz * vs, f.time * f.cloud_speed, &shx, &shz);
          const uint32_t layer = w.tuft_layer[id == VM_TALL_GRASS ? 0 : (id == VM_GRASS_TALL ? 1 : 2)];
          float qt; uint32_t qn;
          if (cross_quad(w, f, ux, uy, uz, ro, rd, layer, vs, shx, shz, sway, &qt, &qn)) {
            h.hit = true; h.t = qt * vs; h.normal = qn;
            h.vx = ux; h.vy = uy; h.vz = uz;
            h.mx = h.my = h.mz = 0u;
            h.id = id;
            return h;
          }
        }
      }
      if (solid && cutout_aware && is_cutout_id(id)) {
        const int32_t wx = __float2int_rz(c.origin[0]) + (int32_t)ux;
        const int32_t wy = __float2int_rz(c.origin[1]) + (int32_t)uy;
        const int32_t wz = __float2int_rz(c.origin[2]) + (int32_t)uz;
        float qt; uint32_t qn; uint32_t qm[3];
        if (cutout_march(wx, wy, wz, ux, uy, uz, ro, rd, inv, t, axis, pdx, pdy, pdz, t > 0.0f, leaf_fill(spec), &qt,
                         &qn, qm)) {
          h.hit = true; h.t = qt * vs; h.normal = qn;
          h.vx = ux; h.vy = uy; h.vz = uz;
          h.mx = qm[0]; h.my = qm[1]; h.mz = qm[2];
          h.id = id;
          return h;
        }
        solid = false;
        skip = 1;
      }
    }
    if (solid) {
      h.hit = true;
      h.t = t * vs;
      const bool pd = axis == 0 ? pdx : (axis == 1 ? pdy : pdz);
      h.normal = axis * 2u + (pd ? 0u : 1u);
      h.vx = ux; h.vy = uy; h.vz = uz;
      uint32_t m[3];
      micro_entry(ux, uy, uz, ro, rd, t, axis, pdx, pdy, pdz, t > 0.0f, m);
      h.mx = m[0]; h.my = m[1]; h.mz = m[2];
      if (WANT_ID) {
        if (!id_known) {
          // leaf_attr (common.wgsl:336-348) from the L1 node in hand
          const uint32_t lfb = cell_bit((ux >> 2) & 3u, (uy >> 2) & 3u, (uz >> 2) & 3u);
          const uint32_t slot = (l1.z & VM_FULL_BIT) != 0u ? lfb : mask_below(l1.x, l1.y, lfb);
          const uint32_t e = attr_needed ? attr : ld_brick(w, (uint64_t)c.attr_base + (l1.w & 0x0FFFFFFFu) + slot);
          id = leaf_block(w, e, ux, uy, uz);
        }
        h.id = id;
      }
      return h;
    }
    if (h.iters >= 64u) {
      if (cx == kx && cy == ky && cz == kz) { h.iters = VM_MAX_ITERS + 1u; break; }
      if ((h.iters & (h.iters - 1u)) == 0u) { kx = cx; ky = cy; kz = cz; }
    }
    const int32_t bx0 = cx - (cx & (skip - 1)), by0 = cy - (cy & (skip - 1)), bz0 = cz - (cz & (skip - 1));
    const float bndx = (float)(pdx ? bx0 + skip : bx0);
    const float bndy = (float)(pdy ? by0 + skip : by0);
    const float bndz = (float)(pdz ? bz0 + skip : bz0);
    const float tnx = (bndx - ro.x) * inv.x, tny = (bndy - ro.y) * inv.y, tnz = (bndz - ro.z) * inv.z;
    if (tnx <= tny && tnx <= tnz) { t = tnx; axis = 0u; }
    else if (tny <= tnz) { t = tny; axis = 1u; }
    else { t = tnz; axis = 2u; }
    if (t >= t_end) break;
    pos = ro + rd * t;
    cx = ffloor_i(pos.x); cy = ffloor_i(pos.y); cz = ffloor_i(pos.z);
    if (axis == 0) cx = pdx ? bx0 + skip : bx0 - 1;
    else if (axis == 1) cy = pdy ? by0 + skip : by0 - 1;
    else cz = pdz ? bz0 + skip : bz0 - 1;
  }
  return h;
}

// SPEC_SNELL_BEND (march.wgsl:23-44): from an underwater camera, a primary
// ray that rises and misses chunk c straight is bent at the flat sea level
// (refract(rd, -y, WATER_IOR)) and marched again from the surface; a hit
// there replaces the miss, with t the whole path (surface distance + bent
// leg) and the iterations of both marches.
template <bool COUNT, bool WANT_ID, bool TUFTS = false>
__device__ __forceinline__ void snell_bend(const DevWorld& w, const vm_frame& f, const Chunk& c, F3 rd, Hit* h,
                                           Traffic* tr) {
  if (!(rd.y > 0.0f)) return;
  const float depth = f.sea_level - f.cam_pos[1];
  if (!(depth > 0.0f)) return;
  const float t_surf = depth / rd.y;
  if (!(t_surf < f.far_)) return;
  const F3 surf = ld3(f.cam_pos) + rd * t_surf;
  const F3 rd2 = refract(rd, f3(0.0f, -1.0f, 0.0f), VM_WATER_IOR);
  if (!(dot(rd2, rd2) > 0.0f)) return;
  const Hit h2 = march_chunk<true, false, false, COUNT, WANT_ID, TUFTS>(w, f, c, make_ray(surf + rd2 * VM_SURFACE_EPS, rd2),
                                                                  f.far_ - t_surf, tr);
  if (h2.hit) {
    const uint32_t straight_iters = h->iters;
    *h = h2;
    h->t = t_surf + h2.t;
    h->iters = straight_iters + h2.iters;
  }
}

// shadow_ray_t: common.wgsl:1156-1195
template <bool COUNT>
__device__ __noinline__ float shadow_ray_t(const DevWorld& w, const vm_frame& f, F3 ro, F3 rd, float max_dist, Traffic* tr) {
  const Ray r = make_ray(ro, rd);
  int32_t cx = ffloor_i(ro.x * INV64), cy = ffloor_i(ro.y * INV64), cz = ffloor_i(ro.z * INV64);
  uint32_t last = VM_NO_CHUNK;
  for (uint32_t i = 0; i < 24u; ++i) {
    uint64_t gi;
    if (!grid_rel(f, cx, cy, cz, &gi)) return -1.0f;
    if (COUNT) tr->grid++;
    const uint32_t ci = ld_grid(w, gi);
    if (ci != VM_NO_CHUNK && ci != last) {
      last = ci;
      const Chunk c = ld_chunk(w, ci);
      const Hit m = march_chunk<true, true, true, COUNT>(w, f, c, r, max_dist, tr);
      if (m.hit) return m.t;
    }
    const float bx = (float)(r.pdx ? cx + 1 : cx) * 64.0f;
    const float by = (float)(r.pdy ? cy + 1 : cy) * 64.0f;
    const float bz = (float)(r.pdz ? cz + 1 : cz) * 64.0f;
    const float tnx = (bx - ro.x) * r.inv.x, tny = (by - ro.y) * r.inv.y, tnz = (bz - ro.z) * r.inv.z;
    float t;
    uint32_t axis = 0u;
    if (tnx <= tny && tnx <= tnz) t = tnx;
    else if (tny <= tnz) { t = tny; axis = 1u; }
    else { t = tnz; axis = 2u; }
    if (t >= max_dist) return -1.0f;
    if (axis == 0) cx += r.pdx ? 1 : -1;
    else if (axis == 1) cy += r.pdy ? 1 : -1;
    else cz += r.pdz ? 1 : -1;
  }
  return -1.0f;
}

// shadow_ray: common.wgsl:1098-1148, the boolean sun test of shade_hit for
// secondary hits: from below the sea level a rising ray (SPEC_WATER_REPAIR)
// starts at the flat sea surface, the rest is shadow_ray_t's walk.
static __device__ __noinline__ bool shadow_ray_hit(const DevWorld& w, const vm_frame& f, F3 ro, F3 rd, float max_dist) {
  F3 r_ro = ro;
  float r_dist = max_dist;
  if ((w.spec & VM_SPEC_WATER_REPAIR) != 0u && rd.y > 1e-4f && ro.y < f.sea_level) {
    const float t_surf = (f.sea_level - ro.y) / rd.y;
    if (t_surf >= r_dist) return false;
    r_ro = ro + rd * t_surf;
    r_dist = r_dist - t_surf;
  }
  const Ray r = make_ray(r_ro, rd);
  int32_t cx = ffloor_i(r_ro.x * INV64), cy = ffloor_i(r_ro.y * INV64), cz = ffloor_i(r_ro.z * INV64);
  uint32_t last = VM_NO_CHUNK;
  for (uint32_t i = 0; i < 24u; ++i) {
    uint64_t gi;
    if (!grid_rel(f, cx, cy, cz, &gi)) return false;
    const uint32_t ci = ld_grid(w, gi);
    if (ci != VM_NO_CHUNK && ci != last) {
      last = ci;
      const Chunk c = ld_chunk(w, ci);
      if (march_chunk<true, true, true, false>(w, f, c, r, r_dist, nullptr).hit) return true;
    }
    const float bx = (float)(r.pdx ? cx + 1 : cx) * 64.0f;
    const float by = (float)(r.pdy ? cy + 1 : cy) * 64.0f;
    const float bz = (float)(r.pdz ? cz + 1 : cz) * 64.0f;
    const float tnx = (bx - r_ro.x) * r.inv.x, tny = (by - r_ro.y) * r.inv.y, tnz = (bz - r_ro.z) * r.inv.z;
    float t;
    uint32_t axis = 0u;
    if (tnx <= tny && tnx <= tnz) t = tnx;
    else if (tny <= tnz) { t = tny; axis = 1u; }
    else { t = tnz; axis = 2u; }
    if (t >= r_dist) return false;
    if (axis == 0) cx += r.pdx ? 1 : -1;
    else if (axis == 1) cy += r.pdy ? 1 : -1;
    else cz += r.pdz ? 1 : -1;
  }
  return false;
}

// shadow_ray_t one chunk-grid cell at a time, for kernels whose lanes take a
// new ray as soon as theirs ends: the state between cells is the cell, the
// last chunk marched and the step count, and each step is the loop body of
// shadow_ray_t above, so the result is the same float.  Returns true when the
// ray is over, with its blocker distance (-1: none) in *out.
struct ShadowWalk {
  Ray r;
  int32_t cx, cy, cz;
  uint32_t last, step;
};
__device__ __forceinline__ ShadowWalk shadow_walk_begin(F3 ro, F3 rd) {
  ShadowWalk s;
  s.r = make_ray(ro, rd);
  s.cx = ffloor_i(ro.x * INV64); s.cy = ffloor_i(ro.y * INV64); s.cz = ffloor_i(ro.z * INV64);
  s.last = VM_NO_CHUNK;
  s.step = 0u;
  return s;
}
template <bool COUNT>
__device__ __forceinline__ bool shadow_walk_step(const DevWorld& w, const vm_frame& f, ShadowWalk& s, float max_dist,
                                                 float* out, Traffic* tr) {
  *out = -1.0f;
  // cells that march nothing (no chunk, the chunk just marched, or a march
  // that returns before its first DDA step) are crossed in the same call, so
  // that the lanes of a warp march together
  for (;;) {
    if (s.step >= 24u) return true;
    uint64_t gi;
    if (!grid_rel(f, s.cx, s.cy, s.cz, &gi)) return true;
    if (COUNT) tr->grid++;
    const uint32_t ci = ld_grid(w, gi);
    bool marched = false;   // a chunk march that took DDA steps
    if (ci != VM_NO_CHUNK && ci != s.last) {
      s.last = ci;
      const Chunk c = ld_chunk(w, ci);
      const Hit m = march_chunk<true, true, true, COUNT>(w, f, c, s.r, max_dist, tr);
      if (m.hit) { *out = m.t; return true; }
      marched = m.iters > 0u;
    }
    const Ray& r = s.r;
    const float bx = (float)(r.pdx ? s.cx + 1 : s.cx) * 64.0f;
    const float by = (float)(r.pdy ? s.cy + 1 : s.cy) * 64.0f;
    const float bz = (float)(r.pdz ? s.cz + 1 : s.cz) * 64.0f;
    const float tnx = (bx - r.o.x) * r.inv.x, tny = (by - r.o.y) * r.inv.y, tnz = (bz - r.o.z) * r.inv.z;
    float t;
    uint32_t axis = 0u;
    if (tnx <= tny && tnx <= tnz) t = tnx;
    else if (tny <= tnz) { t = tny; axis = 1u; }
    else { t = tnz; axis = 2u; }
    if (t >= max_dist) return true;
    if (axis == 0) s.cx += r.pdx ? 1 : -1;
    else if (axis == 1) s.cy += r.pdy ? 1 : -1;
    else s.cz += r.pdz ? 1 : -1;
    ++s.step;
    if (marched) return false;
  }
}

struct WorldHit { bool hit; float t; uint32_t normal; uint32_t vx, vy, vz; uint32_t ci; };

// trace_world: common.wgsl:1205-1253
template <bool SKIP_WATER, bool COUNT, bool TUFTS = false>
__device__ __noinline__ WorldHit trace_world(const DevWorld& w, const vm_frame& f, F3 ro, F3 rd, float max_dist, Traffic* tr) {
  WorldHit out;
  out.hit = false; out.t = max_dist; out.normal = 0u; out.vx = out.vy = out.vz = 0u; out.ci = VM_NO_CHUNK;
  const F3 dir = {tiny_fix(rd.x), tiny_fix(rd.y), tiny_fix(rd.z)};
  const F3 inv = {1.0f / dir.x, 1.0f / dir.y, 1.0f / dir.z};
  const bool pdx = dir.x > 0.0f, pdy = dir.y > 0.0f, pdz = dir.z > 0.0f;
  const Ray r = make_ray(ro, rd);
  int32_t cx = ffloor_i(ro.x * INV64), cy = ffloor_i(ro.y * INV64), cz = ffloor_i(ro.z * INV64);
  for (uint32_t i = 0; i < 16u; ++i) {
    uint64_t gi;
    if (!grid_rel(f, cx, cy, cz, &gi)) return out;
    if (COUNT) tr->grid++;
    const uint32_t ci = ld_grid(w, gi);
    const float bx = (float)(pdx ? cx + 1 : cx) * 64.0f;
    const float by = (float)(pdy ? cy + 1 : cy) * 64.0f;
    const float bz = (float)(pdz ? cz + 1 : cz) * 64.0f;
    const float tnx = (bx - ro.x) * inv.x, tny = (by - ro.y) * inv.y, tnz = (bz - ro.z) * inv.z;
    float t_exit = tnx;
    uint32_t axis = 0u;
    if (tny < t_exit) { t_exit = tny; axis = 1u; }
    if (tnz < t_exit) { t_exit = tnz; axis = 2u; }
    if (ci != VM_NO_CHUNK) {
      const Chunk c = ld_chunk(w, ci);
      const Hit h = march_chunk<SKIP_WATER, true, false, COUNT, false, TUFTS>(w, f, c, r, fminf(t_exit, max_dist), tr);
      if (h.hit) {
        out.hit = true; out.t = h.t; out.normal = h.normal;
        out.vx = h.vx; out.vy = h.vy; out.vz = h.vz; out.ci = ci;
        return out;
      }
    }
    if (t_exit >= max_dist) return out;
    if (axis == 0) cx += pdx ? 1 : -1;
    else if (axis == 1) cy += pdy ? 1 : -1;
    else cz += pdz ? 1 : -1;
  }
  return out;
}

// trace_world one chunk-grid cell at a time, for kernels whose lanes take a
// new ray as soon as theirs ends: the loop body of trace_world above, so the
// hit and its t are the same.  Returns true when the ray is over, with the
// result in *out.
struct WorldWalk {
  Ray r;                 // the march's ray (make_ray of the unmodified direction)
  F3 inv;                // grid stepping: reciprocal of the tiny-fixed direction
  bool pdx, pdy, pdz;
  int32_t cx, cy, cz;
  uint32_t step;
};
__device__ __forceinline__ WorldWalk world_walk_begin(F3 ro, F3 rd) {
  WorldWalk s;
  const F3 dir = {tiny_fix(rd.x), tiny_fix(rd.y), tiny_fix(rd.z)};
  s.inv = {1.0f / dir.x, 1.0f / dir.y, 1.0f / dir.z};
  s.pdx = dir.x > 0.0f; s.pdy = dir.y > 0.0f; s.pdz = dir.z > 0.0f;
  s.r = make_ray(ro, rd);
  s.cx = ffloor_i(ro.x * INV64); s.cy = ffloor_i(ro.y * INV64); s.cz = ffloor_i(ro.z * INV64);
  s.step = 0u;
  return s;
}
template <bool SKIP_WATER, bool COUNT, bool TUFTS = false>
__device__ __forceinline__ bool world_walk_step(const DevWorld& w, const vm_frame& f, WorldWalk& s, float max_dist,
                                                WorldHit* out, Traffic* tr) {
  out->hit = false; out->t = max_dist; out->normal = 0u; out->vx = out->vy = out->vz = 0u; out->ci = VM_NO_CHUNK;
  // cells without a chunk, or whose march takes no DDA step, are crossed in
  // the same call (see shadow_walk_step)
  for (;;) {
    if (s.step >= 16u) return true;
    uint64_t gi;
    if (!grid_rel(f, s.cx, s.cy, s.cz, &gi)) return true;
    if (COUNT) tr->grid++;
    const uint32_t ci = ld_grid(w, gi);
    const float bx = (float)(s.pdx ? s.cx + 1 : s.cx) * 64.0f;
    const float by = (float)(s.pdy ? s.cy + 1 : s.cy) * 64.0f;
    const float bz = (float)(s.pdz ? s.cz + 1 : s.cz) * 64.0f;
    const F3 ro = s.r.o;
    const float tnx = (bx - ro.x) * s.inv.x, tny = (by - ro.y) * s.inv.y, tnz = (bz - ro.z) * s.inv.z;
    float t_exit = tnx;
    uint32_t axis = 0u;
    if (tny < t_exit) { t_exit = tny; axis = 1u; }
    if (tnz < t_exit) { t_exit = tnz; axis = 2u; }
    bool marched = false;   // a chunk march that took DDA steps
    if (ci != VM_NO_CHUNK) {
      const Chunk c = ld_chunk(w, ci);
      const Hit h = march_chunk<SKIP_WATER, true, false, COUNT, false, TUFTS>(w, f, c, s.r, fminf(t_exit, max_dist), tr);
      if (h.hit) {
        out->hit = true; out->t = h.t; out->normal = h.normal;
        out->vx = h.vx; out->vy = h.vy; out->vz = h.vz; out->ci = ci;
        return true;
      }
      marched = h.iters > 0u;
    }
    if (t_exit >= max_dist) return true;
    if (axis == 0) s.cx += s.pdx ? 1 : -1;
    else if (axis == 1) s.cy += s.pdy ? 1 : -1;
    else s.cz += s.pdz ? 1 : -1;
    ++s.step;
    if (marched) return false;
  }
}

// hit_t: common.wgsl:1300-1318
__device__ __forceinline__ float hit_t(const vm_frame& f, const Chunk& c, uint32_t vx, uint32_t vy, uint32_t vz,
                                       uint32_t mx, uint32_t my, uint32_t mz, uint32_t nid, F3 rd) {
  const F3 box_min = ld3(c.origin) + f3((float)vx, (float)vy, (float)vz) * c.vs;
  if (nid >= VM_NORMAL_CROSS_A) {
    if (nid == VM_NORMAL_CROSS_A)
      return ((box_min.x - box_min.z) - (f.cam_pos[0] - f.cam_pos[2])) / (rd.x - rd.z);
    return ((box_min.x + box_min.z + c.vs) - (f.cam_pos[0] + f.cam_pos[2])) / (rd.x + rd.z);
  }
  const uint32_t axis = nid >> 1u;
  const float ms = c.vs * 0.25f;   // == c.vs / 4 exactly
  const uint32_t mi = axis == 0 ? mx : (axis == 1 ? my : mz);
  const float plane = comp(box_min, axis) + (float)(mi + ((nid & 1u) == 1u ? 1u : 0u)) * ms;
  return (plane - f.cam_pos[axis]) / comp(rd, axis);
}

// depth_key / make_key: common.wgsl:1320-1330
__device__ __forceinline__ uint32_t depth_key(const vm_frame& f, float t) {
  float x = 1.0f - t / f.far_;
  x = fminf(fmaxf(x, 0.0f), 1.0f);
  return __float2uint_rz(x * 16777215.0f);
}
__device__ __forceinline__ unsigned long long make_key(const vm_frame& f, const Hit& h, uint32_t ci) {
  const unsigned long long d = depth_key(f, h.t);
  const uint32_t bx = h.vx | (h.mx << 6), by = h.vy | (h.my << 6), bz = h.vz | (h.mz << 6);
  return (d << 40) | ((unsigned long long)h.normal << 37) | ((unsigned long long)ci << 24) |
         (unsigned long long)((bx << 16) | (by << 8) | bz);
}

// tile_select geometry: tile_select.wgsl:1-9
__device__ __forceinline__ bool box_outside(F3 bmin, F3 bmax, F3 n, F3 cam) {
  const F3 p = {n.x > 0.0f ? bmax.x : bmin.x, n.y > 0.0f ? bmax.y : bmin.y, n.z > 0.0f ? bmax.z : bmin.z};
  return dot(n, p - cam) < 0.0f;
}
__device__ __forceinline__ float box_distance(F3 p, F3 bmin, F3 bmax) {
  const F3 d = {fmaxf(fmaxf(bmin.x - p.x, p.x - bmax.x), 0.0f), fmaxf(fmaxf(bmin.y - p.y, p.y - bmax.y), 0.0f),
                fmaxf(fmaxf(bmin.z - p.z, p.z - bmax.z), 0.0f)};
  return sqrtf(dot(d, d));
}

struct TilePlanes { F3 n[4]; float reach; };

// The four corner rays (d00, d10, d11, d01) and the centre ray of the
// size x size pixel square whose top-left pixel is (x0i, y0i), in that order.
__device__ __forceinline__ void square_dirs(const vm_frame& f, uint32_t x0i, uint32_t y0i, float size, F3 d[5]) {
  const float x0 = (float)x0i, y0 = (float)y0i;
  const float x1 = x0 + size, y1 = y0 + size;
  d[0] = ray_dir(f, x0, y0); d[1] = ray_dir(f, x1, y0); d[2] = ray_dir(f, x1, y1); d[3] = ray_dir(f, x0, y1);
  d[4] = ray_dir(f, (x0 + x1) * 0.5f, (y0 + y1) * 0.5f);
}
// square_dirs for a whole warp (all 32 lanes, same square): lane k < 5 traces
// ray k and the others read it by shuffle, so the warp issues one ray_dir
// instead of five.  The floats are those of square_dirs.
__device__ __forceinline__ void square_dirs_warp(const vm_frame& f, uint32_t x0i, uint32_t y0i, float size,
                                                 uint32_t lane, F3 d[5]) {
  const float x0 = (float)x0i, y0 = (float)y0i;
  const float x1 = x0 + size, y1 = y0 + size;
  const uint32_t k = lane < 5u ? lane : 4u;
  const float px = k == 4u ? (x0 + x1) * 0.5f : ((k == 1u || k == 2u) ? x1 : x0);
  const float py = k == 4u ? (y0 + y1) * 0.5f : (k >= 2u ? y1 : y0);
  const F3 mine = ray_dir(f, px, py);
#pragma unroll
  for (int i = 0; i < 5; ++i)
    d[i] = {__shfl_sync(0xFFFFFFFFu, mine.x, i), __shfl_sync(0xFFFFFFFFu, mine.y, i),
            __shfl_sync(0xFFFFFFFFu, mine.z, i)};
}

// The side planes through consecutive corner rays, oriented towards the centre.
__device__ __forceinline__ void side_planes(const F3 d[5], F3 n[4]) {
  n[0] = cross(d[0], d[1]);
  n[1] = cross(d[1], d[2]);
  n[2] = cross(d[2], d[3]);
  n[3] = cross(d[3], d[0]);
#pragma unroll
  for (int i = 0; i < 4; ++i) if (!(dot(n[i], d[4]) >= 0.0f)) n[i] = neg(n[i]);
}

// tile_select.wgsl:17-57 for an 8x8 tile, from its square_dirs
__device__ __forceinline__ TilePlanes planes_of(const vm_frame& f, const F3 d[5]) {
  TilePlanes tp;
  side_planes(d, tp.n);
  float reach = f.far_;
  const uint32_t both = VM_FLAG_UNDERWATER | VM_FLAG_WATER_FAR;
  if ((f.flags & both) == both) {
    const float up = fmaxf(fmaxf(d[0].y, d[1].y), fmaxf(d[2].y, d[3].y));
    const float submerged = fmaxf(f.sea_level - f.cam_pos[1], 0.0f);
    float escape = 1e30f;
    if (up > 0.0f) escape = submerged / up;
    if (escape >= VM_WATER_FAR_DIST) {
      reach = fminf(f.far_, VM_WATER_FAR_DIST);
      const float dep_far = submerged - up * VM_WATER_FAR_DIST;
      if ((f.flags & VM_FLAG_WATER_DARK) != 0u && fminf(submerged, dep_far) >= VM_WATER_DARK_DEPTH)
        reach = fminf(reach, VM_WATER_DARK_DIST);
    }
  }
  tp.reach = reach;
  return tp;
}

// tile_select.wgsl:17-57 for the 8x8 tile whose top-left pixel is (x0i, y0i)
__device__ __forceinline__ TilePlanes tile_planes(const vm_frame& f, uint32_t x0i, uint32_t y0i) {
  F3 d[5];
  square_dirs(f, x0i, y0i, 8.0f, d);
  return planes_of(f, d);
}
// tile_planes for a whole warp (square_dirs_warp)
__device__ __forceinline__ TilePlanes tile_planes_warp(const vm_frame& f, uint32_t x0i, uint32_t y0i, uint32_t lane) {
  F3 d[5];
  square_dirs_warp(f, x0i, y0i, 8.0f, lane, d);
  return planes_of(f, d);
}

// refract per the WGSL builtin definition
__device__ __forceinline__ F3 refract(F3 e1, F3 e2, float e3) {
  const float d = dot(e2, e1);
  const float k = 1.0f - e3 * e3 * (1.0f - d * d);
  if (k < 0.0f) return f3(0.0f, 0.0f, 0.0f);
  return e1 * e3 - e2 * (e3 * d + sqrtf(k));
}
// reflect per the WGSL builtin definition: e1 - 2 dot(e2, e1) e2
__device__ __forceinline__ F3 reflect(F3 e1, F3 e2) {
  const float d = 2.0f * dot(e2, e1);
  return e1 - e2 * d;
}
__device__ __forceinline__ float smoothstep(float e0, float e1, float x) {
  const float t = fminf(fmaxf((x - e0) / (e1 - e0), 0.0f), 1.0f);
  return t * t * (3.0f - 2.0f * t);
}

}  // namespace vmd
