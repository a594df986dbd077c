// ORACLE — test infrastructure only.
//
// A plain CPU restatement of the reference engine's WGSL ray march, used as the
// checker for the CUDA path (tests, the smoke check and the timed CPU baseline
// leg of bench.py).  Nothing in the product links or calls this file.
//
// The reference (Vuk03-boop/voxelcraft-menu) has no CPU march: its headless
// modes run the same WGSL passes.  This file restates those passes line by line
// in C++ with a fixed floating-point contract:
//   * compiled with -ffp-contract=off (no FMA), IEEE division and sqrt;
//   * normalize(v) = v / sqrt(dot(v, v)), dot evaluated left to right;
//   * min/max follow IEEE minNum/maxNum (fminf/fmaxf);
//   * float -> int conversions saturate (as WGSL and PTX cvt do).
// The CUDA kernels are held to bit-exact agreement with this contract.
//
// Parity status: the reference's layout producers, key packing, pair word,
// water-line predicate and camera rays are pinned to the reference's own tests
// (tests/tree.rs, tests/full_march.rs, tests/emitter_gate.rs, tests/cutout.rs,
// tests/pairs.rs, tests/waterline.rs, tests/camera.rs, tests/physics.rs);
// the march outputs themselves are UNPINNED against the reference's GPU march,
// which cannot run here (WGSL needs a graphics stack) and which has no golden
// march outputs.  The hierarchical march is cross-checked against a restated
// unit-voxel DDA (src/player.rs:334-393) on opaque worlds.
//
// Citations are paths inside the reference project.

#include <cmath>
#include <cstdint>
#include <cstring>
#include <cstdio>
#include <vector>
#include <algorithm>
#include <atomic>
#include <omp.h>

#include "../voxelcraft_menu_b200/csrc/vm_types.h"

namespace {

// ----------------------------------------------------------------------------
// error flag: any out-of-bounds pool access sets it (the oracle never reads
// outside the buffers it was given).
std::atomic<int> g_err{0};
char g_err_msg[256];

void set_err(const char* what, uint64_t idx, uint64_t n) {
  int expect = 0;
  if (g_err.compare_exchange_strong(expect, 1)) {
    snprintf(g_err_msg, sizeof g_err_msg, "%s index %llu out of %llu", what,
             (unsigned long long)idx, (unsigned long long)n);
  }
}

struct V3 { float x, y, z; };
struct I3 { int32_t x, y, z; };
struct U3 { uint32_t x, y, z; };

inline V3 v3(float x, float y, float z) { return {x, y, z}; }
inline V3 add(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 sub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 mul(V3 a, V3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
inline V3 muls(V3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
inline V3 divs(V3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }
inline V3 neg(V3 a) { return {-a.x, -a.y, -a.z}; }
inline float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 cross(V3 a, V3 b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
inline V3 vmin(V3 a, V3 b) { return {fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z)}; }
inline V3 vmax(V3 a, V3 b) { return {fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z)}; }
inline float comp(V3 a, uint32_t i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }
inline int32_t comp(I3 a, uint32_t i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }
inline void setc(I3& a, uint32_t i, int32_t v) { if (i == 0) a.x = v; else if (i == 1) a.y = v; else a.z = v; }
inline bool compb(const bool* b, uint32_t i) { return b[i]; }
inline float signf(float x) { return x > 0.0f ? 1.0f : (x < 0.0f ? -1.0f : 0.0f); }
inline V3 normalize(V3 v) { float l = sqrtf(dot(v, v)); return {v.x / l, v.y / l, v.z / l}; }
inline float length(V3 v) { return sqrtf(dot(v, v)); }

// saturating float -> i32 (WGSL conversion semantics; NaN -> 0)
inline int32_t f2i(float x) {
  if (x != x) return 0;
  if (x >= 2147483648.0f) return INT32_MAX;
  if (x <= -2147483648.0f) return INT32_MIN;
  return (int32_t)x;
}
inline uint32_t f2u(float x) {
  if (x != x || x <= 0.0f) return 0;
  if (x >= 4294967296.0f) return UINT32_MAX;
  return (uint32_t)x;
}
inline I3 floor_i(V3 p) { return {f2i(floorf(p.x)), f2i(floorf(p.y)), f2i(floorf(p.z))}; }

inline V3 ld3(const float* p) { return {p[0], p[1], p[2]}; }

// ----------------------------------------------------------------------------
struct World {
  uint32_t spec = VM_SPEC_DEFAULT;   // pipeline specialisations (VM_SPEC_*)
  const vm_frame* f;
  const vm_chunk* chunks; uint32_t n_chunks;
  const uint32_t* inners; uint64_t n_inners;   // count of vec4<u32>
  const uint32_t* leaves; uint64_t n_leaves;   // count of vec2<u32>
  const uint32_t* bricks; uint64_t n_bricks;   // count of u32
  const uint32_t* grid; uint64_t n_grid;
  // the engine's atlas (Rgba8UnormSrgb, 16x16 layers, mips 16, 8, 4, 2) and
  // face table, for the tuft cross-quads; atlas null: tufts transparent
  const uint8_t* atlas = nullptr; uint32_t atlas_layers = 0;
  const uint32_t* faces = nullptr; uint32_t n_faces = 0;
};

// per-thread counters of the traversal's memory traffic (for the roofline)
struct Counters {
  uint64_t chunk_records, l1_fetches, leaf_fetches, attr_fetches, palette_decodes,
      grid_lookups, iters, march_calls, rays;
};
thread_local Counters* t_cnt = nullptr;
inline void cnt_add(uint64_t Counters::*f, uint64_t v = 1) { if (t_cnt) t_cnt->*f += v; }

struct U4 { uint32_t x, y, z, w; };
struct U2 { uint32_t x, y; };

inline U4 inner_at(const World& w, uint64_t i) {
  if (i >= w.n_inners) { set_err("inners", i, w.n_inners); return {0, 0, 0, 0}; }
  const uint32_t* p = w.inners + 4 * i;
  return {p[0], p[1], p[2], p[3]};
}
inline U2 leaf_at(const World& w, uint64_t i) {
  if (i >= w.n_leaves) { set_err("leaves", i, w.n_leaves); return {0, 0}; }
  return {w.leaves[2 * i], w.leaves[2 * i + 1]};
}
inline uint32_t brick_at(const World& w, uint64_t i) {
  if (i >= w.n_bricks) { set_err("bricks", i, w.n_bricks); return 0; }
  return w.bricks[i];
}
inline const vm_chunk& chunk_at(const World& w, uint32_t ci) {
  static const vm_chunk zero{};
  if (ci >= w.n_chunks) { set_err("chunks", ci, w.n_chunks); return zero; }
  return w.chunks[ci];
}
inline uint32_t grid_at(const World& w, uint64_t i) {
  if (i >= w.n_grid) { set_err("grid", i, w.n_grid); return VM_NO_CHUNK; }
  return w.grid[i];
}

// ---- tree helpers: common.wgsl:299-356 ----
inline bool mask_has(U2 m, uint32_t bit) {
  if (bit < 32u) return ((m.x >> bit) & 1u) != 0u;
  return ((m.y >> (bit - 32u)) & 1u) != 0u;
}
inline uint32_t popc(uint32_t x) { return (uint32_t)__builtin_popcount(x); }
inline uint32_t mask_below(U2 m, uint32_t bit) {
  if (bit < 32u) return popc(m.x & ((1u << bit) - 1u));
  if (bit == 32u) return popc(m.x);
  return popc(m.x) + popc(m.y & ((1u << (bit - 32u)) - 1u));
}
inline uint32_t cell_bit(U3 c) { return c.x | (c.y << 2u) | (c.z << 4u); }
inline U3 ushr(U3 a, uint32_t s) { return {a.x >> s, a.y >> s, a.z >> s}; }
inline U3 uand(U3 a, uint32_t m) { return {a.x & m, a.y & m, a.z & m}; }

// leaf_block: common.wgsl:320-334
uint32_t leaf_block(const World& w, uint32_t entry, U3 v) {
  if ((entry & VM_UNIFORM_BIT) != 0u) return entry & 0xFFFFu;
  cnt_add(&Counters::palette_decodes);
  uint32_t hdr = brick_at(w, entry);
  uint32_t n = hdr & 0xFFu;
  uint32_t bits = (hdr >> 8u) & 0xFFu;
  uint32_t pal_words = (n + 1u) / 2u;
  uint32_t vb = cell_bit(uand(v, 3u));
  uint32_t bitpos = vb * bits;
  uint32_t wd = brick_at(w, (uint64_t)entry + 1u + pal_words + (bitpos >> 5u));
  uint32_t idx = (wd >> (bitpos & 31u)) & ((bits >= 32u ? 0u : (1u << bits)) - 1u);
  uint32_t pw = brick_at(w, (uint64_t)entry + 1u + idx / 2u);
  return (pw >> ((idx & 1u) * 16u)) & 0xFFFFu;
}

// leaf_attr: common.wgsl:336-348
uint32_t leaf_attr(const World& w, uint32_t ci, U3 v) {
  const vm_chunk& c = chunk_at(w, ci);
  U2 root_mask{c.root[0], c.root[1]};
  uint32_t l1b = cell_bit(ushr(v, 4u));
  U4 l1;
  if ((c.root[2] & VM_FULL_BIT) != 0u) {
    l1 = {0xFFFFFFFFu, 0xFFFFFFFFu, VM_FULL_BIT, l1b * 64u};
  } else {
    l1 = inner_at(w, (uint64_t)(c.root[2] & VM_PTR_MASK) + mask_below(root_mask, l1b));
  }
  uint32_t lfb = cell_bit(uand(ushr(v, 2u), 3u));
  return brick_at(w, (uint64_t)c.attr_base + (l1.w & 0x0FFFFFFFu) + mask_below(U2{l1.x, l1.y}, lfb));
}

// block_at: common.wgsl:350-356
uint32_t block_at(const World& w, uint32_t ci, U3 v) {
  const vm_chunk& c = chunk_at(w, ci);
  if ((c.attr_flags & VM_ATTR_UNIFORM) != 0u) return c.attr_base;
  return leaf_block(w, leaf_attr(w, ci, v), v);
}

// voxel_occupied: common.wgsl:912-940
bool voxel_occupied(const World& w, uint32_t ci, I3 v) {
  if (v.x < 0 || v.y < 0 || v.z < 0 || v.x > 63 || v.y > 63 || v.z > 63) return false;
  const vm_chunk& c = chunk_at(w, ci);
  U3 uv{(uint32_t)v.x, (uint32_t)v.y, (uint32_t)v.z};
  U2 root_mask{c.root[0], c.root[1]};
  uint32_t l1b = cell_bit(ushr(uv, 4u));
  if (!mask_has(root_mask, l1b)) return false;
  bool occupied = false;
  if ((c.root[2] & VM_FULL_BIT) != 0u) {
    occupied = true;
  } else {
    U4 l1 = inner_at(w, (uint64_t)(c.root[2] & VM_PTR_MASK) + mask_below(root_mask, l1b));
    if ((l1.z & VM_FULL_BIT) != 0u) {
      occupied = true;
    } else {
      U2 l1m{l1.x, l1.y};
      uint32_t lfb = cell_bit(uand(ushr(uv, 2u), 3u));
      if (mask_has(l1m, lfb)) {
        U2 leaf = leaf_at(w, (uint64_t)(l1.z & VM_PTR_MASK) + mask_below(l1m, lfb));
        occupied = mask_has(leaf, cell_bit(uand(uv, 3u)));
      }
    }
  }
  return occupied;
}

inline uint64_t grid_index(const World& w, I3 rel) {
  const uint32_t* gd = w.f->grid_dim;
  return (uint64_t)(uint32_t)rel.x + (uint64_t)(uint32_t)rel.y * gd[0] +
         (uint64_t)(uint32_t)rel.z * gd[0] * gd[1];
}
// i32 subtraction with WGSL's wrapping semantics (a cell from the floor of an
// infinite coordinate saturates to INT32_MAX / INT32_MIN and may overflow)
inline int32_t wsub(int32_t a, int32_t b) { return (int32_t)((uint32_t)a - (uint32_t)b); }
inline I3 grid_rel(const World& w, I3 cell) {
  return {wsub(cell.x, w.f->grid_min[0]), wsub(cell.y, w.f->grid_min[1]), wsub(cell.z, w.f->grid_min[2])};
}
inline bool grid_outside(const World& w, I3 rel) {
  const uint32_t* gd = w.f->grid_dim;
  return rel.x < 0 || rel.y < 0 || rel.z < 0 || rel.x >= (int32_t)gd[0] ||
         rel.y >= (int32_t)gd[1] || rel.z >= (int32_t)gd[2];
}

// world_block_at: common.wgsl:266-277
uint32_t world_block_at(const World& w, V3 p) {
  I3 cell = floor_i(divs(p, 64.0f));
  cell = grid_rel(w, cell);
  if (grid_outside(w, cell)) return 0u;
  cnt_add(&Counters::grid_lookups);
  uint32_t ci = grid_at(w, grid_index(w, cell));
  if (ci == VM_NO_CHUNK) return 0u;
  const vm_chunk& c = chunk_at(w, ci);
  I3 v = floor_i(divs(sub(p, ld3(c.origin)), c.voxel_size));
  if (v.x < 0 || v.y < 0 || v.z < 0 || v.x >= 64 || v.y >= 64 || v.z >= 64) return 0u;
  if (!voxel_occupied(w, ci, v)) return 0u;
  return block_at(w, ci, U3{(uint32_t)v.x, (uint32_t)v.y, (uint32_t)v.z});
}

// ray_dir: common.wgsl:358-368
V3 ray_dir(const vm_frame& f, float px, float py) {
  float ndc_x = ((px + f.jitter[0]) / (float)f.res[0]) * 2.0f - 1.0f;
  float ndc_y = 1.0f - ((py + f.jitter[1]) / (float)f.res[1]) * 2.0f;
  V3 v = add(add(ld3(f.cam_fwd), muls(ld3(f.cam_right), ndc_x * f.tan_half_fov * f.aspect)),
             muls(ld3(f.cam_up), ndc_y * f.tan_half_fov));
  V3 d = normalize(v);
  V3 o;
  o.x = fabsf(d.x) < 1e-6f ? 1e-6f * signf(d.x + 1e-9f) : d.x;
  o.y = fabsf(d.y) < 1e-6f ? 1e-6f * signf(d.y + 1e-9f) : d.y;
  o.z = fabsf(d.z) < 1e-6f ? 1e-6f * signf(d.z + 1e-9f) : d.z;
  return o;
}

inline float fractf(float x) { return x - floorf(x); }

// dither / ray_skips: common.wgsl:370-385
bool ray_skips(const vm_frame& f, float fade, uint32_t px, uint32_t py) {
  if (fade >= 1.0f) return false;
  float p0 = (float)px + 5.588238f * (float)f.frame_index;
  float p1 = (float)py;
  float d = fractf(52.9829189f * fractf(p0 * 0.06711056f + p1 * 0.00583715f));
  if (fade >= 0.0f) return d >= fade;
  return d < -fade;
}

// normal_of: common.wgsl:387-398
V3 normal_of(uint32_t id) {
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

// hash_u32: common.wgsl:1422-1430
inline uint32_t hash_u32(uint32_t x) {
  uint32_t h = x;
  h ^= h >> 16u;
  h *= 0x7feb352du;
  h ^= h >> 15u;
  h *= 0x846ca68bu;
  h ^= h >> 16u;
  return h;
}

// Soft shadows (VM_SPEC_SOFT_RAYS, an extension of the engine): the s-th
// jittered sun direction of pixel (px, py): the sun's tangent basis from a
// fixed up vector, one rotation of the shared disk pattern picked by hash_u32
// of pixel and frame, the offset added in the tangent plane, normalised.
static const float SOFT_DISK[VM_SOFT_ROTATIONS][VM_SOFT_SAMPLES][2] = VM_SOFT_DISK_INIT;
V3 soft_sun_dir(const vm_frame& f, uint32_t px, uint32_t py, uint32_t s) {
  const V3 sun = ld3(f.sun_dir);
  const V3 up = fabsf(sun.y) < 0.99f ? V3{0.0f, 1.0f, 0.0f} : V3{1.0f, 0.0f, 0.0f};
  const V3 c = cross(sun, up);
  const float lc = sqrtf(dot(c, c));
  const V3 tg = {c.x / lc, c.y / lc, c.z / lc};
  const V3 bt = cross(tg, sun);
  const uint32_t r = hash_u32((px * 73856093u) ^ (py * 19349663u) ^ (f.frame_index * 83492791u)) &
                     (VM_SOFT_ROTATIONS - 1u);
  const V3 v = add(add(sun, muls(tg, SOFT_DISK[r][s][0])), muls(bt, SOFT_DISK[r][s][1]));
  const float l = sqrtf(dot(v, v));
  return {v.x / l, v.y / l, v.z / l};
}

// leaf_solid: common.wgsl:514-518
bool leaf_solid(I3 wv, U3 m, float fill = VM_LEAF_FILL) {
  int32_t qx = (int32_t)((uint32_t)wv.x * 4u + m.x);
  int32_t qy = (int32_t)((uint32_t)wv.y * 4u + m.y);
  int32_t qz = (int32_t)((uint32_t)wv.z * 4u + m.z);
  uint32_t h = hash_u32(((uint32_t)qx * 73856093u) ^ ((uint32_t)qy * 19349663u) ^
                        ((uint32_t)qz * 83492791u));
  return (float)(h >> 8u) * (1.0f / 16777216.0f) < fill;
}

// micro_entry: common.wgsl:520-528
U3 micro_entry(U3 uc, V3 ro, V3 rd, float t, uint32_t axis, const bool* pos_dir, bool snap) {
  V3 p = muls(sub(add(ro, muls(rd, t)), v3((float)uc.x, (float)uc.y, (float)uc.z)), 4.0f);
  I3 m = floor_i(p);
  m = {std::min(std::max(m.x, 0), 3), std::min(std::max(m.y, 0), 3), std::min(std::max(m.z, 0), 3)};
  if (snap) setc(m, axis, pos_dir[axis] ? 0 : 3);
  return {(uint32_t)m.x, (uint32_t)m.y, (uint32_t)m.z};
}

struct MicroHit { bool hit; float t; uint32_t normal; U3 micro; };

// cutout_march: common.wgsl:537-577
MicroHit cutout_march(I3 wv, U3 uc, V3 ro, V3 rd, float t_in, uint32_t axis_in,
                      const bool* pos_dir, bool snap, float fill) {
  MicroHit r{false, t_in, 0u, {0u, 0u, 0u}};
  V3 base = v3((float)uc.x, (float)uc.y, (float)uc.z);
  V3 inv = v3(1.0f / rd.x, 1.0f / rd.y, 1.0f / rd.z);
  const float ms = 1.0f / 4.0f;
  U3 me = micro_entry(uc, ro, rd, t_in, axis_in, pos_dir, snap);
  I3 m{(int32_t)me.x, (int32_t)me.y, (int32_t)me.z};
  float t = t_in;
  uint32_t axis = axis_in;
  for (uint32_t i = 0; i < 12u; ++i) {
    if (m.x < 0 || m.y < 0 || m.z < 0 || m.x >= 4 || m.y >= 4 || m.z >= 4) return r;
    if (leaf_solid(wv, U3{(uint32_t)m.x, (uint32_t)m.y, (uint32_t)m.z}, fill)) {
      r.hit = true;
      r.t = t;
      r.normal = axis * 2u + (pos_dir[axis] ? 0u : 1u);
      r.micro = {(uint32_t)m.x, (uint32_t)m.y, (uint32_t)m.z};
      return r;
    }
    V3 bound = v3((float)(pos_dir[0] ? m.x + 1 : m.x), (float)(pos_dir[1] ? m.y + 1 : m.y),
                  (float)(pos_dir[2] ? m.z + 1 : m.z));
    V3 tn = mul(sub(add(base, muls(bound, ms)), ro), inv);
    if (tn.x <= tn.y && tn.x <= tn.z) { t = tn.x; axis = 0u; }
    else if (tn.y <= tn.z) { t = tn.y; axis = 1u; }
    else { t = tn.z; axis = 2u; }
    setc(m, axis, comp(m, axis) + (pos_dir[axis] ? 1 : -1));
  }
  return r;
}

inline bool is_tuft(uint32_t b) { return b == VM_TALL_GRASS || b == VM_GRASS_TALL || b == VM_REEDS; }
inline bool is_cutout_id(uint32_t b) { return b == VM_LEAVES || b == VM_PINE_LEAVES; }
inline bool casts_sun_shadow(uint32_t id) { return id != VM_GLOWSTONE; }  // common.wgsl:264

struct Hit { bool hit; float t; uint32_t normal; U3 voxel; U3 micro; uint32_t iters; };

// textureSampleLevel(atlas, atlas_samp, uv, layer, lod).a with the engine's
// atlas sampler (mag nearest, min / mipmap linear, clamp to edge), the alpha
// of the Rgba8UnormSrgb texels being linear (a / 255)
float atlas_alpha_texel(const World& w, uint32_t mip, uint32_t layer, int32_t x, int32_t y) {
  uint64_t base = 0;
  for (uint32_t m = 0; m < mip; ++m) base += (uint64_t)w.atlas_layers * (16u >> m) * (16u >> m);
  int32_t size = (int32_t)(16u >> mip);
  x = std::min(std::max(x, 0), size - 1);
  y = std::min(std::max(y, 0), size - 1);
  return (float)w.atlas[4 * (base + ((uint64_t)layer * size + y) * size + x) + 3] / 255.0f;
}
float atlas_alpha_bilinear(const World& w, uint32_t mip, uint32_t layer, float u, float v) {
  float size = (float)(16u >> mip);
  float x = u * size - 0.5f, y = v * size - 0.5f;
  float x0 = floorf(x), y0 = floorf(y);
  float ax = x - x0, ay = y - y0;
  int32_t ix = f2i(x0), iy = f2i(y0);
  int32_t ix1 = (int32_t)((uint32_t)ix + 1u), iy1 = (int32_t)((uint32_t)iy + 1u);
  float a0 = atlas_alpha_texel(w, mip, layer, ix, iy) * (1.0f - ax) + atlas_alpha_texel(w, mip, layer, ix1, iy) * ax;
  float a1 = atlas_alpha_texel(w, mip, layer, ix, iy1) * (1.0f - ax) + atlas_alpha_texel(w, mip, layer, ix1, iy1) * ax;
  return a0 * (1.0f - ay) + a1 * ay;
}
float atlas_alpha(const World& w, uint32_t layer, float u, float v, float lod) {
  if (layer >= w.atlas_layers) layer = w.atlas_layers - 1u;
  if (!(lod > 0.0f)) return atlas_alpha_texel(w, 0, layer, f2i(floorf(u * 16.0f)), f2i(floorf(v * 16.0f)));
  float d = fminf(lod, 3.0f), dl = floorf(d), delta = d - dl;
  uint32_t m0 = f2u(dl);
  float a = atlas_alpha_bilinear(w, m0, layer, u, v);
  if (!(delta > 0.0f) || m0 + 1u >= 4u) return a;
  return a * (1.0f - delta) + atlas_alpha_bilinear(w, m0 + 1u, layer, u, v) * delta;
}

// hash_alpha: common.wgsl:400-406
float hash_alpha_p(V3 p) {
  I3 q = floor_i(muls(p, 64.0f));
  uint32_t h = ((uint32_t)q.x * 73856093u) ^ ((uint32_t)q.y * 19349663u) ^ ((uint32_t)q.z * 83492791u);
  h = h ^ (h >> 13u);
  h = h * 1274126177u;
  return (float)((h >> 8u) & 0xFFFFFFu) / 16777216.0f;
}

struct CrossHit { bool hit; float t; uint32_t normal; };

// cross_quad: common.wgsl:425-487 (shear: wind_shear, SPEC_WIND_SWAY)
CrossHit cross_quad(const World& w, U3 uc, V3 ro, V3 rd, uint32_t layer, float vs, bool sway, float shx, float shz) {
  const vm_frame& f = *w.f;
  CrossHit r{false, 0.0f, VM_NORMAL_CROSS_A};
  V3 base = v3((float)uc.x, (float)uc.y, (float)uc.z);
  float ts[2] = {-1.0f, -1.0f};
  if (sway) {
    float dy = ro.y - base.y;
    float ka = shx - shz, kb = shx + shz;
    float da = rd.x - rd.z - ka * rd.y;
    if (fabsf(da) > 1e-6f) ts[0] = ((base.x - base.z) + ka * dy - (ro.x - ro.z)) / da;
    float db = rd.x + rd.z - kb * rd.y;
    if (fabsf(db) > 1e-6f) ts[1] = ((base.x + base.z + 1.0f) + kb * dy - (ro.x + ro.z)) / db;
  } else {
    float da = rd.x - rd.z;
    if (fabsf(da) > 1e-6f) ts[0] = ((base.x - base.z) - (ro.x - ro.z)) / da;
    float db = rd.x + rd.z;
    if (fabsf(db) > 1e-6f) ts[1] = ((base.x + base.z + 1.0f) - (ro.x + ro.z)) / db;
  }
  uint32_t order[2] = {VM_NORMAL_CROSS_A, VM_NORMAL_CROSS_B};
  if (ts[1] < ts[0]) { std::swap(ts[0], ts[1]); std::swap(order[0], order[1]); }
  for (uint32_t i = 0; i < 2u; ++i) {
    float tq = ts[i];
    if (tq < 0.0f) continue;
    V3 p = add(ro, muls(rd, tq));
    V3 local = sub(p, base);
    if (local.x < -1e-4f || local.y < -1e-4f || local.z < -1e-4f || local.x > 1.0f + 1e-4f ||
        local.y > 1.0f + 1e-4f || local.z > 1.0f + 1e-4f)
      continue;
    float footprint = fmaxf(tq * vs, 1e-3f) * 2.0f * f.tan_half_fov / (float)f.res[1] * 16.0f / vs;
    float lod = fminf(fmaxf(log2f(fmaxf(footprint, 1e-4f)) + f.mip_bias, 0.0f), 3.0f);
    float a = atlas_alpha(w, layer, local.x, 1.0f - local.y, lod);
    if (a <= hash_alpha_p(p)) continue;
    r.hit = true; r.t = tq; r.normal = order[i];
    return r;
  }
  return r;
}

// march_chunk: common.wgsl:579-910.  Tufts (ids 18/24/25) are traced as
// cross quads when the world carries the atlas (foliage_trace), else they
// are transparent.
Hit march_chunk(const World& w, uint32_t ci, V3 ro_w, V3 rd, float t_limit, bool skip_water,
                bool skip_foliage, bool skip_glass, bool sun_ray) {
  Hit h{false, 0.0f, 0u, {0u, 0u, 0u}, {0u, 0u, 0u}, 0u};
  cnt_add(&Counters::march_calls);
  cnt_add(&Counters::chunk_records);
  const vm_chunk& c = chunk_at(w, ci);
  float vs = c.voxel_size;
  V3 origin = ld3(c.origin);
  V3 ro = divs(sub(ro_w, origin), vs);
  V3 inv = v3(1.0f / rd.x, 1.0f / rd.y, 1.0f / rd.z);
  V3 bmin = divs(sub(ld3(c.aabb_min), origin), vs);
  V3 bmax = divs(sub(ld3(c.aabb_max), origin), vs);
  V3 t0 = mul(sub(bmin, ro), inv);
  V3 t1 = mul(sub(bmax, ro), inv);
  V3 tmin3 = vmin(t0, t1);
  V3 tmax3 = vmax(t0, t1);
  float t_enter = fmaxf(fmaxf(tmin3.x, tmin3.y), tmin3.z);
  float t_exit = fminf(fminf(tmax3.x, tmax3.y), tmax3.z);
  float t_end = fminf(t_exit, t_limit / vs);
  float t = fmaxf(t_enter, 0.0f);
  if (t >= t_end) return h;
  uint32_t axis;
  if (tmin3.x >= tmin3.y && tmin3.x >= tmin3.z) axis = 0u;
  else if (tmin3.y >= tmin3.z) axis = 1u;
  else axis = 2u;
  bool pos_dir[3] = {rd.x > 0.0f, rd.y > 0.0f, rd.z > 0.0f};
  V3 pos = add(ro, muls(rd, t));
  I3 cell = floor_i(pos);
  if (t_enter > 0.0f) {
    setc(cell, axis, pos_dir[axis] ? f2i(floorf(comp(bmin, axis))) : f2i(ceilf(comp(bmax, axis))) - 1);
  }
  cell = {std::min(std::max(cell.x, 0), 63), std::min(std::max(cell.y, 0), 63),
          std::min(std::max(cell.z, 0), 63)};
  U2 root_mask{c.root[0], c.root[1]};
  uint32_t root_ptr = c.root[2] & VM_PTR_MASK;

  bool water_aware = skip_water && (c.attr_flags & VM_ATTR_HAS_WATER) != 0u;
  if (water_aware && (c.attr_flags & VM_ATTR_UNIFORM) != 0u) {
    if (c.attr_base == VM_WATER) return h;
    water_aware = false;
  }
  bool attr_uniform = (c.attr_flags & VM_ATTR_UNIFORM) != 0u;
  // pipeline specialisations (common.wgsl:635-666): SPEC_FOLIAGE,
  // SPEC_LEAF_CUTOUT, SPEC_GLASS, SPEC_EMITTER_GATHER, SPEC_WATER_REPAIR
  bool foliage_aware = (w.spec & VM_SPEC_FOLIAGE) != 0u && (c.attr_flags & VM_ATTR_HAS_FOLIAGE) != 0u;
  if (foliage_aware && attr_uniform && !is_tuft(c.attr_base)) foliage_aware = false;
  bool cutout_aware = (w.spec & VM_SPEC_LEAF_CUTOUT) != 0u && (c.attr_flags & VM_ATTR_HAS_CUTOUT) != 0u && vs == 1.0f;
  if (cutout_aware && attr_uniform && c.attr_base != VM_LEAVES && c.attr_base != VM_PINE_LEAVES)
    cutout_aware = false;
  bool glass_aware = (w.spec & VM_SPEC_GLASS) != 0u && skip_glass && (c.attr_flags & VM_ATTR_HAS_GLASS) != 0u;
  if (glass_aware && attr_uniform) {
    if (c.attr_base == VM_GLASS) return h;
    glass_aware = false;
  }
  bool noncaster_aware = (w.spec & VM_SPEC_EMITTER_GATHER) != 0u && sun_ray && (c.attr_flags & VM_ATTR_HAS_EMITTER) != 0u;
  if (noncaster_aware && attr_uniform && !casts_sun_shadow(c.attr_base)) return h;
  bool water_interface = (w.spec & VM_SPEC_WATER_REPAIR) != 0u && !skip_water && (c.attr_flags & VM_ATTR_HAS_WATER) != 0u;
  bool attr_needed = (noncaster_aware && !attr_uniform) || (water_interface && !attr_uniform) ||
                     water_aware || glass_aware || ((foliage_aware || cutout_aware) && !attr_uniform);

  U2 trav_mask = root_mask;
  if (water_aware) trav_mask = U2{c.dry_mask[0], c.dry_mask[1]};
  bool root_full = (c.root[2] & VM_FULL_BIT) != 0u;
  // the full-root short cut without SPEC_FULL_MARCH (common.wgsl:677-686)
  if (root_full && (w.spec & VM_SPEC_FULL_MARCH) == 0u && !noncaster_aware && !water_interface) {
    h.hit = true;
    h.t = t * vs;
    h.normal = axis * 2u + (pos_dir[axis] ? 0u : 1u);
    h.voxel = {(uint32_t)cell.x, (uint32_t)cell.y, (uint32_t)cell.z};
    h.micro = micro_entry(h.voxel, ro, rd, t, axis, pos_dir, t > 0.0f);
    return h;
  }
  if (trav_mask.x == 0u && trav_mask.y == 0u) return h;

  uint32_t l1_cached = 0xFFFFFFFFu;
  U4 l1{0u, 0u, 0u, 0u};
  uint32_t leaf_cached = 0xFFFFFFFFu;
  U2 leaf{0u, 0u};
  uint32_t attr = 0u;
  for (;;) {
    h.iters += 1u;
    cnt_add(&Counters::iters);
    if (h.iters > VM_MAX_ITERS) break;
    if (cell.x < 0 || cell.y < 0 || cell.z < 0 || cell.x > 63 || cell.y > 63 || cell.z > 63) break;
    U3 uc{(uint32_t)cell.x, (uint32_t)cell.y, (uint32_t)cell.z};
    int32_t skip = 16;
    bool solid = false;
    uint32_t l1b = cell_bit(ushr(uc, 4u));
    if (mask_has(trav_mask, l1b)) {
      if (l1b != l1_cached) {
        l1_cached = l1b;
        if (root_full) {
          l1 = {0xFFFFFFFFu, 0xFFFFFFFFu, VM_FULL_BIT, (l1b * 64u) | 0xF0000000u};
        } else {
          cnt_add(&Counters::l1_fetches);
          l1 = inner_at(w, (uint64_t)root_ptr + mask_below(root_mask, l1b));
        }
        leaf_cached = 0xFFFFFFFFu;
      }
      bool line_skip = false;
      if (water_aware) {
        uint32_t wl = l1.w >> 28u;
        float ly = (float)(uc.y & 15u);
        if (wl < 15u && ly > (float)wl) {
          line_skip = rd.y >= 0.0f;
          if (!line_skip) {
            float hh = fmaxf(fabsf(rd.x), fabsf(rd.z));
            if (hh > 1e-6f && (ly - (float)wl) > 16.0f * (fabsf(rd.y) / hh)) line_skip = true;
          }
        }
      }
      if (line_skip) {
        skip = 16;
      } else if ((l1.z & VM_FULL_BIT) != 0u) {
        solid = true;
        if (attr_needed) {
          uint32_t lfb = cell_bit(uand(ushr(uc, 2u), 3u));
          if (lfb != leaf_cached) {
            leaf_cached = lfb;
            cnt_add(&Counters::attr_fetches);
            attr = brick_at(w, (uint64_t)c.attr_base + (l1.w & 0x0FFFFFFFu) + lfb);
          }
        }
      } else {
        U2 l1m{l1.x, l1.y};
        uint32_t lfb = cell_bit(uand(ushr(uc, 2u), 3u));
        if (mask_has(l1m, lfb)) {
          if (lfb != leaf_cached) {
            leaf_cached = lfb;
            uint32_t li = mask_below(l1m, lfb);
            cnt_add(&Counters::leaf_fetches);
            leaf = leaf_at(w, (uint64_t)(l1.z & VM_PTR_MASK) + li);
            if (attr_needed) {
              cnt_add(&Counters::attr_fetches);
              attr = brick_at(w, (uint64_t)c.attr_base + (l1.w & 0x0FFFFFFFu) + li);
            }
          }
          uint32_t vb = cell_bit(uand(uc, 3u));
          if (mask_has(leaf, vb)) {
            solid = true;
          } else {
            uint32_t sh = vb & 42u;
            uint32_t lo;
            if (sh == 0u) lo = leaf.x;
            else if (sh < 32u) lo = (leaf.x >> sh) | (leaf.y << (32u - sh));
            else lo = leaf.y >> (sh - 32u);
            skip = (lo & 0x00330033u) == 0u ? 2 : 1;
          }
        } else {
          skip = 4;
        }
      }
    } else {
      uint32_t sh = l1b & 42u;
      uint32_t rlo;
      if (sh == 0u) rlo = trav_mask.x;
      else if (sh < 32u) rlo = (trav_mask.x >> sh) | (trav_mask.y << (32u - sh));
      else rlo = trav_mask.y >> (sh - 32u);
      skip = (rlo & 0x00330033u) == 0u ? 32 : 16;
    }
    if (solid && noncaster_aware) {
      uint32_t id = attr_uniform ? c.attr_base : leaf_block(w, attr, uc);
      if (!casts_sun_shadow(id)) { solid = false; skip = 1; }
    }
    if (solid && water_interface) {
      uint32_t id = attr_uniform ? c.attr_base : leaf_block(w, attr, uc);
      if (id == VM_WATER) {
        uint32_t nid = axis * 2u + (pos_dir[axis] ? 0u : 1u);
        V3 outward = normal_of(nid);
        V3 boundary = add(ro_w, muls(rd, t * vs));
        if (world_block_at(w, add(boundary, muls(outward, 0.002f * vs))) == VM_WATER) {
          solid = false;
          skip = 1;
        }
      }
    }
    if (solid && water_aware) {
      if (leaf_block(w, attr, uc) == VM_WATER) {
        solid = false;
        skip = (attr & VM_UNIFORM_BIT) != 0u ? 4 : 1;
      }
    }
    if (solid && glass_aware) {
      if (leaf_block(w, attr, uc) == VM_GLASS) {
        solid = false;
        skip = (attr & VM_UNIFORM_BIT) != 0u ? 4 : 1;
      }
    }
    if (solid && foliage_aware) {
      uint32_t bid = attr_uniform ? c.attr_base : leaf_block(w, attr, uc);
      if (is_tuft(bid)) {
        solid = false;
        skip = 1;
        if (!skip_foliage && w.atlas != nullptr) {
          bool sway = (w.spec & VM_SPEC_WIND_SWAY) != 0u;
          float shx = 0.0f, shz = 0.0f;
          if (sway) {
            float wx = c.origin[0] + (float)uc.x * vs, wz = c.origin[2] + (float)uc.z * vs;
            float time = w.f->time * w.f->cloud_speed;
            float g = 0.65f * sinf(time * 1.9f + wx * 0.11f + wz * 0.07f) +
                      0.35f * sinf(time * 3.1f + wx * 0.173f + wz * 0.129f + 1.7f);
            shx = g * 0.8f * 0.09f;
            shz = g * 0.6f * 0.09f;
          }
          uint32_t fi = bid * 8u + VM_NORMAL_CROSS_A;
          uint32_t layer = fi < w.n_faces ? (w.faces[fi] & 0xFFFFu) : 0u;
          CrossHit q = cross_quad(w, uc, ro, rd, layer, vs, sway, shx, shz);
          if (q.hit) {
            h.hit = true;
            h.t = q.t * vs;
            h.normal = q.normal;
            h.voxel = uc;
            return h;
          }
        }
      }
    }
    if (solid && cutout_aware) {
      uint32_t bid = attr_uniform ? c.attr_base : leaf_block(w, attr, uc);
      if (is_cutout_id(bid)) {
        I3 wv{f2i(c.origin[0]) + (int32_t)uc.x, f2i(c.origin[1]) + (int32_t)uc.y,
              f2i(c.origin[2]) + (int32_t)uc.z};
        MicroHit q = cutout_march(wv, uc, ro, rd, t, axis, pos_dir, t > 0.0f,
                                  (w.spec & VM_SPEC_LEAF_THIN) ? VM_LEAF_FILL : VM_LEAF_FILL_PRE43);
        if (q.hit) {
          h.hit = true;
          h.t = q.t * vs;
          h.normal = q.normal;
          h.voxel = uc;
          h.micro = q.micro;
          return h;
        }
        solid = false;
        skip = 1;
      }
    }
    if (solid) {
      h.hit = true;
      h.t = t * vs;
      h.normal = axis * 2u + (pos_dir[axis] ? 0u : 1u);
      h.voxel = uc;
      h.micro = micro_entry(uc, ro, rd, t, axis, pos_dir, t > 0.0f);
      return h;
    }
    I3 bmin_i{cell.x - (cell.x & (skip - 1)), cell.y - (cell.y & (skip - 1)), cell.z - (cell.z & (skip - 1))};
    I3 bmax_i{bmin_i.x + skip, bmin_i.y + skip, bmin_i.z + skip};
    V3 bounds = v3((float)(pos_dir[0] ? bmax_i.x : bmin_i.x), (float)(pos_dir[1] ? bmax_i.y : bmin_i.y),
                   (float)(pos_dir[2] ? bmax_i.z : bmin_i.z));
    V3 tn = mul(sub(bounds, ro), inv);
    if (tn.x <= tn.y && tn.x <= tn.z) { t = tn.x; axis = 0u; }
    else if (tn.y <= tn.z) { t = tn.y; axis = 1u; }
    else { t = tn.z; axis = 2u; }
    if (t >= t_end) break;
    pos = add(ro, muls(rd, t));
    cell = floor_i(pos);
    setc(cell, axis, pos_dir[axis] ? comp(bmax_i, axis) : comp(bmin_i, axis) - 1);
  }
  return h;
}

V3 refract(V3 e1, V3 e2, float e3);

// glass is its own surface only with SPEC_GLASS (shadow.wgsl:18, resolve.wgsl:1440)
inline bool glass_leg(const World& w, uint32_t id) { return (w.spec & VM_SPEC_GLASS) != 0u && id == VM_GLASS; }

// SPEC_SNELL_BEND: march.wgsl:23-44 (the straight march of chunk ci missed)
void snell_bend(const World& w, uint32_t ci, V3 rd, Hit& h) {
  const vm_frame& f = *w.f;
  const float depth = f.sea_level - f.cam_pos[1];
  if (!(depth > 0.0f)) return;
  const float t_surf = depth / rd.y;
  if (!(t_surf < f.far_)) return;
  const V3 surf = add(ld3(f.cam_pos), muls(rd, t_surf));
  const V3 rd2 = refract(rd, v3(0.0f, -1.0f, 0.0f), VM_WATER_IOR);
  if (!(dot(rd2, rd2) > 0.0f)) return;
  Hit h2 = march_chunk(w, ci, add(surf, muls(rd2, VM_SURFACE_EPS)), rd2, f.far_ - t_surf, true, false, false, false);
  if (h2.hit) {
    const uint32_t straight_iters = h.iters;
    h = h2;
    h.t = t_surf + h2.t;
    h.iters = straight_iters + h2.iters;
  }
}

// shadow_ray_t: common.wgsl:1156-1195
float shadow_ray_t(const World& w, V3 ro, V3 rd, float max_dist) {
  V3 inv = v3(1.0f / rd.x, 1.0f / rd.y, 1.0f / rd.z);
  bool pos_dir[3] = {rd.x > 0.0f, rd.y > 0.0f, rd.z > 0.0f};
  I3 cell = floor_i(divs(ro, 64.0f));
  float t = 0.0f;
  uint32_t last = VM_NO_CHUNK;
  for (uint32_t i = 0; i < 24u; ++i) {
    I3 rel = grid_rel(w, cell);
    if (grid_outside(w, rel)) return -1.0f;
    cnt_add(&Counters::grid_lookups);
    uint32_t ci = grid_at(w, grid_index(w, rel));
    if (ci != VM_NO_CHUNK && ci != last) {
      last = ci;
      Hit m = march_chunk(w, ci, ro, rd, max_dist, true, true, true, true);
      if (m.hit) return m.t;
    }
    V3 bounds = muls(v3((float)(pos_dir[0] ? cell.x + 1 : cell.x), (float)(pos_dir[1] ? cell.y + 1 : cell.y),
                        (float)(pos_dir[2] ? cell.z + 1 : cell.z)), 64.0f);
    V3 tn = mul(sub(bounds, ro), inv);
    uint32_t axis = 0u;
    if (tn.x <= tn.y && tn.x <= tn.z) { t = tn.x; }
    else if (tn.y <= tn.z) { t = tn.y; axis = 1u; }
    else { t = tn.z; axis = 2u; }
    if (t >= max_dist) return -1.0f;
    setc(cell, axis, comp(cell, axis) + (pos_dir[axis] ? 1 : -1));
  }
  return -1.0f;
}

struct WorldHit { bool hit; float t; uint32_t normal; U3 voxel; uint32_t ci; };

// trace_world: common.wgsl:1205-1253
WorldHit trace_world(const World& w, V3 ro, V3 rd, float max_dist, bool skip_water) {
  WorldHit out{false, max_dist, 0u, {0u, 0u, 0u}, VM_NO_CHUNK};
  V3 dir;
  dir.x = fabsf(rd.x) < 1e-6f ? 1e-6f * signf(rd.x + 1e-9f) : rd.x;
  dir.y = fabsf(rd.y) < 1e-6f ? 1e-6f * signf(rd.y + 1e-9f) : rd.y;
  dir.z = fabsf(rd.z) < 1e-6f ? 1e-6f * signf(rd.z + 1e-9f) : rd.z;
  V3 inv = v3(1.0f / dir.x, 1.0f / dir.y, 1.0f / dir.z);
  bool pos_dir[3] = {dir.x > 0.0f, dir.y > 0.0f, dir.z > 0.0f};
  I3 cell = floor_i(divs(ro, 64.0f));
  for (uint32_t i = 0; i < 16u; ++i) {
    I3 rel = grid_rel(w, cell);
    if (grid_outside(w, rel)) return out;
    cnt_add(&Counters::grid_lookups);
    uint32_t ci = grid_at(w, grid_index(w, rel));
    V3 bounds = muls(v3((float)(pos_dir[0] ? cell.x + 1 : cell.x), (float)(pos_dir[1] ? cell.y + 1 : cell.y),
                        (float)(pos_dir[2] ? cell.z + 1 : cell.z)), 64.0f);
    V3 tn = mul(sub(bounds, ro), inv);
    float t_exit = tn.x;
    uint32_t axis = 0u;
    if (tn.y < t_exit) { t_exit = tn.y; axis = 1u; }
    if (tn.z < t_exit) { t_exit = tn.z; axis = 2u; }
    if (ci != VM_NO_CHUNK) {
      Hit h = march_chunk(w, ci, ro, rd, fminf(t_exit, max_dist), skip_water, false, true, false);
      if (h.hit) {
        out.hit = true; out.t = h.t; out.normal = h.normal; out.voxel = h.voxel; out.ci = ci;
        return out;
      }
    }
    if (t_exit >= max_dist) return out;
    setc(cell, axis, comp(cell, axis) + (pos_dir[axis] ? 1 : -1));
  }
  return out;
}

// hit_t: common.wgsl:1300-1318
float hit_t(const World& w, uint32_t ci, U3 v, U3 micro, uint32_t normal_id, V3 rd) {
  const vm_chunk& c = chunk_at(w, ci);
  const vm_frame& f = *w.f;
  V3 box_min = add(ld3(c.origin), muls(v3((float)v.x, (float)v.y, (float)v.z), c.voxel_size));
  if (normal_id >= VM_NORMAL_CROSS_A) {
    if (normal_id == VM_NORMAL_CROSS_A)
      return ((box_min.x - box_min.z) - (f.cam_pos[0] - f.cam_pos[2])) / (rd.x - rd.z);
    return ((box_min.x + box_min.z + c.voxel_size) - (f.cam_pos[0] + f.cam_pos[2])) / (rd.x + rd.z);
  }
  uint32_t axis = normal_id >> 1u;
  float ms = c.voxel_size / 4.0f;
  uint32_t mi = axis == 0 ? micro.x : (axis == 1 ? micro.y : micro.z);
  float plane = comp(box_min, axis) + (float)(mi + ((normal_id & 1u) == 1u ? 1u : 0u)) * ms;
  return (plane - f.cam_pos[axis]) / comp(rd, axis);
}

// depth_key / make_key: common.wgsl:1320-1330
inline uint32_t depth_key(const vm_frame& f, float t) {
  float x = 1.0f - t / f.far_;
  x = fminf(fmaxf(x, 0.0f), 1.0f);
  return f2u(x * 16777215.0f);
}
inline uint64_t make_key(const vm_frame& f, float t, uint32_t normal, uint32_t ci, U3 v, U3 micro) {
  uint64_t d = depth_key(f, t);
  uint32_t bx = v.x | (micro.x << 6u), by = v.y | (micro.y << 6u), bz = v.z | (micro.z << 6u);
  return (d << 40) | ((uint64_t)normal << 37) | ((uint64_t)ci << 24) |
         (uint64_t)((bx << 16u) | (by << 8u) | bz);
}

// tile_select geometry: tile_select.wgsl:1-9
inline bool box_outside(V3 bmin, V3 bmax, V3 n, V3 cam) {
  V3 p{n.x > 0.0f ? bmax.x : bmin.x, n.y > 0.0f ? bmax.y : bmin.y, n.z > 0.0f ? bmax.z : bmin.z};
  return dot(n, sub(p, cam)) < 0.0f;
}
inline float box_distance(V3 p, V3 bmin, V3 bmax) {
  return length(vmax(vmax(sub(bmin, p), sub(p, bmax)), v3(0.0f, 0.0f, 0.0f)));
}

struct TileCull {
  V3 n[4];
  float reach;
};

// per-tile planes and reach: tile_select.wgsl:11-57
TileCull tile_planes(const vm_frame& f, uint32_t tx, uint32_t ty) {
  float x0 = (float)(tx * 8u), y0 = (float)(ty * 8u);
  float x1 = x0 + 8.0f, y1 = y0 + 8.0f;
  V3 d00 = ray_dir(f, x0, y0), d10 = ray_dir(f, x1, y0), d11 = ray_dir(f, x1, y1), d01 = ray_dir(f, x0, y1);
  V3 center = ray_dir(f, (x0 + x1) * 0.5f, (y0 + y1) * 0.5f);
  TileCull tc;
  tc.n[0] = cross(d00, d10);
  tc.n[1] = cross(d10, d11);
  tc.n[2] = cross(d11, d01);
  tc.n[3] = cross(d01, d00);
  for (int i = 0; i < 4; ++i) if (!(dot(tc.n[i], center) >= 0.0f)) tc.n[i] = neg(tc.n[i]);
  V3 cam = ld3(f.cam_pos);
  float reach = f.far_;
  const uint32_t both = VM_FLAG_UNDERWATER | VM_FLAG_WATER_FAR;
  if ((f.flags & both) == both) {
    float up = fmaxf(fmaxf(d00.y, d10.y), fmaxf(d11.y, d01.y));
    float submerged = fmaxf(f.sea_level - cam.y, 0.0f);
    float escape = 1e30f;
    if (up > 0.0f) escape = submerged / up;
    if (escape >= VM_WATER_FAR_DIST) {
      reach = fminf(f.far_, VM_WATER_FAR_DIST);
      float dep_far = submerged - up * VM_WATER_FAR_DIST;
      if ((f.flags & VM_FLAG_WATER_DARK) != 0u && fminf(submerged, dep_far) >= VM_WATER_DARK_DEPTH)
        reach = fminf(reach, VM_WATER_DARK_DIST);
    }
  }
  tc.reach = reach;
  return tc;
}

// refract per the WGSL builtin definition
V3 refract(V3 e1, V3 e2, float e3) {
  float d = dot(e2, e1);
  float k = 1.0f - e3 * e3 * (1.0f - d * d);
  if (k < 0.0f) return v3(0.0f, 0.0f, 0.0f);
  return sub(muls(e1, e3), muls(e2, e3 * d + sqrtf(k)));
}

// reflect per the WGSL builtin definition: e1 - 2 dot(e2, e1) e2
V3 reflect(V3 e1, V3 e2) {
  float d = 2.0f * dot(e2, e1);
  return sub(e1, muls(e2, d));
}

inline float smoothstep(float e0, float e1, float x) {
  float t = fminf(fmaxf((x - e0) / (e1 - e0), 0.0f), 1.0f);
  return t * t * (3.0f - 2.0f * t);
}

inline U3 key_voxel(uint64_t key) {
  uint32_t low = (uint32_t)(key & 0xFFFFFFull);
  return {(low >> 16u) & 63u, (low >> 8u) & 63u, low & 63u};
}
inline U3 key_micro(uint64_t key) {
  uint32_t low = (uint32_t)(key & 0xFFFFFFull);
  return {(low >> 22u) & 3u, (low >> 14u) & 3u, (low >> 6u) & 3u};
}
inline uint32_t key_ci(uint64_t key) { return (uint32_t)(key >> 24) & 0x1FFFu; }
inline uint32_t key_nid(uint64_t key) { return (uint32_t)(key >> 37) & 7u; }

// ---- bilateral shadow reconstruction (shadow.wgsl:7-31, 49-116) -------------

// Storage through the engine's r16float / rg16float targets: IEEE binary16,
// round to nearest even, read back as f32.  Overflow (|x| >= 65520) gives
// infinity; subnormal halves are kept.
float f16_round(float x) {
  uint32_t b;
  memcpy(&b, &x, 4);
  const uint32_t sign = b & 0x80000000u;
  uint32_t a = b & 0x7FFFFFFFu;
  if (a >= 0x7F800000u) return x;                       // inf, nan
  if (a >= 0x477FF000u) a = 0x7F800000u;                // rounds past 65504
  else if (a < 0x38800000u) {                           // below 2^-14: multiples of 2^-24
    float m;
    memcpy(&m, &a, 4);
    m = nearbyintf(m * 16777216.0f) * (1.0f / 16777216.0f);   // exact scalings, RNE rounding mode
    memcpy(&a, &m, 4);
  } else {                                              // 10 mantissa bits kept
    const uint32_t rem = a & 0x1FFFu;
    a &= ~0x1FFFu;
    if (rem > 0x1000u || (rem == 0x1000u && (a & 0x2000u) != 0u)) a += 0x2000u;
  }
  a |= sign;
  float r;
  memcpy(&r, &a, 4);
  return r;
}

// ShadowGuide / shadow_guide: shadow.wgsl:7-31
struct Guide { V3 hit, n; float t, scale; bool valid; };
Guide shadow_guide(const World& w, const uint64_t* vis, int32_t px, int32_t py) {
  const vm_frame& f = *w.f;
  Guide g{};
  g.valid = false;
  if (px < 0 || py < 0 || px >= (int32_t)f.res[0] || py >= (int32_t)f.res[1]) return g;
  const uint64_t key = vis[(uint64_t)py * f.res[0] + (uint64_t)px];
  if (key == 0ull) return g;
  const uint32_t ci = key_ci(key);
  const U3 v = key_voxel(key);
  const uint32_t id = block_at(w, ci, v);
  if (id == VM_WATER || glass_leg(w, id)) return g;
  const uint32_t nid = key_nid(key);
  const U3 micro = key_micro(key);
  const V3 rd = ray_dir(f, (float)px + 0.5f, (float)py + 0.5f);
  g.n = normal_of(nid);
  if (nid >= VM_NORMAL_CROSS_A && dot(g.n, rd) > 0.0f) g.n = neg(g.n);
  if (dot(g.n, ld3(f.sun_dir)) <= 0.0f) return g;
  g.t = hit_t(w, ci, v, micro, nid, rd);
  g.hit = add(ld3(f.cam_pos), muls(rd, g.t));
  g.scale = chunk_at(w, ci).voxel_size;
  g.valid = g.t >= 0.0f;
  return g;
}

// shadow_radius: shadow.wgsl:49-54 (SUN_ANGLE common.wgsl:1535)
inline float shadow_radius(const vm_frame& f, float distance, float depth, float penumbra, uint32_t limit) {
  const float proj = (float)f.res[1] / (2.0f * fmaxf(f.tan_half_fov, 0.001f));
  const float r = distance * 0.0093f * penumbra * proj / fmaxf(depth, 0.01f);
  return r >= 0.5f ? fminf(r, (float)limit) : 0.0f;
}

// shadow_compatible: shadow.wgsl:55-60
inline bool shadow_compatible(const Guide& a, const Guide& b) {
  if (!b.valid || dot(a.n, b.n) < 0.95f) return false;
  const float tolerance = fmaxf(0.01f, 0.01f * fminf(a.scale, b.scale));
  const V3 d = sub(b.hit, a.hit);
  return fabsf(dot(d, a.n)) <= tolerance && fabsf(dot(d, b.n)) <= tolerance;
}

}  // namespace

// ============================================================================
// C ABI of the oracle (loaded with ctypes by tests/ and bench.py)
// ============================================================================
extern "C" {

typedef struct or_world {
  const vm_frame* frame;
  const vm_chunk* chunks; uint32_t n_chunks;
  const uint32_t* inners; uint64_t n_inners;
  const uint32_t* leaves; uint64_t n_leaves;
  const uint32_t* bricks; uint64_t n_bricks;
  const uint32_t* grid; uint64_t n_grid;
  uint32_t spec;     // VM_SPEC_* pipeline specialisations
  const uint8_t* atlas; uint32_t atlas_layers;   // for the tuft quads; null: tufts transparent
  const uint32_t* faces; uint32_t n_faces;
} or_world;

typedef struct or_hit {
  uint32_t hit; float t; uint32_t normal; uint32_t voxel[3]; uint32_t micro[3]; uint32_t iters;
} or_hit;

typedef struct or_counters {
  uint64_t chunk_records, l1_fetches, leaf_fetches, attr_fetches, palette_decodes, grid_lookups,
      iters, march_calls, rays;
} or_counters;

static World mk(const or_world* o) {
  World w;
  w.f = o->frame; w.chunks = o->chunks; w.n_chunks = o->n_chunks;
  w.inners = o->inners; w.n_inners = o->n_inners;
  w.leaves = o->leaves; w.n_leaves = o->n_leaves;
  w.bricks = o->bricks; w.n_bricks = o->n_bricks;
  w.grid = o->grid; w.n_grid = o->n_grid;
  w.spec = o->spec;
  w.atlas = o->atlas; w.atlas_layers = o->atlas_layers;
  w.faces = o->faces; w.n_faces = o->n_faces;
  return w;
}

int or_last_error(char* buf, int len) {
  int e = g_err.load();
  if (e && buf && len > 0) { strncpy(buf, g_err_msg, len - 1); buf[len - 1] = 0; }
  return e;
}
void or_clear_error(void) { g_err.store(0); g_err_msg[0] = 0; }

void or_ray_dir(const vm_frame* f, float px, float py, float* out) {
  V3 d = ray_dir(*f, px, py);
  out[0] = d.x; out[1] = d.y; out[2] = d.z;
}

void or_soft_sun_dir(const vm_frame* f, uint32_t px, uint32_t py, uint32_t s, float* out) {
  V3 d = soft_sun_dir(*f, px, py, s);
  out[0] = d.x; out[1] = d.y; out[2] = d.z;
}

int or_march_chunk(const or_world* o, uint32_t ci, const float* ro, const float* rd, float t_limit,
                   uint32_t skip_water, uint32_t skip_foliage, uint32_t skip_glass, uint32_t sun_ray,
                   or_hit* out) {
  World w = mk(o);
  Hit h = march_chunk(w, ci, ld3(ro), ld3(rd), t_limit, skip_water, skip_foliage, skip_glass, sun_ray);
  out->hit = h.hit; out->t = h.t; out->normal = h.normal;
  out->voxel[0] = h.voxel.x; out->voxel[1] = h.voxel.y; out->voxel[2] = h.voxel.z;
  out->micro[0] = h.micro.x; out->micro[1] = h.micro.y; out->micro[2] = h.micro.z;
  out->iters = h.iters;
  return g_err.load();
}

float or_shadow_ray_t(const or_world* o, const float* ro, const float* rd, float max_dist) {
  World w = mk(o);
  return shadow_ray_t(w, ld3(ro), ld3(rd), max_dist);
}

int or_trace_world(const or_world* o, const float* ro, const float* rd, float max_dist,
                   uint32_t skip_water, uint32_t* hit, float* t, uint32_t* normal, uint32_t* voxel,
                   uint32_t* ci) {
  World w = mk(o);
  WorldHit h = trace_world(w, ld3(ro), ld3(rd), max_dist, skip_water);
  *hit = h.hit; *t = h.t; *normal = h.normal;
  voxel[0] = h.voxel.x; voxel[1] = h.voxel.y; voxel[2] = h.voxel.z; *ci = h.ci;
  return g_err.load();
}

uint32_t or_block_at(const or_world* o, uint32_t ci, const uint32_t* v) {
  World w = mk(o);
  return block_at(w, ci, U3{v[0], v[1], v[2]});
}

uint32_t or_world_block_at(const or_world* o, const float* p) {
  World w = mk(o);
  return world_block_at(w, ld3(p));
}

uint64_t or_make_key(const vm_frame* f, float t, uint32_t normal, uint32_t ci, const uint32_t* v,
                     const uint32_t* micro) {
  return make_key(*f, t, normal, ci, U3{v[0], v[1], v[2]}, U3{micro[0], micro[1], micro[2]});
}

uint32_t or_depth_key(const vm_frame* f, float t) { return depth_key(*f, t); }

uint32_t or_leaf_solid(const int32_t* wv, const uint32_t* m) {
  return leaf_solid(I3{wv[0], wv[1], wv[2]}, U3{m[0], m[1], m[2]});
}

// The reference's frame: tile_select (+Hi-Z deferral) -> march every pair ->
// [build_hiz -> recover_select -> march recovered] (src/render/mod.rs:1738-1794).
// vis[] receives max() of every pair's key, exactly the atomicMax fold of the
// reference.  hiz_in is the previous frame's tile buffer (read when FLAG_HIZ);
// hiz_out receives this frame's build_hiz result (FLAG_HIZ) or zeros.
// counters: [0] select count, [1] deferred, [2] recovered, [3] pairs marched,
// [4] raw select, [5] raw recover (tile_select.wgsl:112-141).
// Tiles [tile_begin, tile_end) are processed; pixels outside them are untouched.
int or_frame(const or_world* o, const uint32_t* hiz_in, uint64_t* vis, uint32_t* hiz_out,
             uint32_t* counters, uint32_t* dbg, uint32_t tile_begin, uint32_t tile_end,
             int threads, or_counters* traffic) {
  World w = mk(o);
  const vm_frame& f = *w.f;
  const uint32_t tiles_x = f.tiles[0];
  const uint32_t n_tiles = f.tiles[0] * f.tiles[1];
  if (tile_end > n_tiles) tile_end = n_tiles;
  const bool use_hiz = (f.flags & VM_FLAG_HIZ) != 0u;
  const bool underwater = (f.flags & VM_FLAG_UNDERWATER) != 0u;
  const bool heat = (f.flags & VM_FLAG_HEATMAP) != 0u && dbg;
  V3 cam = ld3(f.cam_pos);
  uint64_t c_sel = 0, c_def = 0, c_rec = 0;
  Counters total{};
  if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel reduction(+ : c_sel, c_def, c_rec)
  {
    Counters local{};
    t_cnt = traffic ? &local : nullptr;
    std::vector<uint32_t> sel, def;
#pragma omp for schedule(dynamic, 4)
    for (int64_t tid = tile_begin; tid < (int64_t)tile_end; ++tid) {
      uint32_t tile_id = (uint32_t)tid;
      uint32_t tx = tile_id % tiles_x, ty = tile_id / tiles_x;
      TileCull tc = tile_planes(f, tx, ty);
      uint32_t tile_far = use_hiz && hiz_in ? hiz_in[tile_id] : 0u;
      sel.clear(); def.clear();
      for (uint32_t ci = 0; ci < f.chunk_count; ++ci) {
        const vm_chunk& c = chunk_at(w, ci);
        if (ci == f.camera_chunk) { sel.push_back(ci); continue; }
        V3 bmin = ld3(c.aabb_min), bmax = ld3(c.aabb_max);
        if (box_outside(bmin, bmax, ld3(f.cam_fwd), cam)) continue;
        bool out = false;
        for (int i = 0; i < 4 && !out; ++i) out = box_outside(bmin, bmax, tc.n[i], cam);
        if (out) continue;
        float dmin = box_distance(cam, bmin, bmax);
        if (dmin >= tc.reach) continue;
        if (use_hiz && depth_key(f, dmin) < tile_far) { def.push_back(ci); continue; }
        sel.push_back(ci);
      }
      c_sel += sel.size();
      c_def += def.size();
      auto march_list = [&](const std::vector<uint32_t>& list) {
        for (uint32_t ci : list) {
          const vm_chunk& c = chunk_at(w, ci);
          for (uint32_t ly = 0; ly < 8u; ++ly)
            for (uint32_t lx = 0; lx < 8u; ++lx) {
              uint32_t px = tx * 8u + lx, py = ty * 8u + ly;
              if (px >= f.res[0] || py >= f.res[1]) continue;
              if (ray_skips(f, c.fade, px, py)) continue;
              V3 rd = ray_dir(f, (float)px + 0.5f, (float)py + 0.5f);
              Hit h = march_chunk(w, ci, cam, rd, f.far_, underwater, false, false, false);
              if ((w.spec & VM_SPEC_SNELL_BEND) != 0u && underwater && !h.hit && rd.y > 0.0f)
                snell_bend(w, ci, rd, h);
              uint64_t pix = (uint64_t)py * f.res[0] + px;
              if (h.hit) {
                uint64_t k = make_key(f, h.t, h.normal, ci, h.voxel, h.micro);
                if (k > vis[pix]) vis[pix] = k;
              }
              if (heat) dbg[pix] += h.iters;
            }
        }
      };
      // clear this tile's pixels
      for (uint32_t ly = 0; ly < 8u; ++ly)
        for (uint32_t lx = 0; lx < 8u; ++lx) {
          uint32_t px = tx * 8u + lx, py = ty * 8u + ly;
          if (px >= f.res[0] || py >= f.res[1]) continue;
          vis[(uint64_t)py * f.res[0] + px] = 0;
          cnt_add(&Counters::rays);
          if (heat) dbg[(uint64_t)py * f.res[0] + px] = 0;
        }
      march_list(sel);
      uint32_t hz = 0u;
      if (use_hiz) {
        // build_hiz: march.wgsl:57-76
        uint32_t m = 0xFFFFFFFFu;
        for (uint32_t ly = 0; ly < 8u; ++ly)
          for (uint32_t lx = 0; lx < 8u; ++lx) {
            uint32_t px = tx * 8u + lx, py = ty * 8u + ly;
            uint32_t d = 0u;
            if (px < f.res[0] && py < f.res[1]) d = (uint32_t)(vis[(uint64_t)py * f.res[0] + px] >> 40);
            m = std::min(m, d);
          }
        hz = m;
        // recover_select: tile_select.wgsl:94-110
        std::vector<uint32_t> rec;
        for (uint32_t ci : def) {
          const vm_chunk& c = chunk_at(w, ci);
          float dmin = box_distance(cam, ld3(c.aabb_min), ld3(c.aabb_max));
          if (depth_key(f, dmin) >= hz) rec.push_back(ci);
        }
        c_rec += rec.size();
        march_list(rec);
      }
      if (hiz_out) hiz_out[tile_id] = hz;
    }
    if (traffic) {
#pragma omp critical
      {
        total.chunk_records += local.chunk_records; total.l1_fetches += local.l1_fetches;
        total.leaf_fetches += local.leaf_fetches; total.attr_fetches += local.attr_fetches;
        total.palette_decodes += local.palette_decodes; total.grid_lookups += local.grid_lookups;
        total.iters += local.iters; total.march_calls += local.march_calls; total.rays += local.rays;
      }
    }
    t_cnt = nullptr;
  }
  if (counters) {
    uint32_t mp = f.max_pairs;
    counters[1] = (uint32_t)c_def;
    counters[2] = (uint32_t)c_rec;
    counters[4] = (uint32_t)c_sel;
    counters[3] = std::min<uint32_t>((uint32_t)c_sel, mp);
    counters[5] = (uint32_t)c_rec;
    counters[0] = use_hiz ? std::min<uint32_t>((uint32_t)c_rec, mp) : (uint32_t)c_sel;
  }
  if (traffic) {
    traffic->chunk_records = total.chunk_records; traffic->l1_fetches = total.l1_fetches;
    traffic->leaf_fetches = total.leaf_fetches; traffic->attr_fetches = total.attr_fetches;
    traffic->palette_decodes = total.palette_decodes; traffic->grid_lookups = total.grid_lookups;
    traffic->iters = total.iters; traffic->march_calls = total.march_calls; traffic->rays = total.rays;
  }
  return g_err.load();
}

// The per-tile pair list of tile_select for one tile (ascending chunk index),
// for tests of the culling itself.  Returns the number written (<= cap).
uint32_t or_tile_pairs(const or_world* o, uint32_t tile_id, const uint32_t* hiz_in, uint32_t* out,
                       uint32_t cap, uint32_t* deferred, uint32_t dcap, uint32_t* n_def) {
  World w = mk(o);
  const vm_frame& f = *w.f;
  TileCull tc = tile_planes(f, tile_id % f.tiles[0], tile_id / f.tiles[0]);
  V3 cam = ld3(f.cam_pos);
  const bool use_hiz = (f.flags & VM_FLAG_HIZ) != 0u;
  uint32_t tile_far = use_hiz && hiz_in ? hiz_in[tile_id] : 0u;
  uint32_t n = 0, nd = 0;
  for (uint32_t ci = 0; ci < f.chunk_count; ++ci) {
    const vm_chunk& c = chunk_at(w, ci);
    if (ci == f.camera_chunk) { if (n < cap) out[n] = ci; ++n; continue; }
    V3 bmin = ld3(c.aabb_min), bmax = ld3(c.aabb_max);
    if (box_outside(bmin, bmax, ld3(f.cam_fwd), cam)) continue;
    bool outb = false;
    for (int i = 0; i < 4 && !outb; ++i) outb = box_outside(bmin, bmax, tc.n[i], cam);
    if (outb) continue;
    float dmin = box_distance(cam, bmin, bmax);
    if (dmin >= tc.reach) continue;
    if (use_hiz && depth_key(f, dmin) < tile_far) { if (nd < dcap) deferred[nd] = ci; ++nd; continue; }
    if (n < cap) out[n] = ci;
    ++n;
  }
  if (n_def) *n_def = nd;
  return n;
}

// primary_shadow: shadow.wgsl:8-48 (per pixel blocker distance; 0 = lit).
int or_primary_shadow(const or_world* o, const uint64_t* vis, float* out, uint64_t pix_begin,
                      uint64_t pix_end, int threads, or_counters* traffic) {
  World w = mk(o);
  const vm_frame& f = *w.f;
  uint64_t npix = (uint64_t)f.res[0] * f.res[1];
  if (pix_end > npix) pix_end = npix;
  const bool active = (f.flags & VM_FLAG_SHADOWS) != 0u && (f.flags & VM_FLAG_HEATMAP) == 0u &&
                      f.daylight > 0.01f;
  V3 sun = ld3(f.sun_dir);
  V3 cam = ld3(f.cam_pos);
  Counters total{};
  if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel
  {
    Counters local{};
    t_cnt = traffic ? &local : nullptr;
#pragma omp for schedule(dynamic, 256)
    for (int64_t pi = (int64_t)pix_begin; pi < (int64_t)pix_end; ++pi) {
      uint64_t pix = (uint64_t)pi;
      float distance = 0.0f;
      if (active) {
        uint64_t key = vis[pix];
        if (key != 0ull) {
          uint32_t ci = key_ci(key);
          U3 v = key_voxel(key);
          uint32_t id = block_at(w, ci, v);
          if (!(id == VM_WATER || glass_leg(w, id))) {
            uint32_t nid = key_nid(key);
            U3 micro = key_micro(key);
            uint32_t px = (uint32_t)(pix % f.res[0]), py = (uint32_t)(pix / f.res[0]);
            V3 rd = ray_dir(f, (float)px + 0.5f, (float)py + 0.5f);
            V3 n = normal_of(nid);
            if (nid >= VM_NORMAL_CROSS_A && dot(n, rd) > 0.0f) n = neg(n);
            if (dot(n, sun) > 0.0f) {
              float t = hit_t(w, ci, v, micro, nid, rd);
              V3 hit = add(cam, muls(rd, t));
              float scale = chunk_at(w, ci).voxel_size;
              if (t >= 0.0f) {
                const V3 origin = add(hit, muls(n, 0.02f * scale));
                if ((w.spec & VM_SPEC_SOFT_RAYS) != 0u) {
                  uint32_t blocked = 0;
                  for (uint32_t s = 0; s < VM_SOFT_SAMPLES; ++s) {
                    cnt_add(&Counters::rays);
                    blocked += shadow_ray_t(w, origin, soft_sun_dir(f, px, py, s), f.shadow_dist) >= 0.0f ? 1u : 0u;
                  }
                  distance = (float)blocked * (1.0f / (float)VM_SOFT_SAMPLES);
                } else {
                  cnt_add(&Counters::rays); float blocker = shadow_ray_t(w, origin, sun, f.shadow_dist);
                  if (blocker >= 0.0f) distance = fminf(fmaxf(blocker, 0.001f), 65504.0f);
                }
              }
            }
          }
        }
      }
      out[pix] = distance;
    }
    if (traffic) {
#pragma omp critical
      {
        total.chunk_records += local.chunk_records; total.l1_fetches += local.l1_fetches;
        total.leaf_fetches += local.leaf_fetches; total.attr_fetches += local.attr_fetches;
        total.palette_decodes += local.palette_decodes; total.grid_lookups += local.grid_lookups;
        total.iters += local.iters; total.march_calls += local.march_calls; total.rays += local.rays;
      }
    }
    t_cnt = nullptr;
  }
  if (traffic) {
    traffic->chunk_records = total.chunk_records; traffic->l1_fetches = total.l1_fetches;
    traffic->leaf_fetches = total.leaf_fetches; traffic->attr_fetches = total.attr_fetches;
    traffic->palette_decodes = total.palette_decodes; traffic->grid_lookups = total.grid_lookups;
    traffic->iters = total.iters; traffic->march_calls = total.march_calls; traffic->rays = total.rays;
  }
  return g_err.load();
}

// One water-refraction or glass-transmission secondary ray per visible hit:
// water  -> water_refract_leg (resolve.wgsl:1029-1042), gated as water_sec /
//           water_compose gate it (FLAG_WATER_REFRACT, refract_detail > 0,
//           resolve.wgsl:1098,1524);
// glass  -> shade_glass's transmission trace (resolve.wgsl:1261-1280).
// sec_key: 0 = no secondary ray; else bit 63 = traced, bit 62 = hit, bit 61 =
// glass (else water), bits 37-39 normal, 24-36 chunk, 0-23 voxel (x<<16|y<<8|z).
// sec_t: hit distance along the secondary ray, or its max distance on a miss.
// The reflect leg of every water hit (water_sec resolve.wgsl:1526-1528,
// water_reflect_leg 1044-1058): FLAG_WATER_REFLECT, reflect_detail =
// 1 - smoothstep(512, 1024, t) > 0 (1099), from hit + n * SURFACE_EPS along
// reflect(rd, nt), trace_world(..., 768, skip_water) (880).  nt = n, the face
// normal, unless the surface is waved (FLAG_WAVES on a +Y face, 1107); waved
// pixels get no reflect ray here.  Key as or_secondary's (bit 61 clear).
}  // extern "C"

// ---- water_ctx's reflect direction: resolve.wgsl:902-975,1078-1166 ----
namespace {
const float WAVE_TAU = 6.28318531f, WAVE_GRAZE_MIN = 1e-3f, SHOAL_DEPTH = 6.0f, WAVE_FILTER_K = 1.0f;

// wave_octave: resolve.wgsl:928-942 (slope vector x, z and the variance)
V3 wave_octave(float x, float z, float dx, float dz, float lambda, float slope, float phase, float px, float vhx,
               float vhz, float kk, bool aniso) {
  float fade;
  if (aniso) {
    float d = dx * vhx + dz * vhz;
    float ext = px * sqrtf(1.0f + kk * d * d);
    float u = ext / lambda;
    fade = expf(-WAVE_FILTER_K * u * u);
  } else {
    fade = smoothstep(2.0f, 4.0f, lambda / fmaxf(px, 1e-4f));
  }
  float g = slope * fade * cosf(WAVE_TAU / lambda * (x * dx + z * dz) + phase);
  return v3(dx * g, dz * g, 0.5f * slope * slope * (1.0f - fade * fade));
}

// wave_field: resolve.wgsl:944-965
V3 wave_field(const vm_frame& f, float x, float z, float px, float vhx, float vhz, float kk, bool aniso, float shoal) {
  struct Oct { float dx, dz, div, amp, ph; };
  static const Oct fill[8] = {{-0.438371f, 0.898794f, 1.0f, 0.3086f, 1.0000f},
                              {-0.927184f, 0.374607f, 1.3934f, 0.2584f, 1.1804f},
                              {-0.190809f, 0.981627f, 1.9417f, 0.2163f, 1.3934f},
                              {-0.669131f, 0.743145f, 2.7056f, 0.1810f, 1.6449f},
                              {0.121869f, 0.992546f, 3.7700f, 0.1515f, 1.9417f},
                              {0.694658f, 0.719340f, 5.2533f, 0.1269f, 2.2920f},
                              {0.970296f, 0.241922f, 7.3201f, 0.1062f, 2.7056f},
                              {0.438371f, 0.898794f, 10.2000f, 0.0889f, 3.1937f}};
  static const Oct base[4] = {{0.913089f, 0.407760f, 1.0f, 0.42f, 1.0000f},
                              {-0.388685f, 0.921371f, 2.17f, 0.27f, 1.4731f},
                              {-0.980382f, -0.197108f, 4.71f, 0.19f, 2.1703f},
                              {0.477328f, -0.878725f, 10.20f, 0.12f, 3.1937f}};
  const bool full = (f.flags & VM_FLAG_WAVE_FILL) != 0u;
  const Oct* o = full ? fill : base;
  const int n = full ? 8 : 4;
  const float l0 = f.wave_scale, a = f.wave_amp * shoal, ph = f.time * f.wave_speed * WAVE_TAU;
  V3 s = v3(0.0f, 0.0f, 0.0f);
  for (int i = 0; i < n; ++i) {
    float lambda = i == 0 ? l0 : l0 / o[i].div;
    s = add(s, wave_octave(x, z, o[i].dx, o[i].dz, lambda, a * o[i].amp, ph * o[i].ph, px, vhx, vhz, kk, aniso));
  }
  return s;
}

// water_ctx's mirror_t (resolve.wgsl:1078-1163; SPEC_WATER_LOOK off)
V3 water_mirror_t(const World& w, uint32_t nid, V3 hit, V3 rd, float t) {
  const vm_frame& f = *w.f;
  const V3 n = normal_of(nid);
  V3 nt = n;
  float unresolved = 0.0f;
  const bool waved = (f.flags & VM_FLAG_WAVES) != 0u && nid == VM_NORMAL_PY;
  if (waved) {
    float px_world = fmaxf(t, 1e-3f) * 2.0f * f.tan_half_fov / (float)f.res[1];
    float kk = 0.0f, vhx = 0.0f, vhz = 0.0f;
    const bool aniso = (f.flags & VM_FLAG_WAVE_ANISO) != 0u;
    if (aniso) {
      float k = 1.0f / fmaxf(fabsf(rd.y), WAVE_GRAZE_MIN);
      kk = k * k - 1.0f;
      float r = 1.0f / sqrtf(fmaxf(rd.x * rd.x + rd.z * rd.z, 1e-12f));
      vhx = rd.x * r; vhz = rd.z * r;
    }
    float shoal = 1.0f;
    if ((f.flags & VM_FLAG_WAVE_SHOAL) != 0u) {
      V3 dro = v3(floorf(hit.x) + 0.5f, hit.y - VM_SURFACE_EPS, floorf(hit.z) + 0.5f);
      WorldHit dh = trace_world(w, dro, v3(0.001f, -0.999999f, 0.001f), SHOAL_DEPTH, true);
      shoal = smoothstep(0.0f, SHOAL_DEPTH, dh.hit ? dh.t : SHOAL_DEPTH);
    }
    V3 wf = wave_field(f, hit.x, hit.z, px_world, vhx, vhz, kk, aniso, shoal);
    unresolved = fmaxf(wf.z, 0.0f);
    float gl = sqrtf(wf.x * wf.x + wf.y * wf.y);
    float lim = fminf(1.0f, f.wave_reflect_slope / fmaxf(gl, 1e-6f));
    nt = normalize(v3(-(wf.x * lim), 1.0f, -(wf.y * lim)));
  }
  float rough = fminf(fmaxf(1.0f - expf(-8.0f * unresolved), 0.0f), 1.0f);
  nt = normalize(add(muls(nt, 1.0f - rough), muls(n, rough)));
  V3 m = reflect(rd, nt);
  if (waved) m = normalize(v3(m.x, fmaxf(m.y, 0.0f), m.z));
  return m;
}

uint64_t water_leg_key(const WorldHit& h) {
  uint64_t k = 1ull << 63;
  if (h.hit)
    k |= (1ull << 62) | ((uint64_t)h.normal << 37) | ((uint64_t)h.ci << 24) |
         (uint64_t)((h.voxel.x << 16u) | (h.voxel.y << 8u) | h.voxel.z);
  return k;
}
}  // namespace

extern "C" {

int or_reflect(const or_world* o, const uint64_t* vis, uint64_t* refl_key, float* refl_t, uint64_t pix_begin,
               uint64_t pix_end, int threads) {
  World w = mk(o);
  const vm_frame& f = *w.f;
  uint64_t npix = (uint64_t)f.res[0] * f.res[1];
  if (pix_end > npix) pix_end = npix;
  V3 cam = ld3(f.cam_pos);
  if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel for schedule(dynamic, 256)
  for (int64_t pi = (int64_t)pix_begin; pi < (int64_t)pix_end; ++pi) {
    uint64_t pix = (uint64_t)pi;
    uint64_t out_key = 0ull;
    float out_t = 0.0f;
    uint64_t key = vis[pix];
    if (key != 0ull && (f.flags & VM_FLAG_WATER_REFLECT) != 0u) {
      uint32_t ci = key_ci(key);
      U3 v = key_voxel(key);
      uint32_t nid = key_nid(key);
      if (block_at(w, ci, v) == VM_WATER) {
        U3 micro = key_micro(key);
        uint32_t px = (uint32_t)(pix % f.res[0]), py = (uint32_t)(pix / f.res[0]);
        V3 rd = ray_dir(f, (float)px + 0.5f, (float)py + 0.5f);
        float t = hit_t(w, ci, v, micro, nid, rd);
        float detail = 1.0f - smoothstep(VM_WATER_REFLECT_NEAR, VM_WATER_REFLECT_FAR, t);
        if (detail > 0.0f) {
          V3 hit = add(cam, muls(rd, t));
          V3 n = normal_of(nid);
          V3 ro3 = add(hit, muls(n, VM_SURFACE_EPS));
          WorldHit h3 = trace_world(w, ro3, water_mirror_t(w, nid, hit, rd, t), VM_WATER_REFLECT_DIST, true);
          out_key = water_leg_key(h3);
          out_t = h3.t;
        }
      }
    }
    refl_key[pix] = out_key;
    refl_t[pix] = out_t;
  }
  return g_err.load();
}

// water_sec: resolve.wgsl:1468-1535 (cells row-major, ceil(res / 2^shift))
int or_water_sec(const or_world* o, const uint64_t* vis, uint32_t shift, uint64_t* refr_key, float* refr_t,
                 uint64_t* refl_key, float* refl_t, int threads) {
  World w = mk(o);
  const vm_frame& f = *w.f;
  const uint32_t span = 1u << shift;
  const uint32_t hw = (f.res[0] + span - 1u) >> shift, hh = (f.res[1] + span - 1u) >> shift;
  const V3 cam = ld3(f.cam_pos);
  if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t c = 0; c < (int64_t)hw * hh; ++c) {
    const uint32_t hx = (uint32_t)(c % hw), hy = (uint32_t)(c / hw);
    float best_t = 3.4e38f;
    bool has = false;
    uint32_t bci = 0, bnid = 0, bpx = 0, bpy = 0;
    for (uint32_t i = 0; i < span; ++i)
      for (uint32_t j = 0; j < span; ++j) {
        const uint32_t pxs = span * hx + i, pys = span * hy + j;
        if (pxs >= f.res[0] || pys >= f.res[1]) continue;
        const uint64_t key = vis[(uint64_t)pys * f.res[0] + pxs];
        if (key == 0ull) continue;
        const uint32_t cis = key_ci(key), nids = key_nid(key);
        const U3 vs_ = key_voxel(key), micros = key_micro(key);
        if (block_at(w, cis, vs_) != VM_WATER) continue;
        const V3 rd0 = ray_dir(f, (float)pxs + 0.5f, (float)pys + 0.5f);
        const float ts = hit_t(w, cis, vs_, micros, nids, rd0);
        if (ts < best_t) { best_t = ts; bci = cis; bnid = nids; bpx = pxs; bpy = pys; has = true; }
      }
    (void)bci;
    uint64_t kr = 0ull, km = 0ull;
    float tr = 0.0f, tm = 0.0f;
    if (has) {
      const V3 rd = ray_dir(f, (float)bpx + 0.5f, (float)bpy + 0.5f);
      const V3 hit = add(cam, muls(rd, best_t));
      const V3 n = normal_of(bnid);
      if ((f.flags & VM_FLAG_WATER_REFRACT) != 0u &&
          1.0f - smoothstep(VM_WATER_REFRACT_NEAR, VM_WATER_REFRACT_FAR, best_t) > 0.0f) {
        const V3 rdir = refract(rd, n, 1.0f / VM_WATER_IOR);
        const WorldHit h2 = trace_world(w, add(hit, muls(rdir, VM_SURFACE_EPS)), rdir, VM_WATER_REFRACT_DIST, true);
        kr = water_leg_key(h2);
        tr = h2.t;
      }
      if ((f.flags & VM_FLAG_WATER_REFLECT) != 0u &&
          1.0f - smoothstep(VM_WATER_REFLECT_NEAR, VM_WATER_REFLECT_FAR, best_t) > 0.0f) {
        const WorldHit h3 = trace_world(w, add(hit, muls(n, VM_SURFACE_EPS)), water_mirror_t(w, bnid, hit, rd, best_t),
                                        VM_WATER_REFLECT_DIST, true);
        km = water_leg_key(h3);
        tm = h3.t;
      }
    }
    refr_key[c] = kr; refr_t[c] = tr;
    refl_key[c] = km; refl_t[c] = tm;
  }
  return g_err.load();
}

int or_secondary(const or_world* o, const uint64_t* vis, uint64_t* sec_key, float* sec_t,
                 uint64_t pix_begin, uint64_t pix_end, int threads) {
  World w = mk(o);
  const vm_frame& f = *w.f;
  uint64_t npix = (uint64_t)f.res[0] * f.res[1];
  if (pix_end > npix) pix_end = npix;
  V3 cam = ld3(f.cam_pos);
  const float inv_ior = 1.0f / VM_WATER_IOR;
  if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel for schedule(dynamic, 256)
  for (int64_t pi = (int64_t)pix_begin; pi < (int64_t)pix_end; ++pi) {
    uint64_t pix = (uint64_t)pi;
    uint64_t out_key = 0ull;
    float out_t = 0.0f;
    uint64_t key = vis[pix];
    if (key != 0ull) {
      uint32_t ci = key_ci(key);
      U3 v = key_voxel(key);
      uint32_t id = block_at(w, ci, v);
      bool water = id == VM_WATER, glass = glass_leg(w, id);
      if (water || glass) {
        uint32_t nid = key_nid(key);
        U3 micro = key_micro(key);
        uint32_t px = (uint32_t)(pix % f.res[0]), py = (uint32_t)(pix / f.res[0]);
        V3 rd = ray_dir(f, (float)px + 0.5f, (float)py + 0.5f);
        float t = hit_t(w, ci, v, micro, nid, rd);
        V3 hit = add(cam, muls(rd, t));
        bool traced = false;
        WorldHit h2{};
        if (water) {
          float detail = 1.0f - smoothstep(VM_WATER_REFRACT_NEAR, VM_WATER_REFRACT_FAR, t);
          if ((f.flags & VM_FLAG_WATER_REFRACT) != 0u && detail > 0.0f) {
            V3 rdir = refract(rd, normal_of(nid), inv_ior);
            V3 ro2 = add(hit, muls(rdir, VM_SURFACE_EPS));
            h2 = trace_world(w, ro2, rdir, VM_WATER_REFRACT_DIST, true);
            traced = true;
          }
        } else {
          V3 ro2 = add(hit, muls(rd, VM_SURFACE_EPS));
          h2 = trace_world(w, ro2, rd, fmaxf(VM_GLASS_TRANSMIT_DIST, f.far_), false);
          traced = true;
        }
        if (traced) {
          out_key = (1ull << 63) | (glass ? (1ull << 61) : 0ull);
          if (h2.hit) {
            out_key |= (1ull << 62) | ((uint64_t)h2.normal << 37) | ((uint64_t)h2.ci << 24) |
                       (uint64_t)((h2.voxel.x << 16u) | (h2.voxel.y << 8u) | h2.voxel.z);
          }
          out_t = h2.t;
        }
      }
    }
    sec_key[pix] = out_key;
    sec_t[pix] = out_t;
  }
  return g_err.load();
}

// Expanded visibility (voxel index, face, hit distance) from the raw keys:
// voxel index = X*(Z*y + z) + x over the world box [origin, origin+dims),
// face = the key's normal id, t = hit_t (common.wgsl:1300).  Misses give
// voxel 0xFFFFFFFF, face 0xFF, t 0.
int or_expand(const or_world* o, const uint64_t* vis, const int32_t* wmin, const uint32_t* wdim,
              uint32_t* voxel, uint8_t* face, float* tout, int threads) {
  World w = mk(o);
  const vm_frame& f = *w.f;
  uint64_t npix = (uint64_t)f.res[0] * f.res[1];
  if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel for schedule(static)
  for (int64_t pi = 0; pi < (int64_t)npix; ++pi) {
    uint64_t key = vis[pi];
    if (key == 0ull) { voxel[pi] = 0xFFFFFFFFu; face[pi] = 0xFF; tout[pi] = 0.0f; continue; }
    uint32_t ci = key_ci(key);
    U3 v = key_voxel(key);
    U3 micro = key_micro(key);
    uint32_t nid = key_nid(key);
    const vm_chunk& c = chunk_at(w, ci);
    int32_t vs = f2i(c.voxel_size);
    int32_t wx = f2i(c.origin[0]) + (int32_t)v.x * vs - wmin[0];
    int32_t wy = f2i(c.origin[1]) + (int32_t)v.y * vs - wmin[1];
    int32_t wz = f2i(c.origin[2]) + (int32_t)v.z * vs - wmin[2];
    voxel[pi] = (uint32_t)wx + wdim[0] * ((uint32_t)wz + wdim[2] * (uint32_t)wy);
    face[pi] = (uint8_t)nid;
    uint32_t px = (uint32_t)(pi % f.res[0]), py = (uint32_t)(pi / f.res[0]);
    V3 rd = ray_dir(f, (float)px + 0.5f, (float)py + 0.5f);
    tout[pi] = hit_t(w, ci, v, micro, nid, rd);
  }
  return g_err.load();
}

// Block lookup through the chunk grid (lod-0 chunks), for the unit DDA below.
static uint32_t grid_block(const World& w, int32_t x, int32_t y, int32_t z) {
  I3 cell{x >> 6, y >> 6, z >> 6};
  I3 rel = grid_rel(w, cell);
  if (grid_outside(w, rel)) return 0u;
  uint32_t ci = grid_at(w, grid_index(w, rel));
  if (ci == VM_NO_CHUNK) return 0u;
  const vm_chunk& c = chunk_at(w, ci);
  I3 v{x - f2i(c.origin[0]), y - f2i(c.origin[1]), z - f2i(c.origin[2])};
  if (!voxel_occupied(w, ci, v)) return 0u;
  return block_at(w, ci, U3{(uint32_t)v.x, (uint32_t)v.y, (uint32_t)v.z});
}

uint32_t or_grid_block(const or_world* o, int32_t x, int32_t y, int32_t z) {
  World w = mk(o);
  return grid_block(w, x, y, z);
}

// Unit-voxel Amanatides-Woo walk over block lookups, restating Player::pick
// (src/player.rs:334-393) with a caller-chosen step cap and reach.  A block
// counts as solid when its id is nonzero.  Returns 1 and the block / entry
// normal / distance on a hit.
int or_pick(const or_world* o, const float* orig, const float* dir, uint32_t max_steps, float reach,
            int32_t* block, int32_t* normal, float* dist) {
  World w = mk(o);
  V3 ro = ld3(orig), d = ld3(dir);
  I3 cell = floor_i(ro);
  I3 step{(int32_t)signf(d.x), (int32_t)signf(d.y), (int32_t)signf(d.z)};
  V3 inv{fabsf(1.0f / d.x), fabsf(1.0f / d.y), fabsf(1.0f / d.z)};
  V3 tmax{d.x > 0.0f ? ((float)cell.x + 1.0f - ro.x) * inv.x : (ro.x - (float)cell.x) * inv.x,
          d.y > 0.0f ? ((float)cell.y + 1.0f - ro.y) * inv.y : (ro.y - (float)cell.y) * inv.y,
          d.z > 0.0f ? ((float)cell.z + 1.0f - ro.z) * inv.z : (ro.z - (float)cell.z) * inv.z};
  I3 nrm{0, 0, 0};
  float t = 0.0f;
  for (uint32_t i = 0; i < max_steps; ++i) {
    if (grid_block(w, cell.x, cell.y, cell.z) != 0u) {
      block[0] = cell.x; block[1] = cell.y; block[2] = cell.z;
      normal[0] = nrm.x; normal[1] = nrm.y; normal[2] = nrm.z;
      *dist = t;
      return 1;
    }
    if (tmax.x < tmax.y && tmax.x < tmax.z) {
      t = tmax.x; tmax.x += inv.x; cell.x += step.x; nrm = {-step.x, 0, 0};
    } else if (tmax.y < tmax.z) {
      t = tmax.y; tmax.y += inv.y; cell.y += step.y; nrm = {0, -step.y, 0};
    } else {
      t = tmax.z; tmax.z += inv.z; cell.z += step.z; nrm = {0, 0, -step.z};
    }
    if (t > reach) break;
  }
  return 0;
}

// The engine's own CPU ray walk, Player::pick, as a frame tracer: one
// unit-voxel walk per pixel of rows [row0, row0 + rows) from the camera
// along ray_dir, up to max_steps voxels or the frame's far distance.
// Returns the pixels traced; *hits receives how many hit a block.
uint64_t or_pick_rows(const or_world* o, uint32_t row0, uint32_t rows, uint32_t max_steps, int threads,
                      uint64_t* hits) {
  World w = mk(o);
  const vm_frame& f = *w.f;
  const uint32_t W = f.res[0], H = f.res[1];
  const uint32_t y1 = std::min(H, row0 + rows);
  if (row0 >= y1) { *hits = 0; return 0; }
  uint64_t h = 0;
  if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : h)
  for (int64_t i = 0; i < (int64_t)(y1 - row0) * W; ++i) {
    const uint32_t px = (uint32_t)(i % W), py = row0 + (uint32_t)(i / W);
    const V3 d = ray_dir(f, (float)px + 0.5f, (float)py + 0.5f);
    const float dd[3] = {d.x, d.y, d.z};
    int32_t blk[3], nrm[3];
    float dist;
    h += (uint64_t)or_pick(o, f.cam_pos, dd, max_steps, f.far_, blk, nrm, &dist);
  }
  *hits = h;
  return (uint64_t)(y1 - row0) * W;
}

// shadow_horizontal + shadow_vertical (shadow.wgsl:62-116) with
// SPEC_SOFT_SHADOWS on: dist is primary_shadow's blocker distance per pixel
// (stored as r16float), h receives the horizontal pass (occlusion, support),
// stored as rg16float (2 floats per pixel; may be NULL), and mask the r8unorm
// target's value before quantisation, clamp(1 - occlusion, 0, 1).  limit =
// SHADOW_RADIUS_LIMIT, penumbra = SOFT_PENUMBRA.  shadow_guide is a pure
// function of the pixel, so it is evaluated once per pixel and looked up per
// tap.
int or_soften_shadows(const or_world* o, const uint64_t* vis, const float* dist, uint32_t limit, float penumbra,
                      float* h_out, float* mask, int threads) {
  World w = mk(o);
  const vm_frame& f = *w.f;
  const int32_t W = (int32_t)f.res[0], H = (int32_t)f.res[1];
  const uint64_t npix = (uint64_t)W * (uint64_t)H;
  const bool active = (f.flags & VM_FLAG_SHADOWS) != 0u && (f.flags & VM_FLAG_HEATMAP) == 0u && f.daylight > 0.01f;
  const int32_t L = (int32_t)limit;
  std::vector<Guide> g(npix);
  std::vector<float> d(npix), hx(npix), hy(npix);
  if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel for schedule(dynamic, 256)
  for (int64_t i = 0; i < (int64_t)npix; ++i) {
    g[i] = shadow_guide(w, vis, (int32_t)(i % W), (int32_t)(i / W));
    d[i] = f16_round(dist[i]);
  }
  auto guide = [&](int32_t x, int32_t y) -> Guide {
    if (x < 0 || y < 0 || x >= W || y >= H) { Guide z{}; z.valid = false; return z; }
    return g[(uint64_t)y * W + x];
  };
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t y = 0; y < H; ++y) {
    for (int32_t x = 0; x < W; ++x) {
      const uint64_t i = (uint64_t)y * W + x;
      const float occ = d[i] > 0.0f ? 1.0f : 0.0f;
      float rx = occ, ry = 0.0f;
      if (active && g[i].valid) {
        const Guide& c = g[i];
        const float rc = shadow_radius(f, d[i], c.t, penumbra, limit);
        float sum = occ, weight = 1.0f, support = rc;
        for (int32_t k = -L; k <= L; ++k) {
          if (k == 0) continue;
          const Guide q = guide(x + k, (int32_t)y);
          if (!shadow_compatible(c, q)) continue;
          const float nd = d[i + k];
          const float r = fmaxf(rc, shadow_radius(f, nd, q.t, penumbra, limit));
          if (r < fabsf((float)k)) continue;
          const float wk = expf(-2.0f * (float)(k * k) / fmaxf(r * r, 0.25f));
          sum += (nd > 0.0f ? 1.0f : 0.0f) * wk;
          weight += wk;
          support = fmaxf(support, r);
        }
        rx = sum / weight;
        ry = support;
      }
      hx[i] = f16_round(rx);
      hy[i] = f16_round(ry);
    }
  }
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t y = 0; y < H; ++y) {
    for (int32_t x = 0; x < W; ++x) {
      const uint64_t i = (uint64_t)y * W + x;
      float occ = hx[i];
      if (active && g[i].valid) {
        const Guide& c = g[i];
        float sum = hx[i], weight = 1.0f;
        for (int32_t k = -L; k <= L; ++k) {
          if (k == 0) continue;
          const Guide q = guide(x, (int32_t)y + k);
          if (!shadow_compatible(c, q)) continue;
          const uint64_t j = (uint64_t)((int32_t)y + k) * W + x;
          const float r = fmaxf(hy[i], hy[j]);
          if (r < fabsf((float)k)) continue;
          const float wk = expf(-2.0f * (float)(k * k) / fmaxf(r * r, 0.25f));
          sum += hx[j] * wk;
          weight += wk;
        }
        occ = sum / weight;
      }
      mask[i] = fminf(fmaxf(1.0f - occ, 0.0f), 1.0f);
      if (h_out) { h_out[2 * i] = hx[i]; h_out[2 * i + 1] = hy[i]; }
    }
  }
  return g_err.load();
}

void or_f16_round(const float* x, float* out, uint64_t n) {
  for (uint64_t i = 0; i < n; ++i) out[i] = f16_round(x[i]);
}

}  // extern "C"


// ============================================================================
// The resolve of sky and opaque surfaces: lane 0 of resolve.wgsl:1378-1466,
// shade_hit_legacy_cached (resolve.wgsl:1537-1788), sky_color and the sun
// shafts (common.wgsl:1332-1643).  Texture reads are restated from the
// sampler equations (the engine's atlas sampler: mag nearest, min / mipmap
// linear, clamp to edge; the probe sampler: linear, repeat in u and w, clamp
// in v) on the atlas decoded to linear float by the sRGB transfer function.
// ============================================================================
namespace {

struct Look {
  const float* atlas; uint32_t layers;    // linear RGBA floats, mips 16, 8, 4, 2, each [layer][y][x][4]
  const uint32_t* faces; uint32_t n_faces;
  const uint16_t* probes;                 // RGBA16F 128 x 768 x 128, or null (1.0)
  const float* shaft;                     // 512 x 512 envelope, or null
  uint32_t spec_hi;
  float grad_cos[32], grad_sin[32];
};

constexpr uint32_t HI_SKY_SPECULAR = 1u, HI_SHORE_WET = 8u, HI_CAUSTICS = 64u, HI_TINT_BALANCE = 512u,
                   HI_SKY_LOOK = 1024u, HI_SKY_COOL = 2048u, HI_FOLIAGE_RICH = 8192u, HI_CANOPY_RELIEF = 16384u,
                   HI_LEGACY_LIGHTING = 1048576u;

inline float mixs(float a, float b, float t) { return a * (1.0f - t) + b * t; }
inline V3 mixv(V3 a, V3 b, float t) { return {mixs(a.x, b.x, t), mixs(a.y, b.y, t), mixs(a.z, b.z, t)}; }
inline float clampf(float x, float lo, float hi) { return fminf(fmaxf(x, lo), hi); }
inline bool cool(const Look& L) { return (L.spec_hi & HI_SKY_COOL) != 0u; }
inline bool repair(const Look& L) { return (L.spec_hi & HI_LEGACY_LIGHTING) == 0u; }
// SURFACE_DEBUG = (spec_hi >> 23) & 7 (FLAG_HI_DEBUG_A..C, mod.rs make_spec)
inline uint32_t surface_debug(const Look& L) { return (L.spec_hi >> 23) & 7u; }
const V3 SCATTER_TINT = {1.0000f, 0.4770f, 0.1474f};

// transmittance_from: common.wgsl:1332-1341
float transmittance_from(const vm_frame& f, float y0, float s, V3 rd) {
  float lambda = f.fog_falloff;
  float x = clampf(lambda * s * rd.y, -60.0f, 60.0f);
  float path = s;
  if (fabsf(x) > 1e-4f) path = s * (1.0f - expf(-x)) / x;
  float rho = f.fog_density * expf(-clampf(lambda * (y0 - f.fog_height), -60.0f, 60.0f));
  return expf(-clampf(rho * path, 0.0f, 60.0f));
}

// hg_gain / scatter_lobe / sky_base: common.wgsl:1359-1395
float hg_gain(float cos_t, float g) {
  float g2 = g * g;
  float d = 1.0f + g2 - 2.0f * g * cos_t;
  return (1.0f - g2) / powf(fmaxf(d, 1e-4f), 1.5f);
}
V3 scatter_lobe(const vm_frame& f, V3 rd) {
  float sd = dot(rd, ld3(f.sun_dir));
  return muls(SCATTER_TINT, hg_gain(sd, f.fog_g) * f.fog_scatter * f.daylight);
}
V3 sky_base(const vm_frame& f, const Look& L, V3 rd, float shaft) {
  float day = f.daylight;
  float up = clampf(rd.y, 0.0f, 1.0f);
  V3 horizon = mixv(v3(0.0049f, 0.0060f, 0.0134f), cool(L) ? v3(0.4074f, 0.6057f, 0.9150f) : v3(0.4480f, 0.6210f, 0.8900f), day);
  V3 zenith = mixv(v3(0.0008f, 0.0015f, 0.0039f), cool(L) ? v3(0.0385f, 0.1892f, 0.8600f) : v3(0.0637f, 0.2140f, 0.8276f), day);
  V3 c = mixv(horizon, zenith, powf(up, 0.55f));
  float sd = dot(rd, ld3(f.sun_dir));
  c = add(c, muls(muls(v3(1.0f, 0.8276f, 0.5225f), smoothstep(0.9975f, 0.9990f, sd)), fmaxf(day, 0.2f)));
  c = add(c, muls(scatter_lobe(f, rd), shaft));
  bool look = (L.spec_hi & HI_SKY_LOOK) != 0u;
  if (look && f.haze_warm > 0.0f) {
    float band = powf(1.0f - up, 3.0f);
    float toward = 0.35f + 0.65f * powf(fmaxf(sd, 0.0f), 4.0f);
    c = add(c, muls(SCATTER_TINT, band * toward * f.haze_warm * day * 0.22f));
  }
  if (look && f.zenith_deep > 0.0f) {
    float z = powf(up, 0.55f);
    c = mul(c, mixv(v3(1.0f, 1.0f, 1.0f), v3(0.80f, 0.90f, 1.16f), f.zenith_deep * z * day));
  }
  return mixv(c, muls(horizon, 0.26f), smoothstep(0.0f, -0.35f, rd.y));
}

// cloud_lattice / cloud_noise / cloud_fbm: common.wgsl:1432-1468
float cloud_lattice(int32_t x, int32_t y) {
  uint32_t h = hash_u32((uint32_t)x ^ (hash_u32((uint32_t)y) * 0x9e3779b9u));
  return (float)(h >> 8u) * (1.0f / 16777216.0f);
}
float cloud_noise(float px, float py) {
  float ix = floorf(px), iy = floorf(py);
  float fx = px - ix, fy = py - iy;
  float wx = fx * fx * fx * (fx * (fx * 6.0f - 15.0f) + 10.0f);
  float wy = fy * fy * fy * (fy * (fy * 6.0f - 15.0f) + 10.0f);
  int32_t cx = f2i(ix), cy = f2i(iy);
  int32_t cx1 = (int32_t)((uint32_t)cx + 1u), cy1 = (int32_t)((uint32_t)cy + 1u);
  float a = cloud_lattice(cx, cy), b = cloud_lattice(cx1, cy), d = cloud_lattice(cx, cy1), e = cloud_lattice(cx1, cy1);
  return mixs(mixs(a, b, wx), mixs(d, e, wx), wy);
}
float cloud_fbm(float px, float py, float fp) {
  float freq = 1.0f, amp = 1.0f, sum = 0.0f, norm = 0.0f;
  for (uint32_t i = 0; i < 4u; ++i) {
    float wgt = amp * (1.0f - smoothstep(0.25f, 0.5f, fp * freq));
    if (wgt > 0.0f) {
      sum += wgt * cloud_noise(px * freq, py * freq);
      norm += wgt;
    }
    freq *= 2.0f;
    amp *= 0.5f;
  }
  if (norm <= 0.0f) return 0.5f;
  return sum / norm;
}

// cloud_shade: common.wgsl:1537-1555
float cloud_shade(const vm_frame& f, V3 p, float fp) {
  if (f.cloud_shadow <= 0.0f || f.cloud_cover <= 0.0f) return 1.0f;
  float dy = f.cloud_height - p.y;
  if (dy * f.sun_dir[1] <= 0.0f) return 1.0f;
  float t = dy / f.sun_dir[1];
  if (t > 1.0e5f) return 1.0f;
  float qx = p.x + f.sun_dir[0] * t, qz = p.z + f.sun_dir[2] * t;
  float drift = f.time * f.cloud_speed;
  float dx = 0.94f * drift, dz = 0.34f * drift;
  float n = cloud_fbm((qx + dx) / f.cloud_scale, (qz + dz) / f.cloud_scale, fmaxf(fp, t * 0.0093f) / f.cloud_scale);
  float thr = 1.0f - f.cloud_cover;
  return 1.0f - smoothstep(thr, thr + 0.14f, n) * f.cloud_shadow;
}

// cloud_radiance / sky_color: common.wgsl:1470-1530
V3 cloud_radiance(const vm_frame& f, const Look& L, float dens, float depth, V3 rd) {
  float day = f.daylight;
  float thick = rd.y < 0.0f ? 0.0f : depth;
  float warm = 1.0f - smoothstep(0.02f, 0.30f, f.sun_dir[1]);
  V3 sun_tint = mixv(v3(1.0f, 1.0f, 1.0f), SCATTER_TINT, warm * 0.72f);
  V3 lit = cool(L) ? v3(1.0f, 1.0f, 1.0f) : v3(1.0000f, 0.9575f, 0.8963f);
  V3 base = cool(L) ? v3(0.4420f, 0.4880f, 0.6010f) : v3(0.4854f, 0.5312f, 0.6462f);
  V3 day_c = mixv(mul(lit, sun_tint), base, thick);
  V3 glow = muls(SCATTER_TINT, hg_gain(dot(rd, ld3(f.sun_dir)), 0.82f) * 0.055f * day * (1.0f - dens));
  return add(mixv(v3(0.0021f, 0.0026f, 0.0052f), day_c, day), glow);
}
V3 sky_color(const vm_frame& f, const Look& L, V3 ro, V3 rd, float travelled, float shaft) {
  V3 base = sky_base(f, L, rd, shaft);
  if (f.cloud_cover <= 0.0f) return base;
  float dy = f.cloud_height - ro.y;
  if (dy * rd.y <= 0.0f) return base;
  float t = dy / rd.y;
  if (t > 1.0e5f) return base;
  float px = ro.x + rd.x * t, pz = ro.z + rd.z * t;
  float px_angle = 2.0f * f.tan_half_fov / (float)f.res[1] * exp2f(f.mip_bias);
  float fp = (travelled + t) * px_angle / (fabsf(rd.y) * f.cloud_scale);
  float drift = f.time * f.cloud_speed;
  float qx = px + 0.94f * drift, qz = pz + 0.34f * drift;
  float n = cloud_fbm(qx / f.cloud_scale, qz / f.cloud_scale, fp);
  float thr = 1.0f - f.cloud_cover;
  bool look = (L.spec_hi & HI_SKY_LOOK) != 0u;
  if (look && f.cloud_patch > 0.0f) {
    float m = cloud_fbm(qx / (f.cloud_scale * 6.0f), qz / (f.cloud_scale * 6.0f), fp / 6.0f);
    thr = clampf(thr + (m - 0.5f) * f.cloud_patch, 0.0f, 0.99f);
  }
  float dens = smoothstep(thr, thr + 0.14f, n);
  if (dens <= 0.0f) return base;
  float depth = smoothstep(thr, thr + 0.55f, n);
  if (look && f.cloud_relief > 0.0f) {
    float ax = f.sun_dir[0] + 1.0e-3f, az = f.sun_dir[2];
    float l = sqrtf(ax * ax + az * az);
    ax = ax / l; az = az / l;
    float step = (8.0f + f.sun_dir[1] * 48.0f) / f.cloud_scale;
    float ns = cloud_fbm(qx / f.cloud_scale + ax * step, qz / f.cloud_scale + az * step, fp);
    depth = clampf(depth + (ns - n) * (2.2f * f.cloud_relief), 0.0f, 1.0f);
  }
  float reach = 1.0f - smoothstep(3.0e4f, 1.0e5f, t);
  float a = dens * reach * transmittance_from(f, ro.y, t, rd);
  return mixv(base, cloud_radiance(f, L, dens, depth, rd), a);
}

// shaft_sample / terrain_shade: common.wgsl:1557-1580
float terrain_shade(const vm_frame& f, const Look& L, V3 p) {
  if (!L.shaft) return 1.0f;
  float tx = (p.x - f.shaft_origin[0]) / f.shaft_texel - 0.5f;
  float tz = (p.z - f.shaft_origin[1]) / f.shaft_texel - 0.5f;
  float hi = (float)VM_SHAFT_DIM - 1.0f;
  float cx = clampf(tx, 0.0f, hi), cz = clampf(tz, 0.0f, hi);
  float f0x = floorf(cx), f0z = floorf(cz);
  float frx = cx - f0x, frz = cz - f0z;
  uint32_t i0x = f2u(f0x), i0z = f2u(f0z);
  uint32_t i1x = std::min(i0x + 1u, VM_SHAFT_DIM - 1u), i1z = std::min(i0z + 1u, VM_SHAFT_DIM - 1u);
  auto at = [&](uint32_t x, uint32_t z) { return L.shaft[(uint64_t)z * VM_SHAFT_DIM + x]; };
  float e = mixs(mixs(at(i0x, i0z), at(i1x, i0z), frx), mixs(at(i0x, i1z), at(i1x, i1z), frx), frz);
  return smoothstep(e - f.shaft_soft, e + f.shaft_soft, p.y);
}

float dither_px(const vm_frame& f, uint32_t px, uint32_t py) {
  float p0 = (float)px + 5.588238f * (float)f.frame_index, p1 = (float)py;
  return fractf(52.9829189f * fractf(p0 * 0.06711056f + p1 * 0.00583715f));
}

// sun_shaft: common.wgsl:1582-1643
float sun_shaft(const vm_frame& f, const Look& L, V3 ro, V3 rd, float dist, float alpha, uint32_t px, uint32_t py) {
  bool terrain = (f.flags & VM_FLAG_TERRAIN_SHAFTS) != 0u;
  bool deck = f.cloud_shadow > 0.0f && f.cloud_cover > 0.0f;
  if (f.godray_strength <= 0.0f) return 1.0f;
  if (!deck && !terrain) return 1.0f;
  V3 lobe = scatter_lobe(f, rd);
  float imp = smoothstep(0.0040f, 0.0120f, fmaxf(fmaxf(lobe.x, lobe.y), lobe.z) * alpha);
  if (imp <= 0.0f) return 1.0f;
  float d = fminf(dist, f.godray_dist);
  if (d <= 0.0f) return 1.0f;
  float opac = 1.0f - transmittance_from(f, ro.y, d, rd);
  if (opac <= 1e-6f) return 1.0f;
  float lambda = f.fog_falloff;
  float rho0 = f.fog_density * expf(-clampf(lambda * (ro.y - f.fog_height), -60.0f, 60.0f));
  float k = lambda * rd.y;
  float off = dither_px(f, px, py);
  float px_angle = 2.0f * f.tan_half_fov / (float)f.res[1] * exp2f(f.mip_bias);
  float sum = 0.0f;
  for (uint32_t i = 0; i < f.godray_steps; ++i) {
    float u = ((float)i + off) / (float)f.godray_steps;
    float path = -logf(1.0f - u * opac) / rho0;
    float s = path;
    float kp = k * path;
    if (fabsf(kp) > 1e-4f) s = -logf(fmaxf(1.0f - kp, 1e-6f)) / k;
    s = clampf(s, 0.0f, d);
    V3 p = add(ro, muls(rd, s));
    float v = cloud_shade(f, p, s * px_angle);
    if (terrain) v = v * terrain_shade(f, L, p);
    sum += v;
  }
  float vis = sum / (float)f.godray_steps;
  float covered = 1.0f;
  if (d < dist) {
    float full = 1.0f - transmittance_from(f, ro.y, dist, rd);
    if (full > 1e-6f) covered = fminf(opac / full, 1.0f);
  }
  return fmaxf(mixs(1.0f, vis, imp * f.godray_strength * covered), 0.0f);
}

// light_at / voxel_occludes / world_sample / gather_face: common.wgsl:977-1096
uint32_t light_at(const World& w, uint32_t ci, I3 v) {
  const vm_chunk& c = chunk_at(w, ci);
  if ((c.light_flags & 1u) != 0u) return c.light_base;
  if (v.x < 0 || v.y < 0 || v.z < 0 || v.x > 63 || v.y > 63 || v.z > 63) return 0xF000u;
  U3 uv{(uint32_t)v.x, (uint32_t)v.y, (uint32_t)v.z};
  uint32_t cell = (uv.x >> 2u) | ((uv.y >> 2u) << 4u) | ((uv.z >> 2u) << 8u);
  uint32_t entry = brick_at(w, (uint64_t)c.light_base + cell);
  if ((entry & VM_UNIFORM_BIT) != 0u) return entry & 0xFFFFu;
  uint32_t vb = cell_bit(uand(uv, 3u));
  uint32_t word = brick_at(w, (uint64_t)entry + (vb >> 1u));
  return (word >> ((vb & 1u) * 16u)) & 0xFFFFu;
}
bool voxel_occludes(const World& w, uint32_t ci, I3 v) {
  bool occupied = voxel_occupied(w, ci, v);
  const vm_chunk& c = chunk_at(w, ci);
  if (occupied && (c.attr_flags & (VM_ATTR_HAS_WATER | VM_ATTR_HAS_FOLIAGE)) != 0u) {
    uint32_t b = block_at(w, ci, U3{(uint32_t)v.x, (uint32_t)v.y, (uint32_t)v.z});
    return b != VM_WATER && !is_tuft(b);
  }
  return occupied;
}
U2 world_sample(const World& w, V3 p) {
  I3 cell = grid_rel(w, floor_i(divs(p, 64.0f)));
  if (grid_outside(w, cell)) return U2{0xF000u, 0u};
  uint32_t ci = grid_at(w, grid_index(w, cell));
  if (ci == VM_NO_CHUNK) return U2{0xF000u, 0u};
  const vm_chunk& c = chunk_at(w, ci);
  I3 v = floor_i(divs(sub(p, ld3(c.origin)), c.voxel_size));
  return U2{light_at(w, ci, v), voxel_occludes(w, ci, v) ? 1u : 0u};
}
void gather_face(const World& w, uint32_t ci, I3 base, I3 ta, I3 tb, U2* out) {
  const vm_chunk& c = chunk_at(w, ci);
  bool has_water = (c.attr_flags & VM_ATTR_HAS_WATER) != 0u;
  for (uint32_t i = 0; i < 9u; ++i) {
    int32_t a = (int32_t)(i % 3u) - 1, b = (int32_t)(i / 3u) - 1;
    I3 uv{base.x + ta.x * a + tb.x * b, base.y + ta.y * a + tb.y * b, base.z + ta.z * a + tb.z * b};
    bool solid = voxel_occupied(w, ci, uv);
    if (solid && has_water) solid = block_at(w, ci, U3{(uint32_t)uv.x, (uint32_t)uv.y, (uint32_t)uv.z}) != VM_WATER;
    out[i] = U2{light_at(w, ci, uv), solid ? 1u : 0u};
  }
}

float light_sky(uint32_t p) { return (float)(p >> 12u); }
V3 light_block_rgb(uint32_t p) { return v3((float)((p >> 8u) & 0xFu), (float)((p >> 4u) & 0xFu), (float)(p & 0xFu)); }
float light_block_level(uint32_t p) { V3 c = light_block_rgb(p); return fmaxf(c.x, fmaxf(c.y, c.z)); }
float light_curve(float level) { float l = level / 15.0f; return l * l * (0.6f + 0.4f * l); }
V3 light_curve3(V3 level) {
  V3 l = divs(level, 15.0f);
  return mul(mul(l, l), v3(0.6f + 0.4f * l.x, 0.6f + 0.4f * l.y, 0.6f + 0.4f * l.z));
}
V3 block_ambient(V3 blk, float sk, V3 sky) {
  float bk = fmaxf(blk.x, fmaxf(blk.y, blk.z));
  V3 tint = divs(blk, fmaxf(bk, 1e-4f));
  return muls(mixv(sky, tint, bk / fmaxf(sk + bk, 1e-4f)), fmaxf(sk, bk));
}
const V3 BLOCK_TINT = {1.0000f, 0.6500f, 0.3200f};

// sky_ambient_tint / surface_sky_fill: resolve.wgsl:1-5, 73-89
V3 sky_ambient_tint(const vm_frame& f, V3 n) {
  const V3 sky_tint = {0.6038f, 0.7084f, 1.0000f};
  if ((f.flags & VM_FLAG_SKY_TINT) == 0u) return sky_tint;
  float day = f.daylight;
  V3 horizon = mixv(v3(0.0049f, 0.0060f, 0.0134f), v3(0.4480f, 0.6210f, 0.8900f), day);
  V3 zenith = mixv(v3(0.0008f, 0.0015f, 0.0039f), v3(0.0637f, 0.2140f, 0.8276f), day);
  float wgt = n.y < -0.5f ? 0.0f : (n.y > 0.5f ? 0.78431373f : 0.58578900f);
  V3 c = mixv(horizon, zenith, wgt);
  c = add(c, muls(SCATTER_TINT, f.fog_scatter * day * 4.0f * fmaxf(dot(n, ld3(f.sun_dir)), 0.0f)));
  V3 t = mul(sky_tint, v3(powf(c.x / 0.14658824f, 2.5f), powf(c.y / 0.30178431f, 2.5f), powf(c.z / 0.84105882f, 2.5f)));
  float luma = 0.2126f * t.x + 0.7152f * t.y + 0.0722f * t.z;
  return muls(t, 0.70721556f / fmaxf(luma, 1e-6f));
}
V3 surface_sky_fill(const vm_frame& f, const Look& L, V3 n) {
  V3 sky = sky_ambient_tint(f, n);
  if (!repair(L)) return sky;
  return muls(sky, 0.60f * mixs(0.35f, 1.0f, clampf(n.y * 0.5f + 0.5f, 0.0f, 1.0f)));
}

// textureSampleLevel on the atlas: bilinear taps with clamp to edge, nearest
// texel when the level magnifies (level <= 0), linear blend of two mips
struct F4 { float r, g, b, a; };
inline F4 mix4(F4 x, F4 y, float t) { return {mixs(x.r, y.r, t), mixs(x.g, y.g, t), mixs(x.b, y.b, t), mixs(x.a, y.a, t)}; }
F4 atlas_texel(const Look& L, uint32_t mip, uint32_t layer, int32_t x, int32_t y) {
  uint64_t base = 0;
  for (uint32_t m = 0; m < mip; ++m) base += (uint64_t)L.layers * (16u >> m) * (16u >> m);
  int32_t size = (int32_t)(16u >> mip);
  x = std::min(std::max(x, 0), size - 1);
  y = std::min(std::max(y, 0), size - 1);
  const float* p = L.atlas + 4 * (base + ((uint64_t)layer * size + y) * size + x);
  return {p[0], p[1], p[2], p[3]};
}
F4 atlas_bilinear(const Look& L, uint32_t mip, uint32_t layer, float u, float v) {
  float size = (float)(16u >> mip);
  float x = u * size - 0.5f, y = v * size - 0.5f;
  float x0 = floorf(x), y0 = floorf(y);
  float ax = x - x0, ay = y - y0;
  int32_t ix = f2i(x0), iy = f2i(y0);
  int32_t ix1 = (int32_t)((uint32_t)ix + 1u), iy1 = (int32_t)((uint32_t)iy + 1u);
  return mix4(mix4(atlas_texel(L, mip, layer, ix, iy), atlas_texel(L, mip, layer, ix1, iy), ax),
              mix4(atlas_texel(L, mip, layer, ix, iy1), atlas_texel(L, mip, layer, ix1, iy1), ax), ay);
}
F4 atlas_sample(const Look& L, float u, float v, uint32_t layer, float lod) {
  if (layer >= L.layers) layer = L.layers - 1u;
  if (!(lod > 0.0f)) return atlas_texel(L, 0, layer, f2i(floorf(u * 16.0f)), f2i(floorf(v * 16.0f)));
  float d = fminf(lod, 3.0f);
  float dl = floorf(d);
  float delta = d - dl;
  uint32_t m0 = f2u(dl);
  F4 a = atlas_bilinear(L, m0, layer, u, v);
  if (!(delta > 0.0f) || m0 + 1u >= 4u) return a;
  return mix4(a, atlas_bilinear(L, m0 + 1u, layer, u, v), delta);
}

float half_to_float(uint16_t h) {
  uint32_t sign = (uint32_t)(h >> 15) << 31, e = (h >> 10) & 0x1Fu, m = h & 0x3FFu, bits;
  if (e == 0) {
    if (m == 0) { bits = sign; }
    else {   // subnormal: normalise
      int32_t ex = -1;
      do { m <<= 1; ++ex; } while ((m & 0x400u) == 0);
      bits = sign | ((uint32_t)(127 - 15 - ex) << 23) | ((m & 0x3FFu) << 13);
    }
  } else if (e == 31) {
    bits = sign | 0x7F800000u | (m << 13);
  } else {
    bits = sign | ((e - 15 + 127) << 23) | (m << 13);
  }
  float out;
  memcpy(&out, &bits, 4);
  return out;
}
F4 probe_texel(const Look& L, int32_t x, int32_t y, int32_t z) {
  x = ((x % 128) + 128) % 128;
  z = ((z % 128) + 128) % 128;
  y = std::min(std::max(y, 0), 767);
  const uint16_t* p = L.probes + 4 * (((uint64_t)z * 768 + y) * 128 + x);
  return {half_to_float(p[0]), half_to_float(p[1]), half_to_float(p[2]), half_to_float(p[3])};
}
// probe_field: resolve.wgsl:106-118
F4 probe_field(const Look& L, V3 p, uint32_t nid) {
  if (!L.probes) return {1.0f, 1.0f, 1.0f, 1.0f};
  uint32_t slab = nid >= VM_NORMAL_CROSS_A ? 3u : nid;
  V3 t = muls(p, 1.0f / 4.0f);
  float y = clampf(t.y, 0.5f, 128.0f - 0.5f);
  float u = t.x * (1.0f / 128.0f), v = ((float)slab * 128.0f + y) * (1.0f / (128.0f * 6.0f)), wz = t.z * (1.0f / 128.0f);
  float x = u * 128.0f - 0.5f, yy = v * 768.0f - 0.5f, z = wz * 128.0f - 0.5f;
  float x0 = floorf(x), y0 = floorf(yy), z0 = floorf(z);
  float ax = x - x0, ay = yy - y0, az = z - z0;
  int32_t ix = f2i(x0), iy = f2i(y0), iz = f2i(z0);
  F4 s[2];
  for (int dz = 0; dz < 2; ++dz) {
    F4 a = mix4(probe_texel(L, ix, iy, iz + dz), probe_texel(L, ix + 1, iy, iz + dz), ax);
    F4 b = mix4(probe_texel(L, ix, iy + 1, iz + dz), probe_texel(L, ix + 1, iy + 1, iz + dz), ax);
    s[dz] = mix4(a, b, ay);
  }
  return mix4(s[0], s[1], az);
}

// probe_tap: resolve.wgsl:120-127 (PROBE_TAPS = 1): the probe texture
// through the engine's linear sampler (mod.rs:1070-1077: linear filtering,
// clamp to edge on every axis) at fract(p / (PROBE_DIM * PROBE_SPACING))
F4 probe_texel_clamped(const Look& L, int32_t x, int32_t y, int32_t z) {
  return probe_texel(L, std::min(std::max(x, 0), 127), y, std::min(std::max(z, 0), 127));
}
V3 probe_tap(const Look& L, V3 p) {
  if (!L.probes) return v3(1.0f, 1.0f, 1.0f);
  const float inv_span = 1.0f / (128.0f * 4.0f);
  auto fract = [](float x) { return x - floorf(x); };
  float u = fract(p.x * inv_span), v = fract(p.y * inv_span), wz = fract(p.z * inv_span + 0.0f);
  float x = u * 128.0f - 0.5f, yy = v * 768.0f - 0.5f, z = wz * 128.0f - 0.5f;
  float x0 = floorf(x), y0 = floorf(yy), z0 = floorf(z);
  float ax = x - x0, ay = yy - y0, az = z - z0;
  int32_t ix = f2i(x0), iy = f2i(y0), iz = f2i(z0);
  F4 s[2];
  for (int dz = 0; dz < 2; ++dz) {
    F4 a = mix4(probe_texel_clamped(L, ix, iy, iz + dz), probe_texel_clamped(L, ix + 1, iy, iz + dz), ax);
    F4 b = mix4(probe_texel_clamped(L, ix, iy + 1, iz + dz), probe_texel_clamped(L, ix + 1, iy + 1, iz + dz), ax);
    s[dz] = mix4(a, b, ay);
  }
  F4 r = mix4(s[0], s[1], az);
  return mul(v3(1.0f, 1.0f, 1.0f), v3(r.r, r.g, r.b));
}

// face_uv / perm_key / permute_uv: resolve.wgsl:129-164
void face_uv(uint32_t nid, V3 local, float& u, float& v) {
  if (nid >= VM_NORMAL_CROSS_A) { u = local.x; v = 1.0f - local.y; return; }
  uint32_t axis = nid >> 1u;
  if (axis == 0u) { u = local.z; v = 1.0f - local.y; }
  else if (axis == 1u) { u = local.x; v = local.z; }
  else { u = local.x; v = 1.0f - local.y; }
  if (nid == 1u || nid == 4u) u = 1.0f - u;
}
uint32_t perm_key(V3 box_min, uint32_t nid) {
  I3 c = floor_i(box_min);
  return hash_u32(((uint32_t)c.x * 0x9e3779b9u) ^ ((uint32_t)c.y * 0x85ebca6bu) ^ ((uint32_t)c.z * 0xc2b2ae35u) ^
                  (nid * 0x27d4eb2fu));
}
void permute_uv(float& u, float& v, uint32_t pclass, uint32_t h) {
  bool d4 = pclass == 2u;
  float px = u, py = v;
  if (d4 && (h & 1u) != 0u) { px = v; py = u; }
  if (pclass != 0u && (h & 2u) != 0u) px = 1.0f - px;
  if (d4 && (h & 4u) != 0u) py = 1.0f - py;
  u = px; v = py;
}
// hash_alpha: common.wgsl:400-406
float hash_alpha(V3 p) {
  I3 q = floor_i(muls(p, 64.0f));
  uint32_t h = ((uint32_t)q.x * 73856093u) ^ ((uint32_t)q.y * 19349663u) ^ ((uint32_t)q.z * 83492791u);
  h = h ^ (h >> 13u);
  h = h * 1274126177u;
  return (float)((h >> 8u) & 0xFFFFFFu) / 16777216.0f;
}

// simplex_grad / biome_noise / biome_band_weights / biome_tint: resolve.wgsl:180-285
float simplex_grad(const Look& L, uint32_t seed, uint32_t xp, uint32_t yp, float xd, float yd) {
  uint32_t h = (seed ^ xp ^ yp) * 0x27d4eb2du;
  int32_t hs = (int32_t)h;
  uint32_t idx = (uint32_t)((hs ^ (hs >> 15)) & 254);
  uint32_t k = idx < 240u ? (idx % 48u) >> 1u : 24u + ((idx - 240u) >> 1u);
  return xd * L.grad_cos[k] + yd * L.grad_sin[k];
}
int32_t biome_fast_floor(float f) { return f >= 0.0f ? f2i(f) : f2i(f) - 1; }
float biome_noise(const Look& L, int32_t seed_i, float freq, float px, float pz) {
  uint32_t seed = (uint32_t)seed_i;
  float sqrt3 = 1.7320508075688772f;
  float g2 = (3.0f - sqrt3) / 6.0f;
  float f2 = 0.5f * (sqrt3 - 1.0f);
  float x = px * freq, y = pz * freq;
  float s = (x + y) * f2;
  x = x + s; y = y + s;
  int32_t i0 = biome_fast_floor(x), j0 = biome_fast_floor(y);
  float xi = x - (float)i0, yi = y - (float)j0;
  float t = (xi + yi) * g2;
  float x0 = xi - t, y0 = yi - t;
  uint32_t i = (uint32_t)i0 * 501125321u, j = (uint32_t)j0 * 1136930381u;
  float a = 0.5f - x0 * x0 - y0 * y0;
  float n0 = 0.0f;
  if (a > 0.0f) n0 = (a * a) * (a * a) * simplex_grad(L, seed, i, j, x0, y0);
  float c = (2.0f * (1.0f - 2.0f * g2) * (1.0f / g2 - 2.0f)) * t + ((-2.0f * (1.0f - 2.0f * g2) * (1.0f - 2.0f * g2)) + a);
  float n2 = 0.0f;
  if (c > 0.0f) {
    float x2 = x0 + (2.0f * g2 - 1.0f), y2 = y0 + (2.0f * g2 - 1.0f);
    n2 = (c * c) * (c * c) * simplex_grad(L, seed, i + 501125321u, j + 1136930381u, x2, y2);
  }
  float n1 = 0.0f;
  if (y0 > x0) {
    float x1 = x0 + g2, y1 = y0 + (g2 - 1.0f);
    float b = 0.5f - x1 * x1 - y1 * y1;
    if (b > 0.0f) n1 = (b * b) * (b * b) * simplex_grad(L, seed, i, j + 1136930381u, x1, y1);
  } else {
    float x1 = x0 + (g2 - 1.0f), y1 = y0 + g2;
    float b = 0.5f - x1 * x1 - y1 * y1;
    if (b > 0.0f) n1 = (b * b) * (b * b) * simplex_grad(L, seed, i + 501125321u, j, x1, y1);
  }
  return (n0 + n1 + n2) * 99.83685446303647f;
}
V3 biome_band_weights(float n) {
  float hot = smoothstep(0.22f - 0.18f, 0.22f + 0.18f, n);
  float cold = 1.0f - smoothstep(-0.22f - 0.18f, -0.22f + 0.18f, n);
  return v3(cold, 1.0f - cold - hot, hot);
}
V3 biome_tint(const vm_frame& f, const Look& L, float x, float z) {
  float temperature = biome_noise(L, (int32_t)((uint32_t)f.tint_seed + 7u), f.tint_freq_t, x, z);
  float humidity = biome_noise(L, (int32_t)((uint32_t)f.tint_seed + 8u), f.tint_freq_h, x, z);
  V3 wt = biome_band_weights(temperature), wh = biome_band_weights(humidity);
  V3 plains = (L.spec_hi & HI_TINT_BALANCE) ? v3(0.935f, 1.067f, 0.892f) : v3(1.0f, 1.0f, 1.0f);
  V3 forest = v3(0.664f, 1.045f, 1.000f), savanna = v3(1.842f, 0.935f, 0.793f), desert = v3(2.096f, 0.957f, 0.699f);
  V3 taiga = v3(0.832f, 0.935f, 2.096f), tundra = v3(0.755f, 0.893f, 2.812f);
  V3 dry = add(add(muls(tundra, wt.x), muls(plains, wt.y)), muls(desert, wt.z));
  V3 mid = add(add(muls(taiga, wt.x), muls(plains, wt.y)), muls(savanna, wt.z));
  V3 wet = add(add(muls(taiga, wt.x), muls(forest, wt.y)), muls(forest, wt.z));
  return add(add(muls(dry, wh.x), muls(mid, wh.y)), muls(wet, wh.z));
}

float schlick_ground(float cos_i) {
  float m = clampf(1.0f - cos_i, 0.0f, 1.0f);
  float m2 = m * m;
  float top = fmaxf(1.0f - 0.9f, 0.04f);
  return 0.04f + (top - 0.04f) * m2 * m2 * m;
}
float face_shade(uint32_t nid) {
  switch (nid) {
    case 3u: return 1.00f;
    case 2u: return 0.50f;
    case 4u: case 5u: return 0.80f;
    case 6u: case 7u: return 0.90f;
    default: return 0.62f;
  }
}

// shadow_ray: common.wgsl:1098-1148 (the boolean sun test of secondary hits)
bool shadow_ray(const World& w, V3 ro, V3 rd, float max_dist) {
  const vm_frame& f = *w.f;
  V3 r_ro = ro;
  float r_dist = max_dist;
  if ((w.spec & VM_SPEC_WATER_REPAIR) != 0u && rd.y > 1e-4f && ro.y < f.sea_level) {
    float t_surf = (f.sea_level - ro.y) / rd.y;
    if (t_surf >= r_dist) return false;
    r_ro = add(ro, muls(rd, t_surf));
    r_dist = r_dist - t_surf;
  }
  V3 inv = v3(1.0f / rd.x, 1.0f / rd.y, 1.0f / rd.z);
  bool pos_dir[3] = {rd.x > 0.0f, rd.y > 0.0f, rd.z > 0.0f};
  I3 cell = floor_i(divs(r_ro, 64.0f));
  uint32_t last = VM_NO_CHUNK;
  for (uint32_t i = 0; i < 24u; ++i) {
    I3 rel = grid_rel(w, cell);
    if (grid_outside(w, rel)) return false;
    uint32_t ci = grid_at(w, grid_index(w, rel));
    if (ci != VM_NO_CHUNK && ci != last) {
      last = ci;
      if (march_chunk(w, ci, r_ro, rd, r_dist, true, true, true, true).hit) return true;
    }
    V3 bounds = v3((float)(pos_dir[0] ? cell.x + 1 : cell.x) * 64.0f, (float)(pos_dir[1] ? cell.y + 1 : cell.y) * 64.0f,
                   (float)(pos_dir[2] ? cell.z + 1 : cell.z) * 64.0f);
    V3 tn = mul(sub(bounds, r_ro), inv);
    uint32_t axis = 0u;
    float t;
    if (tn.x <= tn.y && tn.x <= tn.z) t = tn.x;
    else if (tn.y <= tn.z) { t = tn.y; axis = 1u; }
    else { t = tn.z; axis = 2u; }
    if (t >= r_dist) return false;
    setc(cell, axis, comp(cell, axis) + (pos_dir[axis] ? 1 : -1));
  }
  return false;
}

// shade_hit_legacy (resolve.wgsl:289-585) and shade_hit_legacy_cached
// (resolve.wgsl:1537-1788): lit_frame >= 0 is the cached sun visibility,
// lit_frame < 0 traces shadow_ray over shadow_dist.  The compact variants
// (SPEC_COMPACT_SHADE_HIT: shade_hit_compact, resolve.wgsl:587-851, and
// shade_hit_compact_cached, resolve.wgsl:1790-2054) run the same statements
// with the material block after the light block: the same chunk's box_min
// and local, canopy relief from material_ndl = ndl (the same dot(n, sun)),
// and light_rgb * face_scale with face_scale = 1.0, which is exact; their
// colours are the legacy variants' bit for bit, so this one restatement
// serves both.
V3 shade_hit(const World& w, const Look& L, uint32_t ci, U3 v, uint32_t id, uint32_t nid, V3 hit, V3 rd, float dist,
             float shadow_dist, bool smooth_light, bool do_spec, float lit_frame) {
  const vm_frame& f = *w.f;
  const vm_chunk& c = chunk_at(w, ci);
  float vs = c.voxel_size;
  bool foliage = nid >= VM_NORMAL_CROSS_A;
  V3 n = normal_of(nid);
  if (foliage && dot(n, rd) > 0.0f) n = neg(n);
  V3 sun = ld3(f.sun_dir);
  V3 spec_pre = v3(0.0f, 0.0f, 0.0f);
  if ((L.spec_hi & HI_SKY_SPECULAR) != 0u && do_spec)
    spec_pre = muls(sky_base(f, L, reflect(rd, n), 1.0f), schlick_ground(clampf(dot(n, neg(rd)), 0.0f, 1.0f)));
  uint32_t axis = nid >> 1u;
  V3 box_min = add(ld3(c.origin), muls(v3((float)v.x, (float)v.y, (float)v.z), vs));
  V3 lq = divs(sub(hit, box_min), vs);
  V3 local = v3(clampf(lq.x, 0.0f, 1.0f), clampf(lq.y, 0.0f, 1.0f), clampf(lq.z, 0.0f, 1.0f));
  uint32_t fi = id * 8u + nid;
  uint32_t face_word = fi < L.n_faces ? L.faces[fi] : 0u;
  uint32_t layer = face_word & 0xFFFFu;
  float u, tv;
  face_uv(nid, local, u, tv);
  if ((f.flags & VM_FLAG_TEX_VARIATION) != 0u) permute_uv(u, tv, face_word >> 16u, perm_key(box_min, nid));
  float fa, fb;
  I3 ta{0, 0, 0}, tb{0, 0, 0};
  if (axis == 0u) { fa = local.y; fb = local.z; ta.y = 1; tb.z = 1; }
  else if (axis == 1u) { fa = local.x; fb = local.z; ta.x = 1; tb.z = 1; }
  else { fa = local.x; fb = local.y; ta.x = 1; tb.y = 1; }
  float grazing = fmaxf(fabsf(dot(n, rd)), 0.25f);
  float footprint = fmaxf(dist, 1e-3f) * 2.0f * f.tan_half_fov / (float)f.res[1] * 16.0f / vs / grazing;
  float lod = clampf(log2f(fmaxf(footprint, 1e-4f)) + f.mip_bias, 0.0f, 3.0f);
  F4 texel = atlas_sample(L, u, tv, layer, lod);
  V3 albedo = v3(texel.r, texel.g, texel.b);
  float tint_mask = foliage ? 1.0f : texel.a;
  if ((f.flags & VM_FLAG_TINT) != 0u && tint_mask > 0.0f) {
    float k = tint_mask * f.tint_strength;
    albedo = mul(albedo, mixv(v3(1.0f, 1.0f, 1.0f), biome_tint(f, L, hit.x, hit.z), k));
  }
  if ((L.spec_hi & HI_SHORE_WET) != 0u && id == VM_SAND) {
    float wet = 1.0f - smoothstep(f.sea_level, f.sea_level + 1.5f, hit.y);
    albedo = muls(albedo, mixs(1.0f, 0.62f, wet));
  }
  if ((L.spec_hi & HI_FOLIAGE_RICH) != 0u && (foliage || ((id == VM_GRASS || id == VM_MEADOW) && nid == VM_NORMAL_PY))) {
    float hr = hash_alpha(box_min);
    float hv = hash_alpha(add(box_min, v3(17.31f, 7.77f, 3.03f)));
    V3 rich = v3(1.0f, 1.0f, 1.0f);
    if (hr < 0.16f) rich = v3(1.30f, 1.10f, 0.55f);
    else if (hr > 0.97f) rich = v3(1.35f, 0.72f, 0.95f);
    albedo = muls(mul(albedo, rich), mixs(0.88f, 1.10f, hv));
  }
  if ((L.spec_hi & HI_CANOPY_RELIEF) != 0u && is_cutout_id(id)) {
    float clump = cloud_noise(box_min.x * 0.21f + box_min.y * 0.313f, box_min.z * 0.21f + box_min.y * 0.173f);
    float relief = mixs(0.72f, 1.34f, clump * clump);
    float micro = mixs(0.92f, 1.08f, hash_alpha(box_min));
    float toward_sun = clampf(dot(n, sun) * 0.5f + 0.5f, 0.0f, 1.0f);
    albedo = muls(muls(muls(albedo, relief), micro), mixs(0.84f, 1.0f, toward_sun));
  }
  V3 sky_tint = surface_sky_fill(f, L, n);
  bool light_rgb = (f.flags & VM_FLAG_LIGHT_RGB) != 0u;
  bool gather = (w.spec & VM_SPEC_EMITTER_GATHER) != 0u;
  float ao = 1.0f, sky_sm = 0.0f;
  V3 amb = v3(0.0f, 0.0f, 0.0f);
  if (foliage) {
    uint32_t packed = light_at(w, ci, I3{(int32_t)v.x, (int32_t)v.y, (int32_t)v.z});
    float sk = light_curve(light_sky(packed)) * f.daylight;
    sky_sm = sk;
    if (light_rgb) {
      amb = block_ambient(light_curve3(light_block_rgb(packed)), sk, sky_tint);
    } else {
      float bk = light_curve(light_block_level(packed));
      amb = muls(mixv(sky_tint, BLOCK_TINT, bk / fmaxf(sk + bk, 1e-4f)), fmaxf(sk, bk));
    }
  } else if (!smooth_light) {
    I3 air_v1{(int32_t)v.x + (int32_t)n.x, (int32_t)v.y + (int32_t)n.y, (int32_t)v.z + (int32_t)n.z};
    uint32_t packed1;
    if (air_v1.x >= 0 && air_v1.y >= 0 && air_v1.z >= 0 && air_v1.x <= 63 && air_v1.y <= 63 && air_v1.z <= 63)
      packed1 = light_at(w, ci, air_v1);
    else
      packed1 = world_sample(w, add(add(box_min, v3(0.5f * vs, 0.5f * vs, 0.5f * vs)), muls(n, vs))).x;
    float sk1 = light_curve(light_sky(packed1)) * f.daylight;
    sky_sm = sk1;
    if (light_rgb) {
      amb = block_ambient(light_curve3(light_block_rgb(packed1)), sk1, sky_tint);
    } else {
      float bk1 = light_curve(light_block_level(packed1));
      amb = muls(mixv(sky_tint, BLOCK_TINT, bk1 / fmaxf(sk1 + bk1, 1e-4f)), fmaxf(sk1, bk1));
    }
  } else {
    V3 air_c = add(add(box_min, v3(0.5f * vs, 0.5f * vs, 0.5f * vs)), muls(n, vs));
    V3 step_a = muls(v3((float)ta.x, (float)ta.y, (float)ta.z), vs);
    V3 step_b = muls(v3((float)tb.x, (float)tb.y, (float)tb.z), vs);
    I3 air_v{(int32_t)v.x + (int32_t)n.x, (int32_t)v.y + (int32_t)n.y, (int32_t)v.z + (int32_t)n.z};
    I3 span{ta.x + tb.x, ta.y + tb.y, ta.z + tb.z};
    bool local_only = air_v.x - span.x >= 0 && air_v.y - span.y >= 0 && air_v.z - span.z >= 0 &&
                      air_v.x + span.x <= 63 && air_v.y + span.y <= 63 && air_v.z + span.z <= 63;
    U2 nb[9];
    if (local_only) {
      gather_face(w, ci, air_v, ta, tb, nb);
    } else {
      for (uint32_t i = 0; i < 9u; ++i)
        nb[i] = world_sample(w, add(add(air_c, muls(step_a, (float)(i % 3u) - 1.0f)), muls(step_b, (float)(i / 3u) - 1.0f)));
    }
    float sky_n[9], blk_n[9], open_n[9];
    uint32_t any_blk = 0u;
    for (uint32_t i = 0; i < 9u; ++i) {
      sky_n[i] = light_curve(light_sky(nb[i].x)) * f.daylight;
      blk_n[i] = 0.0f;
      if (light_rgb) {
        if (gather) any_blk = any_blk | (nb[i].x & 0xFFFu);
      } else {
        blk_n[i] = light_curve(light_block_level(nb[i].x));
      }
      open_n[i] = 1.0f - (float)nb[i].y;
    }
    V3 blk4 = v3(0.0f, 0.0f, 0.0f);
    if (gather && light_rgb && any_blk != 0u) blk4 = light_curve3(light_block_rgb(nb[4].x));
    bool ao_on = (f.flags & VM_FLAG_AO) != 0u;
    V3 amb_c[4];
    float sky_c[4], ao_c[4];
    for (uint32_t k = 0; k < 4u; ++k) {
      uint32_t ia = (uint32_t)(4 + ((int32_t)(k & 1u) * 2 - 1));
      uint32_t ib = (uint32_t)(4 + ((int32_t)(k >> 1u) * 2 - 1) * 3);
      uint32_t ic = ia + ib - 4u;
      float inv = 1.0f / (1.0f + open_n[ia] + open_n[ib] + open_n[ic]);
      float sk = (sky_n[4] + sky_n[ia] * open_n[ia] + sky_n[ib] * open_n[ib] + sky_n[ic] * open_n[ic]) * inv;
      sky_c[k] = sk;
      if (light_rgb) {
        if (gather && any_blk != 0u) {
          V3 ba = light_curve3(light_block_rgb(nb[ia].x));
          V3 bb = light_curve3(light_block_rgb(nb[ib].x));
          V3 bc = light_curve3(light_block_rgb(nb[ic].x));
          V3 bkv = muls(add(add(add(blk4, muls(ba, open_n[ia])), muls(bb, open_n[ib])), muls(bc, open_n[ic])), inv);
          amb_c[k] = block_ambient(bkv, sk, sky_tint);
        } else {
          amb_c[k] = muls(sky_tint, sk);
        }
      } else {
        float bk = (blk_n[4] + blk_n[ia] * open_n[ia] + blk_n[ib] * open_n[ib] + blk_n[ic] * open_n[ic]) * inv;
        amb_c[k] = muls(mixv(sky_tint, BLOCK_TINT, bk / fmaxf(sk + bk, 1e-4f)), fmaxf(sk, bk));
      }
      float s1 = 1.0f - open_n[ia];
      float s2 = 1.0f - open_n[ib];
      float occ = (s1 > 0.5f && s2 > 0.5f) ? 3.0f : s1 + s2 + 1.0f - open_n[ic];
      ao_c[k] = ao_on ? 1.0f - occ * 0.25f : 1.0f;
    }
    ao = mixs(mixs(ao_c[0], ao_c[1], fa), mixs(ao_c[2], ao_c[3], fa), fb);
    sky_sm = mixs(mixs(sky_c[0], sky_c[1], fa), mixs(sky_c[2], sky_c[3], fa), fb);
    amb = mixv(mixv(amb_c[0], amb_c[1], fa), mixv(amb_c[2], amb_c[3], fa), fb);
  }
  // SPEC_PROBE_AMBIENT / SPEC_PROBE_TAP (resolve.wgsl:500-505): the ambient
  // from the probe tap alone (the light words' ambient unused), or scaled by it
  const bool probe_ambient = (f.flags & VM_FLAG_PROBE_AMBIENT) != 0u;
  if (probe_ambient) amb = probe_tap(L, hit);
  else if ((f.flags & VM_FLAG_PROBE_TAP) != 0u) amb = mul(amb, probe_tap(L, hit));
  float direct = 0.0f, visibility = 1.0f;
  float ndl = dot(n, sun);
  if (ndl > 0.0f && f.daylight > 0.01f) {
    float lit = 1.0f;
    if ((f.flags & VM_FLAG_SHADOWS) != 0u) {
      lit = lit_frame >= 0.0f ? lit_frame : (shadow_ray(w, add(hit, muls(n, 0.02f * vs)), sun, shadow_dist) ? 0.0f : 1.0f);
      if ((f.flags & VM_FLAG_DISTANT_SHADOWS) != 0u && lit > 0.0f)
        lit = lit * terrain_shade(f, L, add(hit, muls(sun, shadow_dist)));
    }
    if (lit > 0.0f) {
      float cloud_fp = fmaxf(dist, 1e-3f) * 2.0f * f.tan_half_fov / (float)f.res[1] * exp2f(f.mip_bias);
      lit = lit * cloud_shade(f, hit, cloud_fp);
    }
    visibility = lit;
    direct = lit * ndl * sky_sm;
    if ((L.spec_hi & HI_CAUSTICS) != 0u) {
      float cdepth = f.sea_level - hit.y;
      if (cdepth > 0.0f && cdepth < 8.0f && direct > 0.0f) {
        float k = cdepth / fmaxf(sun.y, 1e-3f);
        float spx = hit.x - sun.x * k, spz = hit.z - sun.z * k;
        float a = f.wave_amp, l0 = f.wave_scale, ph = f.time * f.wave_speed * WAVE_TAU;
        V3 g0 = wave_octave(spx, spz, 0.913089f, 0.407760f, l0, a * 0.42f, ph, 0.35f, 0.0f, 0.0f, 0.0f, false);
        V3 g1 = wave_octave(spx, spz, -0.388685f, 0.921371f, l0 / 2.17f, a * 0.27f, ph * 1.4731f, 0.35f, 0.0f, 0.0f,
                            0.0f, false);
        float r0 = g0.x * g0.x + g0.y * g0.y;
        float r1 = g1.x * g1.x + g1.y * g1.y;
        float sheets = r0 * r1 * 4000.0f;
        direct = direct * (1.0f + sheets * expf(-cdepth * 0.30f));
      }
    }
  }
  bool probe_cube = (f.flags & VM_FLAG_PROBE_CUBE) != 0u, probe_bounce = (f.flags & VM_FLAG_PROBE_BOUNCE) != 0u;
  F4 probe = {1.0f, 1.0f, 1.0f, 1.0f};
  if (!probe_ambient && (probe_cube || probe_bounce)) probe = probe_field(L, add(hit, muls(n, 2.0f)), nid);
  float shade = 1.0f;
  if (!probe_ambient) {
    shade = repair(L) ? 1.0f : face_shade(nid);
    if (probe_cube) shade = shade * probe.a;
  }
  V3 ambient_rgb = muls(amb, 0.50f);
  V3 sun_rgb = muls(v3(1.0000f, 0.8469f, 0.5647f), direct * (repair(L) ? 0.78f : 0.52f));
  V3 floor_rgb = v3(0.0f, 0.0f, 0.0f);
  V3 prgb = v3(probe.r, probe.g, probe.b);
  if (!probe_ambient) {
    floor_rgb = muls(v3(0.85f, 0.90f, 1.00f), f.ambient);
    if (probe_bounce) floor_rgb = mul(floor_rgb, prgb);
    if ((f.flags & VM_FLAG_PROBE_SUN) != 0u) {
      float gain = (f.flags & VM_FLAG_PROBE_SUN_HIGH) != 0u ? 0.25f : 0.10f;
      floor_rgb = add(floor_rgb, muls(mul(v3(0.85f, 0.90f, 1.00f), prgb), gain * sky_sm));
    }
  }
  uint32_t debug_view = surface_debug(L);   // resolve.wgsl:579-582
  if (debug_view == 1u) return add(muls(n, 0.5f), v3(0.5f, 0.5f, 0.5f));
  if (debug_view == 2u) return v3(visibility, visibility, visibility);
  if (debug_view == 3u) return sun_rgb;
  if (debug_view == 4u) return add(muls(ambient_rgb, ao), floor_rgb);
  V3 spec_rgb = muls(spec_pre, sky_sm * 0.5f);
  V3 light = repair(L) ? add(add(muls(muls(ambient_rgb, ao), shade), sun_rgb), floor_rgb)
                       : muls(add(muls(add(ambient_rgb, sun_rgb), ao), floor_rgb), shade);
  if (repair(L) && id == VM_GLOWSTONE) return mul(albedo, add(muls(v3(1.0f, 0.7111f, 0.3024f), 1.5f), muls(light, 0.15f)));
  return add(mul(albedo, light), spec_rgb);
}

// ---- the water and glass lanes: resolve.wgsl:896-1320 ----------------------
constexpr uint32_t HI_SHORE_FOAM = 16u, HI_WATER_SEC = 32u, HI_GLASS_REFLECT = 128u, HI_WATER_LOOK = 4096u;
constexpr float WATER_LOOK_RIPPLE_AMP = 0.16f;

// look_ripple: resolve.wgsl:995-1008
void look_ripple(const World& w, float px, float pz, float time, float w1, float w2, float& gx, float& gz) {
  const float d1x = 0.86f, d1z = 0.51f, d2x = -0.42f, d2z = 0.91f;
  const float k1 = (float)(6.2832 / 1.15), k2 = (float)(6.2832 / 0.62);
  float ph_x = 0.0f, ph_z = 0.0f;
  if ((w.spec & VM_SPEC_WATER_REPAIR) != 0u) {
    ph_x = sinf(px * 0.071f + pz * 0.113f) * 2.0f;
    ph_z = sinf(px * -0.097f + pz * 0.053f + 1.9f) * 2.0f;
  }
  float a1 = cosf((px * d1x + pz * d1z) * k1 + time * 1.7f + ph_x) * w1;
  float a2 = cosf((px * d2x + pz * d2z) * k2 - time * 2.3f + ph_z) * w2;
  gx = d1x * a1 + d2x * a2;
  gz = d1z * a1 + d2z * a2;
}

inline bool secondary_smooth(const vm_frame& f) { return (f.flags & VM_FLAG_FLAT_SECONDARY) == 0u; }
float medium_light(const vm_frame& f, uint32_t packed) {
  float sky_l = light_curve(light_sky(packed)) * f.daylight;
  float blk_l = light_curve(light_block_level(packed));
  return fmaxf(sky_l, blk_l) * 0.50f + f.ambient;
}
V3 water_medium(const vm_frame& f, V3 c, float d, V3 body) {   // common.wgsl:1262-1265
  float dd = fmaxf(d, 0.0f);
  V3 tr = v3(expf(-0.280f * f.water_absorb * dd), expf(-0.055f * f.water_absorb * dd),
             expf(-0.020f * f.water_absorb * dd));
  return add(mul(c, tr), mul(body, v3(1.0f - tr.x, 1.0f - tr.y, 1.0f - tr.z)));
}
float schlick_f0(float f0, float cos_i) {   // common.wgsl:1267-1279
  float m = clampf(1.0f - cos_i, 0.0f, 1.0f);
  float m2 = m * m;
  return f0 + (1.0f - f0) * m2 * m2 * m;
}

struct WaterCtx {
  V3 body; float ml; V3 n, nw, nt; float gloss; bool waved; float refract_detail, reflect_detail;
  V3 mirror, mirror_t, hit, rd; float t, roughness;
};

// water_ctx: resolve.wgsl:1078-1166 (SPEC_WATER_LOOK off)
WaterCtx water_ctx(const World& w, const Look& L, uint32_t ci, U3 v, uint32_t nid, V3 hit, V3 rd, float t) {
  const vm_frame& f = *w.f;
  WaterCtx x;
  const vm_chunk& c = chunk_at(w, ci);
  float vs = c.voxel_size;
  V3 n = normal_of(nid);
  V3 box_min = add(ld3(c.origin), muls(v3((float)v.x, (float)v.y, (float)v.z), vs));
  V3 lq = divs(sub(hit, box_min), vs);
  V3 local = v3(clampf(lq.x, 0.0f, 1.0f), clampf(lq.y, 0.0f, 1.0f), clampf(lq.z, 0.0f, 1.0f));
  float footprint = fmaxf(t, 1e-3f) * 2.0f * f.tan_half_fov / (float)f.res[1] * 16.0f / vs;
  float lod = clampf(log2f(fmaxf(footprint, 1e-4f)) + f.mip_bias, 0.0f, 3.0f);
  uint32_t fi = VM_WATER * 8u + nid;
  uint32_t layer = (fi < L.n_faces ? L.faces[fi] : 0u) & 0xFFFFu;
  float u, tv;
  face_uv(nid, local, u, tv);
  F4 tint = atlas_sample(L, u, tv, layer, lod);
  if ((w.spec & VM_SPEC_WATER_REPAIR) != 0u) tint = atlas_sample(L, 0.5f, 0.5f, layer, 3.0f);
  x.ml = medium_light(f, light_at(w, ci, I3{(int32_t)v.x, (int32_t)v.y, (int32_t)v.z}));
  x.body = muls(v3(tint.r, tint.g, tint.b), x.ml);
  x.refract_detail = 1.0f - smoothstep(VM_WATER_REFRACT_NEAR, VM_WATER_REFRACT_FAR, t);
  x.reflect_detail = 1.0f - smoothstep(VM_WATER_REFLECT_NEAR, VM_WATER_REFLECT_FAR, t);
  float px_world = fmaxf(t, 1e-3f) * 2.0f * f.tan_half_fov / (float)f.res[1];
  V3 nw = n, nt = n;
  float gloss = 1.0f, unresolved = 0.0f;
  bool waved = (f.flags & VM_FLAG_WAVES) != 0u && nid == VM_NORMAL_PY;
  if (waved) {
    float kk = 0.0f, vhx = 0.0f, vhz = 0.0f;
    bool aniso = (f.flags & VM_FLAG_WAVE_ANISO) != 0u;
    if (aniso) {
      float k = 1.0f / fmaxf(fabsf(rd.y), WAVE_GRAZE_MIN);
      kk = k * k - 1.0f;
      float r = 1.0f / sqrtf(fmaxf(rd.x * rd.x + rd.z * rd.z, 1e-12f));
      vhx = rd.x * r; vhz = rd.z * r;
    }
    float shoal = 1.0f;
    if ((f.flags & VM_FLAG_WAVE_SHOAL) != 0u) {
      V3 dro = v3(floorf(hit.x) + 0.5f, hit.y - VM_SURFACE_EPS, floorf(hit.z) + 0.5f);
      WorldHit dh = trace_world(w, dro, v3(0.001f, -0.999999f, 0.001f), SHOAL_DEPTH, true);
      shoal = smoothstep(0.0f, SHOAL_DEPTH, dh.hit ? dh.t : SHOAL_DEPTH);
    }
    V3 wf = wave_field(f, hit.x, hit.z, px_world, vhx, vhz, kk, aniso, shoal);
    unresolved = fmaxf(wf.z, 0.0f);
    nw = normalize(v3(-wf.x, 1.0f, -wf.y));
    float gl = sqrtf(wf.x * wf.x + wf.y * wf.y);
    float lim = fminf(1.0f, f.wave_reflect_slope / fmaxf(gl, 1e-6f));
    nt = normalize(v3(-(wf.x * lim), 1.0f, -(wf.y * lim)));
    gloss = 1.0f / (1.0f + 0.5f * 320.0f * wf.z);
  }
  if ((L.spec_hi & HI_WATER_LOOK) != 0u && nid == VM_NORMAL_PY) {   // resolve.wgsl:1138-1153
    float pix = px_world / fmaxf(fabsf(rd.y), 1e-3f);
    float range_gate = (1.0f - smoothstep(48.0f, 96.0f, t)) * smoothstep(0.08f, 0.20f, fabsf(rd.y));
    float fade_115 = range_gate * smoothstep(2.0f, 4.0f, 1.15f / fmaxf(pix, 1e-4f));
    float fade_62 = range_gate * smoothstep(2.0f, 4.0f, 0.62f / fmaxf(pix, 1e-4f));
    unresolved += WATER_LOOK_RIPPLE_AMP * WATER_LOOK_RIPPLE_AMP * 0.5f *
                  (0.36f * (1.0f - fade_115 * fade_115) + 0.16f * (1.0f - fade_62 * fade_62));
    float gx, gz;
    look_ripple(w, hit.x, hit.z, f.time * f.wave_speed, 0.60f * fade_115, 0.40f * fade_62, gx, gz);
    nw = normalize(add(nw, muls(v3(gx, 0.0f, gz), WATER_LOOK_RIPPLE_AMP)));
  }
  float rough = clampf(1.0f - expf(-8.0f * unresolved), 0.0f, 1.0f);
  nw = normalize(add(muls(nw, 1.0f - rough), muls(n, rough)));
  nt = normalize(add(muls(nt, 1.0f - rough), muls(n, rough)));
  x.n = n; x.nw = nw; x.nt = nt; x.gloss = gloss; x.waved = waved;
  x.mirror = reflect(rd, nw);
  V3 mt = reflect(rd, nt);
  if (waved) mt = normalize(v3(mt.x, fmaxf(mt.y, 0.0f), mt.z));
  x.mirror_t = mt;
  x.hit = hit; x.rd = rd; x.t = t; x.roughness = rough;
  return x;
}

V3 shade_leg(const World& w, const Look& L, const WorldHit& h, V3 p, V3 d, float dist, float shadow_dist) {
  uint32_t id = block_at(w, h.ci, h.voxel);
  return shade_hit(w, L, h.ci, h.voxel, id, h.normal, p, d, dist, shadow_dist, secondary_smooth(*w.f), false, -1.0f);
}
F4 water_refract_leg(const World& w, const Look& L, V3 hit, V3 n, V3 rd, float t) {   // resolve.wgsl:1029-1042
  V3 rdir = refract(rd, n, 1.0f / VM_WATER_IOR);
  V3 ro2 = add(hit, muls(rdir, VM_SURFACE_EPS));
  WorldHit h2 = trace_world(w, ro2, rdir, VM_WATER_REFRACT_DIST, true);
  V3 under = v3(0.0f, 0.0f, 0.0f);
  float depth = VM_WATER_REFRACT_DIST;
  if (h2.hit) {
    under = shade_leg(w, L, h2, add(ro2, muls(rdir, h2.t)), rdir, t + h2.t, 16.0f);
    depth = h2.t;
  }
  return {under.x, under.y, under.z, depth};
}
F4 water_reflect_leg(const World& w, const Look& L, V3 hit, V3 n, V3 mirror_t, float t) {   // resolve.wgsl:1044-1058
  V3 ro3 = add(hit, muls(n, VM_SURFACE_EPS));
  WorldHit h3 = trace_world(w, ro3, mirror_t, VM_WATER_REFLECT_DIST, true);
  if (!h3.hit) return {0.0f, 0.0f, 0.0f, 0.0f};
  V3 lit = shade_leg(w, L, h3, add(ro3, muls(mirror_t, h3.t)), mirror_t, t + h3.t, w.f->shadow_dist);
  lit = mixv(lit, sky_base(*w.f, L, mirror_t, 1.0f), 1.0f - transmittance_from(*w.f, hit.y, h3.t, mirror_t));
  return {lit.x, lit.y, lit.z, 1.0f};
}

// foam_hash / foam_mottle: resolve.wgsl:1011-1027
float foam_hash(float ix, float iy) {
  int32_t qx = f2i(ix), qy = f2i(iy);
  return (float)((hash_u32((uint32_t)qx * 374761393u + (uint32_t)qy * 668265263u) >> 8u) & 0xFFFFFFu) / 16777216.0f;
}
float foam_mottle(float x, float z, float time) {
  const float k = (float)(1.0 / 0.7);   // the abstract-float constant 1.0 / 0.7 as f32
  float px = x * k, pz = z * k;
  float ix = floorf(px), iz = floorf(pz);
  float wx = px - ix, wz = pz - iz;
  float ux = wx * wx * (3.0f - 2.0f * wx), uz = wz * wz * (3.0f - 2.0f * wz);
  float m0 = mixs(foam_hash(ix, iz), foam_hash(ix + 1.0f, iz), ux);
  float m1 = mixs(foam_hash(ix, iz + 1.0f), foam_hash(ix + 1.0f, iz + 1.0f), ux);
  float m = mixs(m0, m1, uz);
  float ph = time * 0.55f * 4.0f + foam_hash(ix * 2.23f, iz * 2.71f) * 6.28318f;
  return m * (0.5f + 0.5f * sinf(ph));
}

// water_compose: resolve.wgsl:1169-1207
V3 water_compose(const vm_frame& f, const Look& L, const WaterCtx& x, F4 leg_r, F4 leg_m) {
  V3 refr = x.body;
  float column_depth = VM_WATER_REFRACT_DIST;
  if ((f.flags & VM_FLAG_WATER_REFRACT) != 0u && x.refract_detail > 0.0f) {
    refr = mixv(refr, water_medium(f, v3(leg_r.r, leg_r.g, leg_r.b), leg_r.a, x.body), x.refract_detail);
    column_depth = leg_r.a;
  }
  if ((L.spec_hi & HI_WATER_LOOK) != 0u && x.refract_detail > 0.0f) {   // resolve.wgsl:1178-1183
    float depth_f = clampf(column_depth / 7.0f, 0.0f, 1.0f);
    refr = mul(refr, mixv(v3(1.0f, 1.0f, 1.0f), v3(0.82f, 0.90f, 0.70f), depth_f));
    float shall = 1.0f - smoothstep(0.0f, 2.0f, column_depth);
    refr = mixv(refr, muls(v3(0.55f, 0.74f, 0.68f), x.ml), shall * 0.45f * x.refract_detail);
  }
  if ((L.spec_hi & HI_SHORE_FOAM) != 0u && x.refract_detail > 0.0f && column_depth < 2.5f) {
    float shall = 1.0f - smoothstep(0.0f, 2.5f, column_depth);
    float m = foam_mottle(x.hit.x, x.hit.z, f.time * f.wave_speed);
    float foam = shall * smoothstep(0.45f, 0.75f, m) * x.refract_detail;
    refr = mixv(refr, muls(v3(0.92f, 0.97f, 1.0f), x.ml), clampf(foam, 0.0f, 1.0f) * 0.85f);
  }
  V3 refl = add(sky_color(f, L, x.hit, x.mirror, x.t, 1.0f),
                muls(v3(1.0000f, 0.8469f, 0.5647f),
                     powf(fmaxf(dot(x.mirror, ld3(f.sun_dir)), 0.0f), 320.0f * x.gloss) * 2.5f * x.gloss * f.daylight));
  if ((f.flags & VM_FLAG_WATER_REFLECT) != 0u && x.reflect_detail > 0.0f && leg_m.a > 0.0f)
    refl = mixv(refl, v3(leg_m.r, leg_m.g, leg_m.b), x.reflect_detail);
  uint32_t debug_view = surface_debug(L);   // resolve.wgsl:1200-1202
  if (debug_view == 5u) return add(muls(x.n, 0.5f), v3(0.5f, 0.5f, 0.5f));
  if (debug_view == 6u) return refl;
  if (debug_view == 7u) return refr;
  refl = mixv(refl, sky_base(f, L, x.n, 1.0f), x.roughness * 0.65f);
  return mixv(refr, refl, schlick_f0(0.02f, fmaxf(-dot(x.rd, x.nw), 1e-3f)));
}

V3 shade_water(const World& w, const Look& L, uint32_t ci, U3 v, uint32_t nid, V3 hit, V3 rd, float t) {
  const vm_frame& f = *w.f;
  WaterCtx x = water_ctx(w, L, ci, v, nid, hit, rd, t);
  F4 leg_r{0.0f, 0.0f, 0.0f, VM_WATER_REFRACT_DIST};
  if ((f.flags & VM_FLAG_WATER_REFRACT) != 0u && x.refract_detail > 0.0f) leg_r = water_refract_leg(w, L, hit, x.n, rd, t);
  F4 leg_m{0.0f, 0.0f, 0.0f, 0.0f};
  if ((f.flags & VM_FLAG_WATER_REFLECT) != 0u && x.reflect_detail > 0.0f)
    leg_m = water_reflect_leg(w, L, hit, x.n, x.mirror_t, t);
  return water_compose(f, L, x, leg_r, leg_m);
}

// shade_glass: resolve.wgsl:1261-1319
V3 shade_glass(const World& w, const Look& L, uint32_t ci, U3 v, uint32_t nid, V3 hit, V3 rd, float t) {
  const vm_frame& f = *w.f;
  const vm_chunk& c = chunk_at(w, ci);
  float vs = c.voxel_size;
  V3 n = normal_of(nid);
  if (dot(n, rd) > 0.0f) n = neg(n);
  V3 box_min = add(ld3(c.origin), muls(v3((float)v.x, (float)v.y, (float)v.z), vs));
  V3 lq = divs(sub(hit, box_min), vs);
  V3 local = v3(clampf(lq.x, 0.0f, 1.0f), clampf(lq.y, 0.0f, 1.0f), clampf(lq.z, 0.0f, 1.0f));
  float footprint = fmaxf(t, 1e-3f) * 2.0f * f.tan_half_fov / (float)f.res[1] * 16.0f / vs;
  float lod = clampf(log2f(fmaxf(footprint, 1e-4f)) + f.mip_bias, 0.0f, 3.0f);
  uint32_t fi = VM_GLASS * 8u + nid;
  uint32_t layer = (fi < L.n_faces ? L.faces[fi] : 0u) & 0xFFFFu;
  float u, tv;
  face_uv(nid, local, u, tv);
  F4 tx = atlas_sample(L, u, tv, layer, lod);
  V3 tint = v3(tx.r, tx.g, tx.b);
  V3 ro2 = add(hit, muls(rd, VM_SURFACE_EPS));
  float reach = fmaxf(VM_GLASS_TRANSMIT_DIST, f.far_);
  WorldHit h2 = trace_world(w, ro2, rd, reach, false);
  V3 through = sky_color(f, L, ro2, rd, t, 1.0f);
  if (h2.hit) {
    V3 p2 = add(ro2, muls(rd, h2.t));
    if (block_at(w, h2.ci, h2.voxel) == VM_WATER)
      through = shade_water(w, L, h2.ci, h2.voxel, h2.normal, p2, rd, t + h2.t);
    else
      through = shade_leg(w, L, h2, p2, rd, t + h2.t, 48.0f);
    through = mixv(through, sky_base(f, L, rd, 1.0f), 1.0f - transmittance_from(f, hit.y, h2.t, rd));
  }
  V3 mirror = reflect(rd, n);
  V3 refl = sky_color(f, L, hit, mirror, t, 1.0f);
  if ((L.spec_hi & HI_GLASS_REFLECT) != 0u) {
    V3 origin = add(hit, muls(n, VM_SURFACE_EPS));
    WorldHit r = trace_world(w, origin, mirror, reach, false);
    if (r.hit) {
      V3 point = add(origin, muls(mirror, r.t));
      if (block_at(w, r.ci, r.voxel) == VM_WATER)
        refl = shade_water(w, L, r.ci, r.voxel, r.normal, point, mirror, t + r.t);
      else
        refl = shade_leg(w, L, r, point, mirror, t + r.t, 48.0f);
      refl = mixv(refl, sky_base(f, L, mirror, 1.0f), 1.0f - transmittance_from(f, hit.y, r.t, mirror));
    }
  }
  return mixv(mul(through, tint), refl, schlick_f0(0.0426f, fmaxf(-dot(rd, n), 1e-3f)));
}

// water_share_safe: resolve.wgsl:1223-1245
bool water_share_safe(const World& w, const uint64_t* vis, uint32_t shift, uint32_t px, uint32_t py, uint32_t nid,
                      V3 hit, float t) {
  const vm_frame& f = *w.f;
  if (nid != VM_NORMAL_PY) return false;
  uint32_t span = 1u << shift;
  uint32_t bx = (px >> shift) * span, by = (py >> shift) * span;
  for (uint32_t y = 0; y < span; ++y)
    for (uint32_t x = 0; x < span; ++x) {
      uint32_t qx = bx + x, qy = by + y;
      if (qx >= f.res[0] || qy >= f.res[1]) continue;
      uint64_t key = vis[(uint64_t)qy * f.res[0] + qx];
      if (key == 0) return false;
      if (key_nid(key) != nid) return false;
      uint32_t ci = key_ci(key);
      U3 v = key_voxel(key), micro = key_micro(key);
      if (block_at(w, ci, v) != VM_WATER) return false;
      V3 rd = ray_dir(f, (float)qx + 0.5f, (float)qy + 0.5f);
      float td = hit_t(w, ci, v, micro, nid, rd);
      V3 hd = add(ld3(f.cam_pos), muls(rd, td));
      if (fabsf(hd.y - hit.y) > 0.01f || fabsf(td - t) > fmaxf(0.1f, fminf(1.0f, t * 0.02f))) return false;
    }
  return true;
}

// the water_sec pass's colour (resolve.wgsl:1468-1535) of block (hx, hy):
// the water pixel of least hit distance, its legs, through the rgba16float
// targets' rounding
void water_sec_legs(const World& w, const Look& L, const uint64_t* vis, uint32_t shift, uint32_t hx, uint32_t hy,
                    F4* leg_r_out, F4* leg_m_out) {
  const vm_frame& f = *w.f;
  uint32_t span = 1u << shift;
  F4 leg_r{0.0f, 0.0f, 0.0f, VM_WATER_REFRACT_DIST}, leg_m{0.0f, 0.0f, 0.0f, 0.0f};
  float best_t = 3.4e38f;
  bool has = false;
  uint32_t bci = 0, bnid = 0, bpx = 0, bpy = 0;
  U3 bv{0, 0, 0};
  for (uint32_t i = 0; i < span; ++i)
    for (uint32_t j = 0; j < span; ++j) {
      uint32_t pxs = span * hx + i, pys = span * hy + j;
      if (pxs >= f.res[0] || pys >= f.res[1]) continue;
      uint64_t key = vis[(uint64_t)pys * f.res[0] + pxs];
      if (key == 0) continue;
      uint32_t nids = key_nid(key), cis = key_ci(key);
      U3 vs_ = key_voxel(key), micros = key_micro(key);
      if (block_at(w, cis, vs_) != VM_WATER) continue;
      V3 rd0 = ray_dir(f, (float)pxs + 0.5f, (float)pys + 0.5f);
      float ts = hit_t(w, cis, vs_, micros, nids, rd0);
      if (ts < best_t) { best_t = ts; bci = cis; bv = vs_; bnid = nids; bpx = pxs; bpy = pys; has = true; }
    }
  if (has) {
    V3 rd_d = ray_dir(f, (float)bpx + 0.5f, (float)bpy + 0.5f);
    V3 hit_d = add(ld3(f.cam_pos), muls(rd_d, best_t));
    WaterCtx x = water_ctx(w, L, bci, bv, bnid, hit_d, rd_d, best_t);
    if ((f.flags & VM_FLAG_WATER_REFRACT) != 0u && x.refract_detail > 0.0f)
      leg_r = water_refract_leg(w, L, hit_d, x.n, rd_d, best_t);
    if ((f.flags & VM_FLAG_WATER_REFLECT) != 0u && x.reflect_detail > 0.0f)
      leg_m = water_reflect_leg(w, L, hit_d, x.n, x.mirror_t, best_t);
  }
  *leg_r_out = {f16_round(leg_r.r), f16_round(leg_r.g), f16_round(leg_r.b), f16_round(leg_r.a)};
  *leg_m_out = {f16_round(leg_m.r), f16_round(leg_m.g), f16_round(leg_m.b), f16_round(leg_m.a)};
}

float srgb_to_linear(uint8_t u) {
  float c = (float)u / 255.0f;
  return c <= 0.04045f ? c / 12.92f : powf((c + 0.055f) / 1.055f, 2.4f);
}

}  // namespace

extern "C" {

typedef struct or_look {
  const uint8_t* atlas_srgb; uint32_t layers;   // Rgba8UnormSrgb, 16x16, 4 mips as the engine uploads them
  const uint32_t* faces; uint32_t n_faces;
  const uint16_t* probes;                       // RGBA16F 128 x 768 x 128, or null
  const float* shaft;                           // 512 x 512, or null
  uint32_t spec_hi;
} or_look;

// The resolve's colour (RGBA, alpha 1; water and glass pixels 0) of pixels
// [pix_begin, pix_end) from the frame's keys and the sun visibility of each
// pixel (the engine's primary_sun: r8unorm of the soft mask, or 1 - blocked).
// ---- the underwater resolve: resolve.wgsl:1321-1376,1449-1464 ----------------
constexpr uint32_t FLAG_SNELL = 8388608u;   // mod.rs FLAG_SNELL
// water_path: common.wgsl:1293-1298
float water_path(const vm_frame& f, float t, V3 rd) {
  if (rd.y <= 0.0f) return t;
  return clampf((f.sea_level - f.cam_pos[1]) / rd.y, 0.0f, t);
}
// underwater_body: resolve.wgsl:1321-1323 (WATER_BODY, resolve.wgsl:894)
V3 underwater_body(const World& w) {
  return muls(v3(0.0100f, 0.0947f, 0.1474f), medium_light(*w.f, world_sample(w, ld3(w.f->cam_pos)).x));
}
// surface_from_below: resolve.wgsl:1325-1376 (SNELL_MIN_DEPTH 3, WATER_DARK_DEPTH
// 15, SNELL_DIM_MAX 0.9: common.wgsl:167-171)
V3 surface_from_below(const World& w, V3 above, V3 rd, float dist) {
  const vm_frame& f = *w.f;
  if ((f.flags & FLAG_SNELL) == 0u) return above;
  float depth = f.sea_level - f.cam_pos[1];
  float s = smoothstep(3.0f, 15.0f, depth);
  if (s <= 0.0f) return above;
  if (rd.y <= 0.0f) return above;
  float t_surf = (f.sea_level - f.cam_pos[1]) / rd.y;
  if (t_surf >= dist || t_surf <= 0.0f) return above;
  V3 surf = add(ld3(f.cam_pos), muls(rd, t_surf));
  float mirror_detail = 1.0f - smoothstep(VM_WATER_REFRACT_NEAR, VM_WATER_REFRACT_FAR, t_surf);
  V3 nup = v3(0.0f, 1.0f, 0.0f);
  if ((f.flags & VM_FLAG_WAVES) != 0u && mirror_detail > 0.0f) {
    float px_world = fmaxf(t_surf, 1e-3f) * 2.0f * f.tan_half_fov / (float)f.res[1];
    float kk = 0.0f, vhx = 0.0f, vhz = 0.0f;
    bool aniso = (f.flags & VM_FLAG_WAVE_ANISO) != 0u;
    if (aniso) {
      float k = 1.0f / fmaxf(fabsf(rd.y), 1e-3f);
      kk = k * k - 1.0f;
      float r = 1.0f / sqrtf(fmaxf(rd.x * rd.x + rd.z * rd.z, 1e-12f));
      vhx = rd.x * r; vhz = rd.z * r;
    }
    V3 wf = wave_field(f, surf.x, surf.z, px_world, vhx, vhz, kk, aniso, 1.0f);
    nup = normalize(v3(-wf.x, 1.0f, -wf.y));   // wave_normal
  }
  float cos_i = clampf(dot(rd, nup), 1e-3f, 1.0f);
  float sin2_t = VM_WATER_IOR * VM_WATER_IOR * (1.0f - cos_i * cos_i);
  float fr = 1.0f;
  if (sin2_t < 1.0f) fr = schlick_f0(0.02f, sqrtf(1.0f - sin2_t));
  V3 below = underwater_body(w);
  V3 transmitted = mixv(above, underwater_body(w), s * 0.9f);
  return mixv(transmitted, below, fr * s);
}

// heat: resolve.wgsl:36-44, the heat-map view of a FLAG_HEATMAP frame
// (resolve.wgsl:1389-1394): every pixel's summed march iterations / 300
int or_resolve_heat(const or_world* o, const uint32_t* dbg, float* rgba, uint64_t pix_begin, uint64_t pix_end) {
  const vm_frame& f = *o->frame;
  const uint64_t npix = (uint64_t)f.res[0] * f.res[1];
  if (pix_end > npix) pix_end = npix;
  for (uint64_t pix = pix_begin; pix < pix_end; ++pix) {
    float t = clampf((float)dbg[pix] / 300.0f, 0.0f, 1.0f);
    float c[3] = {smoothstep(0.35f, 0.85f, t), smoothstep(0.0f, 0.45f, t) - smoothstep(0.65f, 1.0f, t),
                  1.0f - smoothstep(0.0f, 0.45f, t)};
    float* out = rgba + 4 * (pix - pix_begin);
    for (int ch = 0; ch < 3; ++ch) out[ch] = powf(c[ch], 2.2f);
    out[3] = 1.0f;
  }
  return 0;
}

int or_resolve(const or_world* o, const or_look* lk, const uint64_t* vis, const float* sun_vis, float* rgba,
               uint64_t pix_begin, uint64_t pix_end, int threads) {
  World w = mk(o);
  const vm_frame& f = *w.f;
  size_t texels = 0;
  for (uint32_t m = 0; m < 4; ++m) texels += (size_t)lk->layers * (16u >> m) * (16u >> m);
  std::vector<float> lin(texels * 4);
  for (size_t i = 0; i < texels; ++i) {
    for (int ch = 0; ch < 3; ++ch) lin[i * 4 + ch] = srgb_to_linear(lk->atlas_srgb[i * 4 + ch]);
    lin[i * 4 + 3] = (float)lk->atlas_srgb[i * 4 + 3] / 255.0f;
  }
  Look L;
  L.atlas = lin.data(); L.layers = lk->layers;
  L.faces = lk->faces; L.n_faces = lk->n_faces;
  L.probes = lk->probes; L.shaft = lk->shaft; L.spec_hi = lk->spec_hi;
  for (uint32_t k = 0; k < 32; ++k) {
    float a = k < 24 ? 1.4398966328953218f - 0.26179938779914946f * (float)k
                     : 1.1780972450961724f - 0.7853981633974483f * (float)(k - 24);
    L.grad_cos[k] = cosf(a);
    L.grad_sin[k] = sinf(a);
  }
  const uint64_t npix = (uint64_t)f.res[0] * f.res[1];
  if (pix_end > npix) pix_end = npix;
  if (threads > 0) omp_set_num_threads(threads);
  V3 cam = ld3(f.cam_pos);
#pragma omp parallel for schedule(dynamic, 256)
  for (int64_t pi = (int64_t)pix_begin; pi < (int64_t)pix_end; ++pi) {
    uint64_t pix = (uint64_t)pi;
    uint32_t px = (uint32_t)(pix % f.res[0]), py = (uint32_t)(pix / f.res[0]);
    V3 rd = ray_dir(f, (float)px + 0.5f, (float)py + 0.5f);
    uint64_t key = vis[pix];
    V3 color;
    float* out = rgba + 4 * (pix - pix_begin);
    const bool underwater = (f.flags & VM_FLAG_UNDERWATER) != 0u;
    float dist = f.far_;
    if (key == 0) {
      float shaft = underwater ? 1.0f : sun_shaft(f, L, cam, rd, f.far_, 1.0f, px, py);
      color = sky_color(f, L, cam, rd, 0.0f, shaft);
    } else {
      uint32_t nid = key_nid(key), ci = key_ci(key);
      U3 v = key_voxel(key), micro = key_micro(key);
      float t = hit_t(w, ci, v, micro, nid, rd);
      V3 hit = add(cam, muls(rd, t));
      uint32_t id = block_at(w, ci, v);
      if (id == VM_WATER) {
        // shade_water_sec (resolve.wgsl:1247-1259), or shade_water without SPEC_WATER_SEC
        bool shared = (lk->spec_hi & HI_WATER_SEC) != 0u &&
                      !((w.spec & VM_SPEC_WATER_REPAIR) != 0u && !water_share_safe(w, vis, 1u, px, py, nid, hit, t));
        if (shared) {
          WaterCtx x = water_ctx(w, L, ci, v, nid, hit, rd, t);
          F4 leg_r, leg_m;
          water_sec_legs(w, L, vis, 1u, px >> 1, py >> 1, &leg_r, &leg_m);
          color = water_compose(f, L, x, leg_r, leg_m);
        } else {
          color = shade_water(w, L, ci, v, nid, hit, rd, t);
        }
      } else if (glass_leg(w, id)) {
        color = shade_glass(w, L, ci, v, nid, hit, rd, t);
      } else {
        color = shade_hit(w, L, ci, v, id, nid, hit, rd, t, f.shadow_dist, true, true, sun_vis[pix]);
      }
      dist = t;
      float wet = underwater && surface_debug(L) == 0u ? water_path(f, t, rd) : 0.0f;
      float alpha = 1.0f - transmittance_from(f, cam.y + wet * rd.y, t - wet, rd);
      float shaft = underwater ? 1.0f : sun_shaft(f, L, cam, rd, t, alpha, px, py);
      if (surface_debug(L) == 0u) color = mixv(color, sky_base(f, L, rd, shaft), alpha);
    }
    if (underwater && surface_debug(L) == 0u) {
      color = surface_from_below(w, color, rd, dist);
      color = water_medium(f, color, water_path(f, dist, rd), underwater_body(w));
    }
    out[0] = color.x; out[1] = color.y; out[2] = color.z; out[3] = 1.0f;
  }
  return g_err.load();
}

}  // extern "C"
