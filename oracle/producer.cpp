// Oracle-side world producer -- test infrastructure, never part of the product.
//
// A restatement of the engine's CPU producers: the dense -> 64-tree encoder
// build_local (src/voxel/tree.rs:89-204) with encode_leaf
// (src/voxel/attributes.rs:90-139), the run pools with content dedup and
// reference counts (src/voxel/geometry.rs:64-219), the word pool
// (src/voxel/attributes.rs:6-88), World::insert_local / remove / get_block /
// l1_node (src/voxel/world.rs:63-277), and the per-frame chunk list, grid and
// GpuFrame fill (src/render/mod.rs:82-138,1447-1564,1640-1707; Frustum
// src/math.rs:74-117; camera basis src/player.rs:122-126, src/scene.rs:334-339;
// pairs_for mod.rs:27-30; halton_jitter src/math.rs:119-134).
//
// It gives the oracle march its own inputs, built independently of the
// product's world store (voxelcraft_menu_b200/csrc/store.cpp), so that the
// parity tests and the CPU reference arm of the benchmark never go through
// the product library.  The synthetic terrain comes from recipe.h, the
// workload's definition shared by both producers.  Exported as orw_*.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include "voxelcraft_menu_b200/csrc/vm_types.h"
#include "voxelcraft_menu_b200/csrc/recipe.h"
#include "include/voxmarch_world.h"

namespace orp {

struct Inner {          // src/voxel/geometry.rs:11-18 (16 bytes, = vec4<u32>)
  uint64_t mask = 0;
  uint32_t run_ptr = 0;
  uint32_t leaf_prefix = 0;
  bool is_full() const { return (run_ptr & VM_FULL_BIT) != 0; }
  bool is_empty() const { return mask == 0; }
  uint32_t run() const { return run_ptr & ~VM_FULL_BIT; }
  uint32_t count() const { return (uint32_t)__builtin_popcountll(mask); }
  static Inner full(uint32_t leaf_prefix) { Inner n; n.mask = ~0ull; n.run_ptr = VM_FULL_BIT; n.leaf_prefix = leaf_prefix; return n; }
  bool operator==(const Inner& o) const { return mask == o.mask && run_ptr == o.run_ptr && leaf_prefix == o.leaf_prefix; }
};
static_assert(sizeof(Inner) == 16, "Inner is one vec4<u32>");

struct LocalL1 {        // src/voxel/tree.rs:37-46
  uint64_t mask = 0;
  uint32_t leaf_start = 0;
  uint32_t leaf_prefix = 0;
  bool full = false;
  uint8_t water_line = 0;
};

struct LocalTree {      // src/voxel/tree.rs:48-77
  uint64_t root_mask = 0, dry_mask = 0;
  std::vector<LocalL1> l1;
  std::vector<uint64_t> leaves;
  std::vector<uint32_t> attrs, palette;
  int32_t uniform = -1;
  bool has_water = false, has_foliage = false, has_cutout = false, has_glass = false, has_emitter = false;
  uint32_t emitters = 0, solid_count = 0, leaf_count = 0;
  uint8_t aabb_min[3] = {0, 0, 0}, aabb_max[3] = {0, 0, 0};
};

LocalTree build_local(const uint16_t* dense);   // dense index x | z<<6 | y<<12

// Run pool with content dedup and refcounts (src/voxel/geometry.rs:64-219).
template <class T>
struct RunPool {
  std::vector<T> data;
  std::vector<uint32_t> refs;
  std::vector<uint8_t> lens;
  std::unordered_multimap<uint64_t, uint32_t> table;
  std::vector<std::vector<uint32_t>> free_lists = std::vector<std::vector<uint32_t>>(65);
  uint64_t live_elems = 0, referenced_elems = 0;
  std::pair<uint32_t, bool> intern(const T* run, uint32_t len);
  void add_ref(uint32_t off);
  bool release(uint32_t off);
 private:
  uint32_t alloc(uint32_t len);
};

// Power-of-two size-class word pool (src/voxel/attributes.rs:6-88).
struct WordPool {
  std::vector<uint32_t> data;
  std::vector<std::vector<uint32_t>> free_lists = std::vector<std::vector<uint32_t>>(32);
  uint64_t used_words = 0;
  uint32_t alloc(size_t len);
  void free(uint32_t off, size_t len);
  uint32_t alloc_write(const std::vector<uint32_t>& w);
};

struct ChunkKey {
  uint8_t lod = 0;
  int32_t x = 0, y = 0, z = 0;
  bool operator==(const ChunkKey& o) const { return lod == o.lod && x == o.x && y == o.y && z == o.z; }
  int32_t size() const { return 64 << lod; }
  int32_t voxel_size() const { return 1 << lod; }
};
struct ChunkKeyHash {
  size_t operator()(const ChunkKey& k) const {
    uint64_t h = (uint64_t)(uint32_t)k.x * 0x9E3779B97F4A7C15ull ^ (uint64_t)(uint32_t)k.y * 0xC2B2AE3D27D4EB4Full ^
                 (uint64_t)(uint32_t)k.z * 0x165667B19E3779F9ull ^ k.lod;
    return (size_t)(h ^ (h >> 29));
  }
};

struct ChunkRecord {    // src/voxel/chunk.rs:63-93 (march-relevant fields)
  ChunkKey key;
  Inner root;
  bool attr_uniform = true;
  uint32_t attr_value = 0;      // uniform id or table base
  uint32_t attr_len = 0;
  std::vector<std::pair<uint32_t, size_t>> regions;
  int32_t aabb_min[3] = {0, 0, 0}, aabb_max[3] = {0, 0, 0};
  uint32_t solid_count = 0, leaf_count = 0;
  bool has_water = false, has_foliage = false, has_cutout = false, has_glass = false, has_emitter = false;
  uint64_t dry_mask = 0;
  uint32_t emitters = 0;
  uint64_t order = 0;           // insertion order (render-set order)
  float fade = 1.0f;            // the render item's LOD cross-fade (src/lod.rs:56-80)
};

struct World {          // src/voxel/world.rs:16-29
  RunPool<uint64_t> leaves;
  RunPool<Inner> inners;
  WordPool bricks;
  std::unordered_map<ChunkKey, ChunkRecord, ChunkKeyHash> chunks;
  uint64_t next_order = 0;
  void insert_local(const ChunkKey& key, const LocalTree& t);
  bool remove_chunk(const ChunkKey& key);
  uint16_t get_block(int32_t x, int32_t y, int32_t z) const;
  bool l1_node(const Inner& root, uint32_t l1b, Inner* out) const;
 private:
  Inner make_root(uint64_t root_mask, const std::vector<Inner>& run);
  void release_root(const Inner& root);
};

}  // namespace orp

namespace orp {

// ---------------------------------------------------------------------------
// build_local: src/voxel/tree.rs:89-204 (dense 64^3 -> LocalTree)
// ---------------------------------------------------------------------------
static inline uint32_t cell_bit(uint32_t x, uint32_t y, uint32_t z) { return x | (y << 2) | (z << 4); }
static inline size_t dense_index(uint32_t x, uint32_t y, uint32_t z) { return x | (z << 6) | (y << 12); }

static bool is_foliage(uint16_t id) { return id == VM_TALL_GRASS || id == VM_GRASS_TALL || id == VM_REEDS; }
static bool is_cutout(uint16_t id) { return id == VM_LEAVES || id == VM_PINE_LEAVES; }
static bool is_glass(uint16_t id) { return id == VM_GLASS; }
static bool is_emitter(uint16_t id) {
  return id == VM_GLOWSTONE || id == VM_AMBER_LAMP || id == VM_AZURE_LAMP || id == VM_VERDANT_LAMP;
}

static uint32_t bits_for(size_t n) {     // src/voxel/attributes.rs:90-97
  if (n <= 2) return 1;
  if (n <= 4) return 2;
  if (n <= 16) return 4;
  return 8;
}

// encode_leaf: src/voxel/attributes.rs:99-139
static uint32_t encode_leaf(const uint16_t* ids, uint64_t present, std::vector<uint32_t>& out) {
  uint16_t pal[64];
  size_t n = 0;
  for (int i = 0; i < 64; ++i) {
    if ((present >> i) & 1) {
      uint16_t id = ids[i];
      bool seen = false;
      for (size_t k = 0; k < n; ++k) if (pal[k] == id) { seen = true; break; }
      if (!seen) pal[n++] = id;
    }
  }
  if (n <= 1) return VM_UNIFORM_BIT | pal[0];
  uint32_t bits = bits_for(n);
  uint32_t off = (uint32_t)out.size();
  out.push_back((uint32_t)n | (bits << 8));
  for (size_t w = 0; w < (n + 1) / 2; ++w) {
    uint32_t lo = pal[2 * w];
    uint32_t hi = 2 * w + 1 < n ? pal[2 * w + 1] : 0;
    out.push_back(lo | (hi << 16));
  }
  size_t idx_words = (64 * bits) / 32;
  size_t idx_base = out.size();
  out.resize(idx_base + idx_words, 0);
  for (int i = 0; i < 64; ++i) {
    if (!((present >> i) & 1)) continue;
    uint32_t idx = 0;
    while (pal[idx] != ids[i]) ++idx;
    uint32_t bitpos = (uint32_t)i * bits;
    out[idx_base + (bitpos >> 5)] |= idx << (bitpos & 31);
  }
  return off;
}

LocalTree build_local(const uint16_t* dense) {
  LocalTree t;
  uint16_t ids[64] = {0};
  int first = -1;
  bool all_same = true;
  uint8_t amin[3] = {64, 64, 64}, amax[3] = {0, 0, 0};
  for (uint32_t l1z = 0; l1z < 4; ++l1z)
    for (uint32_t l1y = 0; l1y < 4; ++l1y)
      for (uint32_t l1x = 0; l1x < 4; ++l1x) {
        uint64_t l1mask = 0;
        uint32_t leaf_start = (uint32_t)t.leaves.size();
        bool all_full = true, l1_dry = false;
        uint32_t max_nonwater_y = 0;
        for (uint32_t lz = 0; lz < 4; ++lz)
          for (uint32_t ly = 0; ly < 4; ++ly)
            for (uint32_t lx = 0; lx < 4; ++lx) {
              uint64_t m = 0;
              uint32_t bx = l1x * 16 + lx * 4, by = l1y * 16 + ly * 4, bz = l1z * 16 + lz * 4;
              for (uint32_t vz = 0; vz < 4; ++vz)
                for (uint32_t vy = 0; vy < 4; ++vy) {
                  size_t row = dense_index(bx, by + vy, bz + vz);
                  for (uint32_t vx = 0; vx < 4; ++vx) {
                    uint16_t id = dense[row + vx];
                    if (id == VM_AIR) continue;
                    uint32_t vb = cell_bit(vx, vy, vz);
                    m |= 1ull << vb;
                    ids[vb] = id;
                    t.has_water |= id == VM_WATER;
                    l1_dry |= id != VM_WATER;
                    if (id != VM_WATER) max_nonwater_y = std::max(max_nonwater_y, ly * 4 + vy);
                    t.has_foliage |= is_foliage(id);
                    t.has_cutout |= is_cutout(id);
                    t.has_glass |= is_glass(id);
                    bool e = is_emitter(id);
                    t.has_emitter |= e;
                    t.emitters += e;
                    if (first < 0) first = id;
                    else if (first != id) all_same = false;
                    uint8_t x = (uint8_t)(bx + vx), y = (uint8_t)(by + vy), z = (uint8_t)(bz + vz);
                    amin[0] = std::min(amin[0], x); amin[1] = std::min(amin[1], y); amin[2] = std::min(amin[2], z);
                    amax[0] = std::max<uint8_t>(amax[0], x + 1);
                    amax[1] = std::max<uint8_t>(amax[1], y + 1);
                    amax[2] = std::max<uint8_t>(amax[2], z + 1);
                  }
                }
              if (m != 0) {
                l1mask |= 1ull << cell_bit(lx, ly, lz);
                t.leaves.push_back(m);
                t.attrs.push_back(encode_leaf(ids, m, t.palette));
                if (m != ~0ull) all_full = false;
              } else {
                all_full = false;
              }
            }
        if (l1mask != 0) {
          if (l1_dry) t.dry_mask |= 1ull << cell_bit(l1x, l1y, l1z);
          bool full = all_full && l1mask == ~0ull;
          if (full) t.leaves.resize(leaf_start);
          LocalL1 n;
          n.mask = l1mask;
          n.leaf_start = leaf_start;
          n.leaf_prefix = t.leaf_count;
          n.full = full;
          n.water_line = l1_dry ? (uint8_t)max_nonwater_y : 15;
          t.l1.push_back(n);
          t.leaf_count += (uint32_t)__builtin_popcountll(l1mask);
          t.root_mask |= 1ull << cell_bit(l1x, l1y, l1z);
        }
      }
  uint32_t solid = 0;
  for (uint64_t m : t.leaves) solid += (uint32_t)__builtin_popcountll(m);
  for (const LocalL1& n : t.l1) if (n.full) solid += 4096;
  t.solid_count = solid;
  if (first >= 0 && all_same) {
    t.uniform = first;
    t.attrs.clear();
    t.palette.clear();
  }
  if (t.solid_count > 0) {
    memcpy(t.aabb_min, amin, 3);
    memcpy(t.aabb_max, amax, 3);
  }
  return t;
}

// ---------------------------------------------------------------------------
// RunPool / WordPool
// ---------------------------------------------------------------------------
template <class T>
static uint64_t hash_run(const T* run, uint32_t len) {
  uint64_t h = 1469598103934665603ull ^ len;
  const uint8_t* p = reinterpret_cast<const uint8_t*>(run);
  for (size_t i = 0; i < (size_t)len * sizeof(T); ++i) { h ^= p[i]; h *= 1099511628211ull; }
  return h;
}

template <class T>
uint32_t RunPool<T>::alloc(uint32_t len) {
  if (!free_lists[len].empty()) { uint32_t off = free_lists[len].back(); free_lists[len].pop_back(); return off; }
  uint32_t off = (uint32_t)data.size();
  data.resize(off + len, T{});
  refs.resize(off + len, 0);
  lens.resize(off + len, 0);
  return off;
}

template <class T>
std::pair<uint32_t, bool> RunPool<T>::intern(const T* run, uint32_t len) {
  uint64_t h = hash_run(run, len);
  auto range = table.equal_range(h);
  for (auto it = range.first; it != range.second; ++it) {
    uint32_t o = it->second;
    if (lens[o] == len && std::equal(run, run + len, data.begin() + o)) {
      refs[o] += 1;
      referenced_elems += len;
      return {o, false};
    }
  }
  uint32_t off = alloc(len);
  std::copy(run, run + len, data.begin() + off);
  refs[off] = 1;
  lens[off] = (uint8_t)len;
  table.emplace(h, off);
  live_elems += len;
  referenced_elems += len;
  return {off, true};
}

template <class T>
void RunPool<T>::add_ref(uint32_t off) {
  refs[off] += 1;
  referenced_elems += lens[off];
}

template <class T>
bool RunPool<T>::release(uint32_t off) {
  uint32_t len = lens[off];
  refs[off] -= 1;
  referenced_elems -= len;
  if (refs[off] != 0) return false;
  uint64_t h = hash_run(data.data() + off, len);
  auto range = table.equal_range(h);
  for (auto it = range.first; it != range.second; ++it)
    if (it->second == off) { table.erase(it); break; }
  free_lists[len].push_back(off);
  live_elems -= len;
  return true;
}

template struct RunPool<uint64_t>;
template struct RunPool<Inner>;

static std::pair<int, size_t> class_of(size_t len) {
  size_t size = std::max<size_t>(len, 4);
  size_t p = 1;
  while (p < size) p <<= 1;
  return {__builtin_ctzll(p), p};
}

uint32_t WordPool::alloc(size_t len) {
  auto [cls, size] = class_of(len);
  used_words += size;
  if (!free_lists[cls].empty()) { uint32_t off = free_lists[cls].back(); free_lists[cls].pop_back(); return off; }
  uint32_t off = (uint32_t)data.size();
  data.resize(off + size, 0);
  return off;
}
void WordPool::free(uint32_t off, size_t len) {
  auto [cls, size] = class_of(len);
  used_words -= size;
  free_lists[cls].push_back(off);
}
uint32_t WordPool::alloc_write(const std::vector<uint32_t>& w) {
  uint32_t off = alloc(w.size());
  std::copy(w.begin(), w.end(), data.begin() + off);
  return off;
}

// ---------------------------------------------------------------------------
// World: src/voxel/world.rs:63-277
// ---------------------------------------------------------------------------
void World::insert_local(const ChunkKey& key, const LocalTree& t) {
  if (chunks.count(key)) remove_chunk(key);
  std::vector<Inner> run;
  run.reserve(t.l1.size());
  std::vector<uint32_t> temp;
  for (const LocalL1& n : t.l1) {
    uint32_t prefix = n.leaf_prefix | ((uint32_t)n.water_line << 28);
    if (n.full) {
      run.push_back(Inner::full(prefix));
    } else {
      uint32_t cnt = (uint32_t)__builtin_popcountll(n.mask);
      auto [off, fresh] = leaves.intern(t.leaves.data() + n.leaf_start, cnt);
      (void)fresh;
      temp.push_back(off);
      Inner in;
      in.mask = n.mask;
      in.run_ptr = off;
      in.leaf_prefix = prefix;
      run.push_back(in);
    }
  }
  Inner root = make_root(t.root_mask, run);
  for (uint32_t off : temp) leaves.release(off);

  ChunkRecord rec;
  rec.key = key;
  rec.root = root;
  if (t.uniform >= 0) {
    rec.attr_uniform = true; rec.attr_value = (uint32_t)t.uniform;
  } else if (t.attrs.empty()) {
    rec.attr_uniform = true; rec.attr_value = VM_AIR;
  } else {
    uint32_t pal_base = 0;
    if (!t.palette.empty()) {
      pal_base = bricks.alloc_write(t.palette);
      rec.regions.push_back({pal_base, t.palette.size()});
    }
    std::vector<uint32_t> table(t.attrs.size());
    for (size_t i = 0; i < t.attrs.size(); ++i) {
      uint32_t e = t.attrs[i];
      table[i] = (e & VM_UNIFORM_BIT) ? e : e + pal_base;
    }
    rec.attr_uniform = false;
    rec.attr_value = bricks.alloc_write(table);
    rec.attr_len = (uint32_t)table.size();
  }
  for (int i = 0; i < 3; ++i) { rec.aabb_min[i] = t.aabb_min[i]; rec.aabb_max[i] = t.aabb_max[i]; }
  rec.solid_count = t.solid_count;
  rec.leaf_count = t.leaf_count;
  rec.has_water = t.has_water;
  rec.dry_mask = t.dry_mask;
  rec.has_foliage = t.has_foliage;
  rec.has_cutout = t.has_cutout;
  rec.has_glass = t.has_glass;
  rec.has_emitter = t.has_emitter;
  rec.emitters = t.emitters;
  rec.order = next_order++;
  chunks[key] = std::move(rec);
}

Inner World::make_root(uint64_t root_mask, const std::vector<Inner>& run) {
  if (run.empty()) return Inner{};
  bool all_full = run.size() == 64;
  for (const Inner& n : run) all_full = all_full && n.is_full();
  if (all_full) return Inner::full(0);
  auto [off, fresh] = inners.intern(run.data(), (uint32_t)run.size());
  if (fresh)
    for (const Inner& n : run) if (!n.is_full()) leaves.add_ref(n.run());
  Inner r;
  r.mask = root_mask;
  r.run_ptr = off;
  r.leaf_prefix = 0;
  return r;
}

void World::release_root(const Inner& root) {
  if (root.is_full() || root.is_empty()) return;
  std::vector<Inner> nodes(inners.data.begin() + root.run(), inners.data.begin() + root.run() + root.count());
  if (inners.release(root.run()))
    for (const Inner& n : nodes) if (!n.is_full()) leaves.release(n.run());
}

bool World::remove_chunk(const ChunkKey& key) {
  auto it = chunks.find(key);
  if (it == chunks.end()) return false;
  ChunkRecord rec = std::move(it->second);
  chunks.erase(it);
  release_root(rec.root);
  if (!rec.attr_uniform) bricks.free(rec.attr_value, rec.attr_len);
  for (auto& r : rec.regions) bricks.free(r.first, r.second);
  return true;
}

bool World::l1_node(const Inner& root, uint32_t l1b, Inner* out) const {   // world.rs:225-234
  if (!((root.mask >> l1b) & 1)) return false;
  if (root.is_full()) { *out = Inner::full(l1b * 64); return true; }
  uint32_t below = (uint32_t)__builtin_popcountll(root.mask & ((1ull << l1b) - 1));
  *out = inners.data[root.run() + below];
  return true;
}

static uint16_t decode_leaf(const std::vector<uint32_t>& words, uint32_t entry, uint32_t vb) {
  if (entry & VM_UNIFORM_BIT) return (uint16_t)entry;        // attributes.rs:141-156
  uint32_t hdr = words[entry];
  uint32_t n = hdr & 0xFF, bits = (hdr >> 8) & 0xFF;
  size_t idx_base = entry + 1 + (n + 1) / 2;
  uint32_t bitpos = vb * bits;
  uint32_t w = words[idx_base + (bitpos >> 5)];
  uint32_t idx = (w >> (bitpos & 31)) & ((1u << bits) - 1);
  uint32_t pw = words[entry + 1 + idx / 2];
  return (uint16_t)(pw >> ((idx & 1) * 16));
}

uint16_t World::get_block(int32_t x, int32_t y, int32_t z) const {   // world.rs:258-277
  if (y < 0 || y >= 512) return VM_AIR;
  ChunkKey k;
  k.lod = 0; k.x = x >> 6; k.y = y >> 6; k.z = z >> 6;
  auto it = chunks.find(k);
  if (it == chunks.end()) return VM_AIR;
  const ChunkRecord& rec = it->second;
  uint32_t lx = x & 63, ly = y & 63, lz = z & 63;
  Inner l1;
  if (!l1_node(rec.root, cell_bit(lx >> 4, ly >> 4, lz >> 4), &l1)) return VM_AIR;
  uint32_t lfb = cell_bit((lx >> 2) & 3, (ly >> 2) & 3, (lz >> 2) & 3);
  uint64_t m = 0;
  if ((l1.mask >> lfb) & 1) {
    if (l1.is_full()) m = ~0ull;
    else m = leaves.data[l1.run() + (uint32_t)__builtin_popcountll(l1.mask & ((1ull << lfb) - 1))];
  }
  uint32_t vb = cell_bit(lx & 3, ly & 3, lz & 3);
  if (!((m >> vb) & 1)) return VM_AIR;
  if (rec.attr_uniform) return (uint16_t)rec.attr_value;
  uint32_t li = (l1.leaf_prefix & VM_PREFIX_MASK) + (uint32_t)__builtin_popcountll(l1.mask & ((1ull << lfb) - 1));
  return decode_leaf(bricks.data, bricks.data[rec.attr_value + li], vb);
}

}  // namespace orp


// ===========================================================================
// Synthetic worlds, chunk list, frame; C ABI (include/voxmarch_world.h)
// ===========================================================================
using namespace orp;

struct orw_world {
  World w;
  std::mutex mu;
  std::string err;
};

namespace {

// glam-style normalize (v * (1/length)) used by the engine's host math
struct H3 { float x, y, z; };
inline H3 hnorm(H3 v, H3 fallback) {
  float l = sqrtf(v.x * v.x + v.y * v.y + v.z * v.z);
  float r = 1.0f / l;
  if (!std::isfinite(r) || r <= 0.0f) return fallback;
  return {v.x * r, v.y * r, v.z * r};
}
inline H3 hcross(H3 a, H3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline float hdot(H3 a, H3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

}  // namespace

extern "C" {

orw_world* orw_create(void) { return new orw_world(); }
void orw_destroy(orw_world* w) { delete w; }

int orw_insert_dense(orw_world* w, uint8_t lod, int32_t x, int32_t y, int32_t z, const uint16_t* dense) {
  if (!w || !dense) return 1;
  LocalTree t = build_local(dense);
  ChunkKey k; k.lod = lod; k.x = x; k.y = y; k.z = z;
  std::lock_guard<std::mutex> g(w->mu);
  w->w.insert_local(k, t);
  return 0;
}

int orw_build_tree(const uint16_t* dense, uint32_t palette_cap, vm_tree_info* info, vm_tree_l1* l1,
                   uint64_t* leaves, uint32_t* attrs, uint32_t* palette) {
  if (!dense || !info || !l1 || !leaves || !attrs || (palette_cap && !palette)) return 1;
  const LocalTree t = build_local(dense);
  memset(info, 0, sizeof *info);
  info->root_mask = t.root_mask;
  info->dry_mask = t.dry_mask;
  info->uniform = t.uniform;
  info->flags = (t.has_water ? VM_TREE_WATER : 0u) | (t.has_foliage ? VM_TREE_FOLIAGE : 0u) |
                (t.has_cutout ? VM_TREE_CUTOUT : 0u) | (t.has_glass ? VM_TREE_GLASS : 0u) |
                (t.has_emitter ? VM_TREE_EMITTER : 0u);
  info->emitters = t.emitters;
  info->solid_count = t.solid_count;
  info->leaf_count = t.leaf_count;
  info->n_l1 = (uint32_t)t.l1.size();
  info->n_leaves = (uint32_t)t.leaves.size();
  info->n_attrs = (uint32_t)t.attrs.size();
  info->n_palette = (uint32_t)t.palette.size();
  memcpy(info->aabb_min, t.aabb_min, 3);
  memcpy(info->aabb_max, t.aabb_max, 3);
  for (size_t i = 0; i < t.l1.size(); ++i) {
    memset(&l1[i], 0, sizeof l1[i]);
    l1[i].mask = t.l1[i].mask;
    l1[i].leaf_start = t.l1[i].leaf_start;
    l1[i].leaf_prefix = t.l1[i].leaf_prefix;
    l1[i].full = t.l1[i].full ? 1 : 0;
    l1[i].water_line = t.l1[i].water_line;
  }
  if (!t.leaves.empty()) memcpy(leaves, t.leaves.data(), t.leaves.size() * 8);
  if (!t.attrs.empty()) memcpy(attrs, t.attrs.data(), t.attrs.size() * 4);
  if (t.palette.size() > palette_cap) info->flags |= VM_TREE_PALETTE_OVERFLOW;
  const size_t np = std::min<size_t>(t.palette.size(), palette_cap);
  if (np) memcpy(palette, t.palette.data(), np * 4);
  return 0;
}

int orw_insert_tree(orw_world* w, uint8_t lod, int32_t x, int32_t y, int32_t z, const vm_tree_info* info,
                    const vm_tree_l1* l1, const uint64_t* leaves, const uint32_t* attrs, const uint32_t* palette) {
  if (!w || !info || (info->flags & VM_TREE_PALETTE_OVERFLOW) || info->n_l1 > VM_TREE_L1 ||
      info->n_leaves > VM_TREE_LEAVES || info->n_attrs > VM_TREE_LEAVES)
    return 1;
  LocalTree t;
  t.root_mask = info->root_mask;
  t.dry_mask = info->dry_mask;
  t.uniform = info->uniform;
  t.has_water = (info->flags & VM_TREE_WATER) != 0u;
  t.has_foliage = (info->flags & VM_TREE_FOLIAGE) != 0u;
  t.has_cutout = (info->flags & VM_TREE_CUTOUT) != 0u;
  t.has_glass = (info->flags & VM_TREE_GLASS) != 0u;
  t.has_emitter = (info->flags & VM_TREE_EMITTER) != 0u;
  t.emitters = info->emitters;
  t.solid_count = info->solid_count;
  t.leaf_count = info->leaf_count;
  memcpy(t.aabb_min, info->aabb_min, 3);
  memcpy(t.aabb_max, info->aabb_max, 3);
  for (uint32_t i = 0; i < info->n_l1; ++i) {
    LocalL1 n;
    n.mask = l1[i].mask;
    n.leaf_start = l1[i].leaf_start;
    n.leaf_prefix = l1[i].leaf_prefix;
    n.full = l1[i].full != 0;
    n.water_line = l1[i].water_line;
    if (!n.full && (uint64_t)n.leaf_start + (uint32_t)__builtin_popcountll(n.mask) > info->n_leaves) return 1;
    t.l1.push_back(n);
  }
  t.leaves.assign(leaves, leaves + info->n_leaves);
  t.attrs.assign(attrs, attrs + info->n_attrs);
  t.palette.assign(palette, palette + info->n_palette);
  ChunkKey k; k.lod = lod; k.x = x; k.y = y; k.z = z;
  std::lock_guard<std::mutex> g(w->mu);
  w->w.insert_local(k, t);
  return 0;
}

int orw_remove(orw_world* w, uint8_t lod, int32_t x, int32_t y, int32_t z) {
  ChunkKey k; k.lod = lod; k.x = x; k.y = y; k.z = z;
  return w->w.remove_chunk(k) ? 0 : 1;
}

uint32_t orw_get_block(const orw_world* w, int32_t x, int32_t y, int32_t z) { return w->w.get_block(x, y, z); }

// The render item's fade (src/lod.rs:56-80): 1 solid; f in (0, 1) a fading-in
// child, -f its fading-out parent.
int orw_set_fade(orw_world* w, uint8_t lod, int32_t x, int32_t y, int32_t z, float fade) {
  ChunkKey k; k.lod = lod; k.x = x; k.y = y; k.z = z;
  auto it = w->w.chunks.find(k);
  if (it == w->w.chunks.end()) return 1;
  it->second.fade = fade;
  return 0;
}

int orw_get_chunk_info(const orw_world* w, uint8_t lod, int32_t x, int32_t y, int32_t z, vmw_chunk_info* out) {
  ChunkKey k; k.lod = lod; k.x = x; k.y = y; k.z = z;
  auto it = w->w.chunks.find(k);
  if (it == w->w.chunks.end()) return 1;
  const ChunkRecord& r = it->second;
  memset(out, 0, sizeof *out);
  out->root[0] = (uint32_t)r.root.mask; out->root[1] = (uint32_t)(r.root.mask >> 32);
  out->root[2] = r.root.run_ptr; out->root[3] = r.root.leaf_prefix;
  out->attr_uniform = r.attr_uniform; out->attr_value = r.attr_value;
  for (int i = 0; i < 3; ++i) { out->aabb_min[i] = r.aabb_min[i]; out->aabb_max[i] = r.aabb_max[i]; }
  out->solid_count = r.solid_count; out->leaf_count = r.leaf_count;
  out->dry_mask = r.dry_mask;
  out->has_water = r.has_water; out->has_foliage = r.has_foliage; out->has_cutout = r.has_cutout;
  out->has_glass = r.has_glass; out->has_emitter = r.has_emitter;
  return 0;
}

int orw_l1_node(const orw_world* w, uint8_t lod, int32_t x, int32_t y, int32_t z, uint32_t l1b, uint32_t* out4) {
  ChunkKey k; k.lod = lod; k.x = x; k.y = y; k.z = z;
  auto it = w->w.chunks.find(k);
  if (it == w->w.chunks.end()) return -1;
  Inner n;
  if (!w->w.l1_node(it->second.root, l1b, &n)) return 0;
  out4[0] = (uint32_t)n.mask; out4[1] = (uint32_t)(n.mask >> 32); out4[2] = n.run_ptr; out4[3] = n.leaf_prefix;
  return 1;
}

void orw_pool_stats(const orw_world* w, vmw_pool_stats_t* s) {
  s->n_inners = w->w.inners.data.size();
  s->n_leaves = w->w.leaves.data.size();
  s->n_bricks = w->w.bricks.data.size();
  s->live_inners = w->w.inners.live_elems;
  s->live_leaves = w->w.leaves.live_elems;
  s->referenced_inners = w->w.inners.referenced_elems;
  s->referenced_leaves = w->w.leaves.referenced_elems;
  s->used_words = w->w.bricks.used_words;
  s->n_chunks = w->w.chunks.size();
}

const uint32_t* orw_inners(const orw_world* w) { return reinterpret_cast<const uint32_t*>(w->w.inners.data.data()); }
const uint32_t* orw_leaves(const orw_world* w) { return reinterpret_cast<const uint32_t*>(w->w.leaves.data.data()); }
const uint32_t* orw_bricks(const orw_world* w) { return w->w.bricks.data.data(); }

int orw_generate(orw_world* w, const vmw_recipe* r) {
  if (!w || !r) return 1;
  for (int i = 0; i < 3; ++i) if (r->size[i] == 0 || r->size[i] % 64 != 0) return 2;
  const vmr::Heights hs = vmr::make_heights(*r);
  int32_t nx = r->size[0] / 64, ny = r->size[1] / 64, nz = r->size[2] / 64;
  int64_t total = (int64_t)nx * ny * nz;
  std::vector<LocalTree> trees((size_t)total);
#pragma omp parallel
  {
    std::vector<uint16_t> dense(64 * 64 * 64);
#pragma omp for schedule(dynamic, 1)
    for (int64_t i = 0; i < total; ++i) {
      int32_t cx = (int32_t)(i % nx), cy = (int32_t)((i / nx) % ny), cz = (int32_t)(i / ((int64_t)nx * ny));
      vmr::fill_chunk(*r, hs, cx, cy, cz, dense.data());
      trees[i] = build_local(dense.data());
    }
  }
  std::lock_guard<std::mutex> g(w->mu);
  for (int64_t i = 0; i < total; ++i) {
    ChunkKey k; k.lod = 0; k.x = (int32_t)(i % nx); k.y = (int32_t)((i / nx) % ny); k.z = (int32_t)(i / ((int64_t)nx * ny));
    w->w.insert_local(k, trees[i]);
  }
  return 0;
}

int orw_recipe_dense_all(const vmw_recipe* r, uint16_t* dense) {
  if (!r || !dense) return 1;
  for (int i = 0; i < 3; ++i) if (r->size[i] == 0 || r->size[i] % 64 != 0) return 2;
  const vmr::Heights hs = vmr::make_heights(*r);
  int32_t nx = r->size[0] / 64, ny = r->size[1] / 64, nz = r->size[2] / 64;
  int64_t total = (int64_t)nx * ny * nz;
#pragma omp parallel for schedule(dynamic, 1)
  for (int64_t i = 0; i < total; ++i) {
    int32_t cx = (int32_t)(i % nx), cy = (int32_t)((i / nx) % ny), cz = (int32_t)(i / ((int64_t)nx * ny));
    vmr::fill_chunk(*r, hs, cx, cy, cz, dense + (size_t)i * 64 * 64 * 64);
  }
  return 0;
}

int orw_recipe_dense(const vmw_recipe* r, int32_t cx, int32_t cy, int32_t cz, uint16_t* dense) {
  const vmr::Heights hs = vmr::make_heights(*r);
  vmr::fill_chunk(*r, hs, cx, cy, cz, dense);
  return 0;
}

int orw_recipe_dense_lod(const vmw_recipe* r, uint32_t lod, int32_t cx, int32_t cy, int32_t cz, uint16_t* dense) {
  if (!r || !dense || lod > 4) return 1;
  vmr::fill_chunk_lod(*r, lod, cx, cy, cz, dense);
  return 0;
}

int32_t orw_recipe_height(const vmw_recipe* r, int32_t x, int32_t z) {
  return (int32_t)floorf(r->base + r->amplitude * vmr::fbm((float)x, (float)z, *r));
}

// Camera basis: src/player.rs:122-126 (look_dir) and src/scene.rs:334-339.
void orw_camera_basis(float yaw, float pitch, float* fwd, float* right, float* up) {
  float sy = sinf(yaw), cy = cosf(yaw), sp = sinf(pitch), cp = cosf(pitch);
  H3 f = hnorm(H3{cy * cp, sp, sy * cp}, H3{0, 0, 0});
  H3 r = hnorm(hcross(f, H3{0, 1, 0}), H3{1, 0, 0});
  H3 u = hnorm(hcross(r, f), H3{0, 1, 0});
  fwd[0] = f.x; fwd[1] = f.y; fwd[2] = f.z;
  right[0] = r.x; right[1] = r.y; right[2] = r.z;
  up[0] = u.x; up[1] = u.y; up[2] = u.z;
}

uint32_t orw_pairs_for(uint32_t tiles_x, uint32_t tiles_y) {   // src/render/mod.rs:27-30
  uint64_t want = (uint64_t)tiles_x * tiles_y * VM_PAIRS_PER_TILE;
  want = std::max<uint64_t>(want, VM_MAX_PAIRS_FLOOR);
  want = std::min<uint64_t>(want, (uint64_t)UINT32_MAX / 2);
  return (uint32_t)want;
}

// Frame + chunk list + grid for one view (src/render/mod.rs:1447-1564 and the
// GpuFrame fill at 1640-1707; Frustum from src/math.rs:74-117).
int orw_build_view(const orw_world* wp, const vmw_camera* cam, vm_frame* frame, vm_chunk* chunks_out,
                   uint32_t cap, uint32_t* n_chunks_out, uint32_t* grid_out) {
  const World& w = wp->w;
  H3 fwd, right, up;
  if (cam->use_basis) {
    fwd = {cam->fwd[0], cam->fwd[1], cam->fwd[2]};
    right = {cam->right[0], cam->right[1], cam->right[2]};
    up = {cam->up[0], cam->up[1], cam->up[2]};
  } else {
    float f3[3], r3[3], u3[3];
    orw_camera_basis(cam->yaw, cam->pitch, f3, r3, u3);
    fwd = {f3[0], f3[1], f3[2]}; right = {r3[0], r3[1], r3[2]}; up = {u3[0], u3[1], u3[2]};
  }
  H3 pos{cam->pos[0], cam->pos[1], cam->pos[2]};
  float tan_half = tanf(cam->fov_y * 0.5f);
  float aspect = (float)cam->width / (float)cam->height;
  uint32_t gdim[3] = {VM_GRID_X, VM_GRID_Y, VM_GRID_Z};
  if (cam->grid_dim[0]) for (int i = 0; i < 3; ++i) gdim[i] = cam->grid_dim[i];
  int32_t ccx = (int32_t)floorf(pos.x / 64.0f), ccz = (int32_t)floorf(pos.z / 64.0f);
  int32_t gmin[3] = {ccx - (int32_t)gdim[0] / 2, 0, ccz - (int32_t)gdim[2] / 2};
  if (cam->grid_min_set) for (int i = 0; i < 3; ++i) gmin[i] = cam->grid_min[i];

  // frustum planes
  struct Plane { H3 n; float d; };
  auto mk = [&](H3 n) { n = hnorm(n, H3{0, 0, 0}); return Plane{n, -hdot(n, pos)}; };
  float hx = tan_half * aspect, hy = tan_half;
  Plane planes[6];
  planes[0] = mk(H3{fwd.x * hx + right.x, fwd.y * hx + right.y, fwd.z * hx + right.z});
  planes[1] = mk(H3{fwd.x * hx - right.x, fwd.y * hx - right.y, fwd.z * hx - right.z});
  planes[2] = mk(H3{fwd.x * hy + up.x, fwd.y * hy + up.y, fwd.z * hy + up.z});
  planes[3] = mk(H3{fwd.x * hy - up.x, fwd.y * hy - up.y, fwd.z * hy - up.z});
  planes[4] = mk(fwd);
  {
    H3 n{-fwd.x, -fwd.y, -fwd.z};
    H3 pf{pos.x + fwd.x * cam->far_, pos.y + fwd.y * cam->far_, pos.z + fwd.z * cam->far_};
    planes[5] = Plane{n, -hdot(n, pf)};
  }
  auto contains = [&](const float* mn, const float* mx) {
    for (const Plane& p : planes) {
      H3 q{p.n.x > 0 ? mx[0] : mn[0], p.n.y > 0 ? mx[1] : mn[1], p.n.z > 0 ? mx[2] : mn[2]};
      if (hdot(p.n, q) + p.d < 0.0f) return false;
    }
    return true;
  };
  auto grid_span = [&](const ChunkKey& k, int32_t* lo, int32_t* hi) {   // mod.rs:93-107
    int32_t span = 1 << k.lod;
    int32_t base[3] = {k.x * span - gmin[0], k.y * span - gmin[1], k.z * span - gmin[2]};
    for (int i = 0; i < 3; ++i) {
      lo[i] = std::max(base[i], 0);
      hi[i] = std::min(base[i] + span, (int32_t)gdim[i]);
    }
    return lo[0] < hi[0] && lo[1] < hi[1] && lo[2] < hi[2];
  };

  // render set in insertion order, skipping empty chunks
  std::vector<const ChunkRecord*> set;
  set.reserve(w.chunks.size());
  for (auto& kv : w.chunks) if (kv.second.solid_count > 0) set.push_back(&kv.second);
  std::sort(set.begin(), set.end(), [](const ChunkRecord* a, const ChunkRecord* b) { return a->order < b->order; });

  struct Item { float d; const ChunkRecord* r; float mn[3], mx[3]; };
  std::vector<Item> visible, offscreen;
  for (const ChunkRecord* r : set) {
    Item it;
    it.r = r;
    float o[3] = {(float)(r->key.x * r->key.size()), (float)(r->key.y * r->key.size()), (float)(r->key.z * r->key.size())};
    float vs = (float)r->key.voxel_size();
    for (int i = 0; i < 3; ++i) { it.mn[i] = o[i] + (float)r->aabb_min[i] * vs; it.mx[i] = o[i] + (float)r->aabb_max[i] * vs; }
    H3 dd{std::max(std::max(it.mn[0] - pos.x, pos.x - it.mx[0]), 0.0f),
          std::max(std::max(it.mn[1] - pos.y, pos.y - it.mx[1]), 0.0f),
          std::max(std::max(it.mn[2] - pos.z, pos.z - it.mx[2]), 0.0f)};
    it.d = sqrtf(hdot(dd, dd));
    int32_t lo[3], hi[3];
    if (contains(it.mn, it.mx)) visible.push_back(it);
    else if (cam->offscreen_shadows && grid_span(r->key, lo, hi)) offscreen.push_back(it);
  }
  auto by_d = [](const Item& a, const Item& b) { return a.d < b.d; };
  std::stable_sort(visible.begin(), visible.end(), by_d);
  uint32_t max_chunks = cam->max_chunks ? cam->max_chunks : VM_MAX_CHUNKS;
  if (visible.size() > max_chunks) visible.resize(max_chunks);
  std::stable_sort(offscreen.begin(), offscreen.end(), by_d);
  if (offscreen.size() > max_chunks - visible.size()) offscreen.resize(max_chunks - visible.size());

  uint32_t n = (uint32_t)(visible.size() + offscreen.size());
  *n_chunks_out = n;
  if (n > cap) return 3;
  uint32_t camera_chunk = VM_NO_CHUNK;
  std::vector<Item> all;
  all.reserve(n);
  all.insert(all.end(), visible.begin(), visible.end());
  all.insert(all.end(), offscreen.begin(), offscreen.end());
  for (uint32_t i = 0; i < n; ++i) {
    const Item& it = all[i];
    const ChunkRecord& r = *it.r;
    if (i < visible.size() && camera_chunk == VM_NO_CHUNK && pos.x >= it.mn[0] && pos.y >= it.mn[1] &&
        pos.z >= it.mn[2] && pos.x <= it.mx[0] && pos.y <= it.mx[1] && pos.z <= it.mx[2])
      camera_chunk = i;
    vm_chunk& c = chunks_out[i];
    memset(&c, 0, sizeof c);
    for (int k = 0; k < 3; ++k) { c.aabb_min[k] = it.mn[k]; c.aabb_max[k] = it.mx[k]; }
    c.voxel_size = (float)r.key.voxel_size();
    c.lod = r.key.lod;
    c.origin[0] = (float)(r.key.x * r.key.size());
    c.origin[1] = (float)(r.key.y * r.key.size());
    c.origin[2] = (float)(r.key.z * r.key.size());
    c.fade = r.fade;
    c.root[0] = (uint32_t)r.root.mask; c.root[1] = (uint32_t)(r.root.mask >> 32);
    c.root[2] = r.root.run_ptr; c.root[3] = r.root.leaf_prefix;
    c.attr_base = r.attr_value;
    c.attr_flags = r.attr_uniform ? VM_ATTR_UNIFORM : 0u;
    if (r.has_water) c.attr_flags |= VM_ATTR_HAS_WATER;
    if (r.has_foliage) c.attr_flags |= VM_ATTR_HAS_FOLIAGE;
    if (r.has_cutout) c.attr_flags |= VM_ATTR_HAS_CUTOUT;
    if (r.has_emitter) c.attr_flags |= VM_ATTR_HAS_EMITTER;
    if (r.has_glass) c.attr_flags |= VM_ATTR_HAS_GLASS;
    c.light_base = 0xF000u;
    c.light_flags = 1u;
    c.dry_mask[0] = (uint32_t)r.dry_mask;
    c.dry_mask[1] = (uint32_t)(r.dry_mask >> 32);
  }
  // grid: NO_CHUNK fill, then chunks sorted by (share, coarser first), a
  // stable sort (src/render/mod.rs:1536-1552 with shadow_share on); share =
  // RenderItem::share (src/lod.rs:69-75)
  uint64_t glen = (uint64_t)gdim[0] * gdim[1] * gdim[2];
  for (uint64_t i = 0; i < glen; ++i) grid_out[i] = VM_NO_CHUNK;
  std::vector<uint32_t> order(n);
  for (uint32_t i = 0; i < n; ++i) order[i] = i;
  auto share = [&](uint32_t i) { float f = all[i].r->fade; return f >= 0.0f ? f : 1.0f + f; };
  std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) {
    float sa = share(a), sb = share(b);
    if (sa < sb) return true;
    if (sb < sa) return false;
    return all[a].r->key.lod > all[b].r->key.lod;
  });
  for (uint32_t i : order) {
    int32_t lo[3], hi[3];
    if (!grid_span(all[i].r->key, lo, hi)) continue;
    for (int32_t z = lo[2]; z < hi[2]; ++z)
      for (int32_t y = lo[1]; y < hi[1]; ++y)
        for (int32_t x = lo[0]; x < hi[0]; ++x)
          grid_out[(uint64_t)x + (uint64_t)y * gdim[0] + (uint64_t)z * gdim[0] * gdim[1]] = i;
  }

  memset(frame, 0, sizeof *frame);
  frame->cam_pos[0] = pos.x; frame->cam_pos[1] = pos.y; frame->cam_pos[2] = pos.z;
  frame->cam_fwd[0] = fwd.x; frame->cam_fwd[1] = fwd.y; frame->cam_fwd[2] = fwd.z;
  frame->cam_right[0] = right.x; frame->cam_right[1] = right.y; frame->cam_right[2] = right.z;
  frame->cam_up[0] = up.x; frame->cam_up[1] = up.y; frame->cam_up[2] = up.z;
  frame->tan_half_fov = tan_half;
  frame->aspect = aspect;
  frame->far_ = cam->far_;
  for (int i = 0; i < 3; ++i) frame->sun_dir[i] = cam->sun_dir[i];
  frame->daylight = cam->daylight;
  frame->res[0] = cam->width; frame->res[1] = cam->height;
  frame->tiles[0] = (cam->width + VM_TILE - 1) / VM_TILE;
  frame->tiles[1] = (cam->height + VM_TILE - 1) / VM_TILE;
  frame->chunk_count = (uint32_t)visible.size();
  frame->camera_chunk = camera_chunk;
  frame->flags = cam->flags;
  frame->max_pairs = orw_pairs_for(frame->tiles[0], frame->tiles[1]);
  frame->shadow_dist = 220.0f;
  frame->ambient = 1.0f;
  for (int i = 0; i < 3; ++i) { frame->grid_min[i] = gmin[i]; frame->grid_dim[i] = gdim[i]; }
  frame->sea_level = cam->sea_level;
  frame->water_absorb = 1.0f;
  frame->jitter[0] = cam->jitter[0]; frame->jitter[1] = cam->jitter[1];
  frame->taa_feedback = 1.0f;
  // the wave parameters of the engine's default configuration
  // (src/config.rs:318-321 through src/render/mod.rs:1690-1694)
  frame->wave_amp = 0.12f;
  frame->wave_scale = 32.0f;
  frame->wave_speed = 0.32f;
  frame->wave_reflect_slope = 0.0f;
  frame->frame_index = cam->frame_index % 64u;
  return 0;
}

// Halton(2,3) jitter, src/math.rs:119-134
void orw_halton_jitter(uint64_t index, float* out2) {
  auto halton = [](uint32_t i, uint32_t base) {
    float f = 1.0f, r = 0.0f;
    while (i > 0) { f /= (float)base; r += f * (float)(i % base); i /= base; }
    return r;
  };
  uint32_t i = (uint32_t)(index % 8u) + 1;
  out2[0] = halton(i, 2) - 0.5f;
  out2[1] = halton(i, 3) - 0.5f;
}

}  // extern "C"
