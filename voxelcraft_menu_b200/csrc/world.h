// Host-side world store: the engine's dense -> 64-tree encoder, its run and
// word pools, the per-frame chunk list and grid, and the synthetic world
// recipes the benchmarks use.  These produce exactly the buffers the engine
// uploads (inner / leaf / brick pools, GpuChunk list, 32x8x32 grid), so the
// march kernels can be fed either by the engine itself or by this store.
#pragma once
#include <cstdint>
#include <vector>
#include <unordered_map>
#include "vm_types.h"

namespace vm {

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

}  // namespace vm
