// The product's host world store: encoded chunks in the flat tree layout
// (vm_tree_info, vm_types.h) that the GPU encoder writes, packed on demand
// into the three pools the march reads (inner nodes, leaf masks, attribute /
// palette words), and the per-frame chunk list and grid.
//
// Design: a chunk is kept as its encoded tree; the pools are a derived,
// immutable product rebuilt from all chunks when a frame or a caller needs
// them after an edit (Store::pack).  Packing walks the chunks in insertion
// order and hash-conses the runs it emits (a leaf-mask run or an inner-node
// run already in the pool is referenced, not copied), so no reference counts
// or free lists exist and a removal is just a map erase.  Engines that keep
// their own producer only need the march ABI (include/voxmarch.h).
#pragma once
#include <cstdint>
#include <unordered_map>
#include <vector>

#include "vm_types.h"

namespace vms {

// One chunk in the encoder's flat output layout.
struct Tree {
  vm_tree_info info{};
  std::vector<vm_tree_l1> l1;        // info.n_l1 nodes, ascending cell order
  std::vector<uint64_t> leaves;      // kept leaf masks (not those of full L1 nodes)
  std::vector<uint32_t> attrs;       // one entry per present leaf (empty when uniform)
  std::vector<uint32_t> palette;     // palette / index words the entries point into
};

// Dense 64^3 block ids (index x | z<<6 | y<<12) -> Tree, on the host, in the
// same passes as the GPU encoder k_encode: per-leaf statistics, prefix sums
// over the 4096 leaves in ascending cell order, then the output at those
// offsets.  Bit-identical to vm_encode_trees.
void encode_host(const uint16_t* dense, Tree& out);

struct Key {
  uint8_t lod = 0;
  int32_t x = 0, y = 0, z = 0;
  bool operator==(const Key& o) const { return lod == o.lod && x == o.x && y == o.y && z == o.z; }
  int32_t size() const { return 64 << lod; }
};
struct KeyHash {
  size_t operator()(const Key& k) const {
    uint64_t h = ((uint64_t)(uint32_t)k.x << 32 | (uint32_t)k.z) * 0x9E3779B97F4A7C15ull;
    h ^= ((uint64_t)(uint32_t)k.y << 8 | k.lod) * 0xD1B54A32D192ED03ull;
    return (size_t)(h ^ (h >> 31));
  }
};

// Where a chunk landed in the packed pools.
struct Placement {
  uint32_t root[4] = {0, 0, 0, 0};   // the root Inner as the chunk record carries it
  uint32_t attr_base = 0;            // uniform id, or the attribute table's offset in the word pool
  bool attr_uniform = true;
};

struct Entry {
  Key key;
  Tree tree;
  uint64_t seq = 0;       // insertion order: the render set's order
  float fade = 1.0f;      // LOD cross-fade of the render item (1 = solid)
  Placement place;
};

class Store {
 public:
  void insert(const Key& k, Tree&& t);
  bool remove(const Key& k);
  bool set_fade(const Key& k, float fade);
  const Entry* find(const Key& k) const;
  uint16_t block(int32_t x, int32_t y, int32_t z) const;   // lod-0 chunks
  size_t size() const { return map_.size(); }
  // Rebuild the pools if an edit happened since the last pack.
  void pack();
  // The chunks in insertion order (after pack, with their placements).
  std::vector<const Entry*> ordered() const;
  const std::vector<uint32_t>& inners() const { return inners_; }   // 4 words per node
  const std::vector<uint32_t>& leaves() const { return leaves_; }   // 2 words per mask
  const std::vector<uint32_t>& words() const { return words_; }
  uint64_t leaf_refs() const { return leaf_refs_; }
  uint64_t inner_refs() const { return inner_refs_; }

 private:
  std::unordered_map<Key, Entry, KeyHash> map_;
  uint64_t seq_ = 0;
  bool dirty_ = true;
  std::vector<uint32_t> inners_, leaves_, words_;
  uint64_t leaf_refs_ = 0, inner_refs_ = 0;
};

}  // namespace vms
