// The product's host world store (store.h), the per-frame chunk list and grid,
// and the C ABI of include/voxmarch_world.h.
#include "store.h"
#include "recipe.h"
#include "../../include/voxmarch_world.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>

namespace vms {

namespace {

constexpr uint32_t NONE = 0xFFFFFFFFu;

inline uint32_t cell(uint32_t x, uint32_t y, uint32_t z) { return x | (y << 2) | (z << 4); }
inline uint32_t below(uint64_t m, uint32_t bit) { return (uint32_t)__builtin_popcountll(m & ((1ull << bit) - 1ull)); }
inline bool foliage_id(uint32_t id) { return id == VM_TALL_GRASS || id == VM_GRASS_TALL || id == VM_REEDS; }
inline bool cutout_id(uint32_t id) { return id == VM_LEAVES || id == VM_PINE_LEAVES; }
inline bool emitter_id(uint32_t id) {
  return id == VM_GLOWSTONE || id == VM_AMBER_LAMP || id == VM_AZURE_LAMP || id == VM_VERDANT_LAMP;
}
// index bits per voxel for a palette of n ids, and the words a leaf's palette
// takes (none for a single id: the entry holds it)
inline uint32_t index_bits(uint32_t n) { return n <= 2u ? 1u : (n <= 4u ? 2u : (n <= 16u ? 4u : 8u)); }
inline uint32_t palette_words(uint32_t n) { return n <= 1u ? 0u : 1u + (n + 1u) / 2u + 2u * index_bits(n); }

// The 64 block ids of leaf g (L1 cell g >> 6, leaf cell g & 63) in voxel cell order.
inline void leaf_ids(const uint16_t* dense, uint32_t g, uint16_t ids[64]) {
  const uint32_t li = g >> 6, j = g & 63u;
  const uint32_t bx = (li & 3u) * 16u + (j & 3u) * 4u;
  const uint32_t by = ((li >> 2) & 3u) * 16u + ((j >> 2) & 3u) * 4u;
  const uint32_t bz = (li >> 4) * 16u + (j >> 4) * 4u;
  for (uint32_t vb = 0; vb < 64u; ++vb)
    ids[vb] = dense[(bx + (vb & 3u)) | ((bz + (vb >> 4)) << 6) | ((by + ((vb >> 2) & 3u)) << 12)];
}

// Distinct ids of the present voxels in order of first appearance (pal) and
// each present voxel's palette index (slot); returns their number.
inline uint32_t distinct(const uint16_t ids[64], uint64_t m, uint16_t pal[64], uint8_t slot[64]) {
  uint32_t n = 0;
  for (uint64_t r = m; r; r &= r - 1) {
    const uint32_t vb = (uint32_t)__builtin_ctzll(r);
    uint32_t k = 0;
    while (k < n && pal[k] != ids[vb]) ++k;
    if (k == n) pal[n++] = ids[vb];
    slot[vb] = (uint8_t)k;
  }
  return n;
}

}  // namespace

void encode_host(const uint16_t* dense, Tree& out) {
  // ---- pass 1: per-leaf statistics --------------------------------------
  std::vector<uint64_t> mask(4096);
  std::vector<uint16_t> first(4096);
  std::vector<uint8_t> words(4096);
  uint8_t l1_full[64], l1_dry[64], l1_top[64];
  uint32_t flags = 0, emitters = 0, lo[3] = {64, 64, 64}, hi[3] = {0, 0, 0};
  uint16_t ids[64], pal[64];
  uint8_t slot[64];
  for (uint32_t li = 0; li < 64u; ++li) {
    bool full = true, dry = false;
    uint32_t top = 0;   // 1 + highest non-water y inside the node
    for (uint32_t j = 0; j < 64u; ++j) {
      const uint32_t g = li * 64u + j;
      leaf_ids(dense, g, ids);
      uint64_t m = 0;
      for (uint32_t vb = 0; vb < 64u; ++vb) m |= (uint64_t)(ids[vb] != VM_AIR) << vb;
      mask[g] = m;
      if (m != ~0ull) full = false;
      if (m == 0) { first[g] = 0; words[g] = 0; continue; }
      const uint32_t n = distinct(ids, m, pal, slot);
      first[g] = pal[0];
      words[g] = (uint8_t)palette_words(n);
      const uint32_t ly = (j >> 2) & 3u;
      for (uint64_t r = m; r; r &= r - 1) {
        const uint32_t vb = (uint32_t)__builtin_ctzll(r), id = ids[vb];
        if (id == VM_WATER) flags |= VM_TREE_WATER;
        else { dry = true; top = std::max(top, ly * 4u + ((vb >> 2) & 3u) + 1u); }
        if (foliage_id(id)) flags |= VM_TREE_FOLIAGE;
        if (cutout_id(id)) flags |= VM_TREE_CUTOUT;
        if (id == VM_GLASS) flags |= VM_TREE_GLASS;
        emitters += emitter_id(id) ? 1u : 0u;
        const uint32_t p[3] = {(li & 3u) * 16u + (j & 3u) * 4u + (vb & 3u),
                               ((li >> 2) & 3u) * 16u + ly * 4u + ((vb >> 2) & 3u),
                               (li >> 4) * 16u + (j >> 4) * 4u + (vb >> 4)};
        for (int a = 0; a < 3; ++a) { lo[a] = std::min(lo[a], p[a]); hi[a] = std::max(hi[a], p[a] + 1u); }
      }
    }
    l1_full[li] = full ? 1 : 0;
    l1_dry[li] = dry ? 1 : 0;
    l1_top[li] = (uint8_t)top;
  }
  if (emitters) flags |= VM_TREE_EMITTER;

  // ---- prefix sums over the leaves in ascending cell order ---------------
  uint32_t attr_at[64], kept_at[64], word_at[64];
  uint32_t n_attr = 0, n_kept = 0, n_word = 0, solid = 0, first_leaf = NONE;
  uint64_t root = 0, dry_mask = 0;
  for (uint32_t li = 0; li < 64u; ++li) {
    attr_at[li] = n_attr; kept_at[li] = n_kept; word_at[li] = n_word;
    for (uint32_t j = 0; j < 64u; ++j) {
      const uint32_t g = li * 64u + j;
      if (!mask[g]) continue;
      if (first_leaf == NONE) first_leaf = g;
      root |= 1ull << li;
      ++n_attr;
      if (!l1_full[li]) ++n_kept;
      n_word += words[g];
      solid += (uint32_t)__builtin_popcountll(mask[g]);
    }
    if (((root >> li) & 1ull) && l1_dry[li]) dry_mask |= 1ull << li;
  }
  bool uniform = first_leaf != NONE;
  for (uint32_t g = 0; g < 4096u && uniform; ++g)
    if (mask[g] && (words[g] || first[g] != first[first_leaf])) uniform = false;

  // ---- pass 2: the output at those offsets --------------------------------
  out.l1.clear();
  out.leaves.assign(n_kept, 0);
  out.attrs.assign(uniform ? 0u : n_attr, 0u);
  out.palette.assign(uniform ? 0u : n_word, 0u);
  for (uint32_t li = 0; li < 64u; ++li) {
    if (!((root >> li) & 1ull)) continue;
    vm_tree_l1 node;
    memset(&node, 0, sizeof node);
    for (uint32_t j = 0; j < 64u; ++j) node.mask |= (uint64_t)(mask[li * 64u + j] != 0) << j;
    node.leaf_start = kept_at[li];
    node.leaf_prefix = attr_at[li];
    node.full = l1_full[li];
    node.water_line = l1_dry[li] ? (uint8_t)(l1_top[li] - 1u) : 15;
    out.l1.push_back(node);
    uint32_t a = attr_at[li], k = kept_at[li], w = word_at[li];
    for (uint32_t j = 0; j < 64u; ++j) {
      const uint32_t g = li * 64u + j;
      const uint64_t m = mask[g];
      if (!m) continue;
      if (!l1_full[li]) out.leaves[k++] = m;
      if (!uniform) {
        if (!words[g]) {
          out.attrs[a] = VM_UNIFORM_BIT | first[g];
        } else {
          out.attrs[a] = w;
          leaf_ids(dense, g, ids);
          const uint32_t n = distinct(ids, m, pal, slot), bits = index_bits(n), npw = (n + 1u) / 2u;
          uint32_t* p = out.palette.data() + w;
          p[0] = n | (bits << 8);
          for (uint32_t q = 0; q < npw; ++q)
            p[1 + q] = (uint32_t)pal[2 * q] | ((2 * q + 1 < n ? (uint32_t)pal[2 * q + 1] : 0u) << 16);
          uint32_t* idx = p + 1 + npw;
          for (uint64_t r = m; r; r &= r - 1) {
            const uint32_t vb = (uint32_t)__builtin_ctzll(r), bit = vb * bits;
            idx[bit >> 5] |= (uint32_t)slot[vb] << (bit & 31u);
          }
        }
      }
      ++a;
      w += words[g];
    }
  }
  vm_tree_info& in = out.info;
  memset(&in, 0, sizeof in);
  in.root_mask = root;
  in.dry_mask = dry_mask;
  in.uniform = uniform ? (int32_t)first[first_leaf] : -1;
  in.flags = flags;
  in.emitters = emitters;
  in.solid_count = solid;
  in.leaf_count = n_attr;
  in.n_l1 = (uint32_t)out.l1.size();
  in.n_leaves = n_kept;
  in.n_attrs = (uint32_t)out.attrs.size();
  in.n_palette = (uint32_t)out.palette.size();
  if (solid > 0)
    for (int a = 0; a < 3; ++a) { in.aabb_min[a] = (uint8_t)lo[a]; in.aabb_max[a] = (uint8_t)hi[a]; }
}

// ---------------------------------------------------------------------------
void Store::insert(const Key& k, Tree&& t) {
  Entry& e = map_[k];
  e.key = k;
  e.tree = std::move(t);
  e.seq = seq_++;
  e.fade = 1.0f;
  dirty_ = true;
}

bool Store::remove(const Key& k) {
  dirty_ = true;
  return map_.erase(k) != 0;
}

bool Store::set_fade(const Key& k, float fade) {
  auto it = map_.find(k);
  if (it == map_.end()) return false;
  it->second.fade = fade;
  return true;
}

const Entry* Store::find(const Key& k) const {
  auto it = map_.find(k);
  return it == map_.end() ? nullptr : &it->second;
}

std::vector<const Entry*> Store::ordered() const {
  std::vector<const Entry*> v;
  v.reserve(map_.size());
  for (auto& kv : map_) v.push_back(&kv.second);
  std::sort(v.begin(), v.end(), [](const Entry* a, const Entry* b) { return a->seq < b->seq; });
  return v;
}

namespace {

// Hash-consing of fixed-width word runs appended to a pool: a run equal to
// one already emitted is given that run's offset.
class Interner {
 public:
  Interner(std::vector<uint32_t>& pool, uint32_t width) : pool_(pool), width_(width) {}
  // offset (in elements of `width` words) of the run of n elements at p
  uint32_t put(const uint32_t* p, uint32_t n, uint64_t* refs) {
    uint64_t h = 0x243F6A8885A308D3ull ^ n;
    for (uint32_t i = 0; i < n * width_; ++i) h = (h ^ p[i]) * 0x100000001B3ull;
    auto& bucket = table_[h];
    for (uint32_t off : bucket)
      if (len_[off] == n && std::equal(p, p + n * width_, pool_.begin() + (size_t)off * width_)) {
        *refs += n;
        return off;
      }
    const uint32_t off = (uint32_t)(pool_.size() / width_);
    pool_.insert(pool_.end(), p, p + n * width_);
    len_[off] = n;
    bucket.push_back(off);
    *refs += n;
    return off;
  }

 private:
  std::vector<uint32_t>& pool_;
  uint32_t width_;
  std::unordered_map<uint64_t, std::vector<uint32_t>> table_;
  std::unordered_map<uint32_t, uint32_t> len_;
};

}  // namespace

void Store::pack() {
  if (!dirty_) return;
  inners_.clear(); leaves_.clear(); words_.clear();
  leaf_refs_ = inner_refs_ = 0;
  Interner leaf_runs(leaves_, 2), inner_runs(inners_, 4);
  std::vector<uint32_t> run;
  for (const Entry* ce : ordered()) {
    Entry& e = const_cast<Entry&>(*ce);
    const Tree& t = e.tree;
    Placement pl;
    run.clear();
    bool all_full = t.l1.size() == 64;
    for (const vm_tree_l1& n : t.l1) {
      const uint32_t prefix = n.leaf_prefix | ((uint32_t)n.water_line << 28);
      if (n.full) {
        run.insert(run.end(), {0xFFFFFFFFu, 0xFFFFFFFFu, VM_FULL_BIT, prefix});
      } else {
        all_full = false;
        const uint32_t cnt = (uint32_t)__builtin_popcountll(n.mask);
        const uint32_t off = leaf_runs.put(reinterpret_cast<const uint32_t*>(t.leaves.data() + n.leaf_start), cnt,
                                           &leaf_refs_);
        run.insert(run.end(), {(uint32_t)n.mask, (uint32_t)(n.mask >> 32), off, prefix});
      }
    }
    if (t.l1.empty()) {
      // an empty chunk: the zero root
    } else if (all_full) {
      pl.root[0] = pl.root[1] = 0xFFFFFFFFu; pl.root[2] = VM_FULL_BIT; pl.root[3] = 0;
    } else {
      pl.root[0] = (uint32_t)t.info.root_mask;
      pl.root[1] = (uint32_t)(t.info.root_mask >> 32);
      pl.root[2] = inner_runs.put(run.data(), (uint32_t)t.l1.size(), &inner_refs_);
      pl.root[3] = 0;
    }
    if (t.info.uniform >= 0) {
      pl.attr_uniform = true; pl.attr_base = (uint32_t)t.info.uniform;
    } else if (t.attrs.empty()) {
      pl.attr_uniform = true; pl.attr_base = VM_AIR;
    } else {
      const uint32_t pal = (uint32_t)words_.size();
      words_.insert(words_.end(), t.palette.begin(), t.palette.end());
      pl.attr_uniform = false;
      pl.attr_base = (uint32_t)words_.size();
      for (uint32_t a : t.attrs) words_.push_back((a & VM_UNIFORM_BIT) ? a : a + pal);
    }
    e.place = pl;
  }
  dirty_ = false;
}

uint16_t Store::block(int32_t x, int32_t y, int32_t z) const {
  if (y < 0) return VM_AIR;
  Key k;
  k.x = x >> 6; k.y = y >> 6; k.z = z >> 6;
  const Entry* e = find(k);
  if (!e) return VM_AIR;
  const Tree& t = e->tree;
  const uint32_t lx = x & 63, ly = y & 63, lz = z & 63;
  const uint32_t l1b = cell(lx >> 4, ly >> 4, lz >> 4);
  if (!((t.info.root_mask >> l1b) & 1ull)) return VM_AIR;
  const vm_tree_l1& n = t.l1[below(t.info.root_mask, l1b)];
  const uint32_t lfb = cell((lx >> 2) & 3u, (ly >> 2) & 3u, (lz >> 2) & 3u);
  if (!((n.mask >> lfb) & 1ull)) return VM_AIR;
  const uint32_t vb = cell(lx & 3u, ly & 3u, lz & 3u);
  const uint64_t m = n.full ? ~0ull : t.leaves[n.leaf_start + below(n.mask, lfb)];
  if (!((m >> vb) & 1ull)) return VM_AIR;
  if (t.info.uniform >= 0) return (uint16_t)t.info.uniform;
  const uint32_t entry = t.attrs[n.leaf_prefix + below(n.mask, lfb)];
  if (entry & VM_UNIFORM_BIT) return (uint16_t)entry;
  const uint32_t hdr = t.palette[entry], cnt = hdr & 0xFFu, bits = (hdr >> 8) & 0xFFu;
  const uint32_t bit = vb * bits;
  const uint32_t idx = (t.palette[entry + 1 + (cnt + 1) / 2 + (bit >> 5)] >> (bit & 31u)) & ((1u << bits) - 1u);
  return (uint16_t)(t.palette[entry + 1 + idx / 2] >> ((idx & 1u) * 16u));
}

}  // namespace vms

// ===========================================================================
// Chunk list, grid and frame for one view
// ===========================================================================
namespace {

using vms::Entry;
using vms::Key;

struct V3 { float x, y, z; };
inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 operator*(V3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
inline float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 cross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
// glam's normalize_or: v * (1 / |v|), or the fallback when that is not finite
inline V3 unit_or(V3 v, V3 fallback) {
  const float r = 1.0f / sqrtf(dot(v, v));
  return (std::isfinite(r) && r > 0.0f) ? v * r : fallback;
}
inline V3 ld(const float* p) { return {p[0], p[1], p[2]}; }

// Frustum of src/math.rs:74-117: four side planes, the near plane through the
// camera and the far plane, each an inward unit normal and an offset.
struct Frustum {
  V3 n[6];
  float d[6];
  Frustum(V3 pos, V3 fwd, V3 right, V3 up, float tan_half, float aspect, float far_) {
    const float hx = tan_half * aspect, hy = tan_half;
    const V3 side[5] = {fwd * hx + right, fwd * hx - right, fwd * hy + up, fwd * hy - up, fwd};
    for (int i = 0; i < 5; ++i) {
      n[i] = unit_or(side[i], V3{0, 0, 0});
      d[i] = -dot(n[i], pos);
    }
    n[5] = V3{-fwd.x, -fwd.y, -fwd.z};
    d[5] = -dot(n[5], pos + fwd * far_);
  }
  bool holds(const float* lo, const float* hi) const {
    for (int i = 0; i < 6; ++i) {
      const V3 p{n[i].x > 0 ? hi[0] : lo[0], n[i].y > 0 ? hi[1] : lo[1], n[i].z > 0 ? hi[2] : lo[2]};
      if (dot(n[i], p) + d[i] < 0.0f) return false;
    }
    return true;
  }
};

// The grid cells [lo, hi) a chunk of key k covers (src/render/mod.rs:93-107);
// false when it covers none.
bool cells_of(const Key& k, const int32_t gmin[3], const uint32_t gdim[3], int32_t lo[3], int32_t hi[3]) {
  const int32_t span = 1 << k.lod;
  const int32_t base[3] = {k.x * span - gmin[0], k.y * span - gmin[1], k.z * span - gmin[2]};
  for (int i = 0; i < 3; ++i) {
    lo[i] = std::max(base[i], 0);
    hi[i] = std::min(base[i] + span, (int32_t)gdim[i]);
    if (lo[i] >= hi[i]) return false;
  }
  return true;
}

}  // namespace

struct vmw_world {
  vms::Store s;
  std::mutex mu;
};

extern "C" {

vmw_world* vmw_create(void) { return new vmw_world(); }
void vmw_destroy(vmw_world* w) { delete w; }

int vmw_insert_dense(vmw_world* w, uint8_t lod, int32_t x, int32_t y, int32_t z, const uint16_t* dense) {
  if (!w || !dense) return 1;
  vms::Tree t;
  vms::encode_host(dense, t);
  Key k; k.lod = lod; k.x = x; k.y = y; k.z = z;
  std::lock_guard<std::mutex> g(w->mu);
  w->s.insert(k, std::move(t));
  return 0;
}

int vmw_build_tree(const uint16_t* dense, uint32_t palette_cap, vm_tree_info* info, vm_tree_l1* l1,
                   uint64_t* leaves, uint32_t* attrs, uint32_t* palette) {
  if (!dense || !info || !l1 || !leaves || !attrs || (palette_cap && !palette)) return 1;
  vms::Tree t;
  vms::encode_host(dense, t);
  *info = t.info;
  if (!t.l1.empty()) memcpy(l1, t.l1.data(), t.l1.size() * sizeof(vm_tree_l1));
  if (!t.leaves.empty()) memcpy(leaves, t.leaves.data(), t.leaves.size() * 8);
  if (!t.attrs.empty()) memcpy(attrs, t.attrs.data(), t.attrs.size() * 4);
  if (t.palette.size() > palette_cap) info->flags |= VM_TREE_PALETTE_OVERFLOW;
  const size_t np = std::min<size_t>(t.palette.size(), palette_cap);
  if (np) memcpy(palette, t.palette.data(), np * 4);
  return 0;
}

int vmw_insert_tree(vmw_world* w, uint8_t lod, int32_t x, int32_t y, int32_t z, const vm_tree_info* info,
                    const vm_tree_l1* l1, const uint64_t* leaves, const uint32_t* attrs, const uint32_t* palette) {
  if (!w || !info || (info->flags & VM_TREE_PALETTE_OVERFLOW) || info->n_l1 > VM_TREE_L1 ||
      info->n_leaves > VM_TREE_LEAVES || info->n_attrs > VM_TREE_LEAVES)
    return 1;
  vms::Tree t;
  t.info = *info;
  t.l1.assign(l1, l1 + info->n_l1);
  // every node's leaf run and attribute range must lie inside the arrays
  for (const vm_tree_l1& n : t.l1) {
    const uint32_t cnt = (uint32_t)__builtin_popcountll(n.mask);
    if (!n.full && (uint64_t)n.leaf_start + cnt > info->n_leaves) return 1;
    if (info->n_attrs && (uint64_t)n.leaf_prefix + cnt > info->n_attrs) return 1;
  }
  t.leaves.assign(leaves, leaves + info->n_leaves);
  t.attrs.assign(attrs, attrs + info->n_attrs);
  t.palette.assign(palette, palette + info->n_palette);
  for (uint32_t a : t.attrs)
    if (!(a & VM_UNIFORM_BIT) && a >= info->n_palette) return 1;
  Key k; k.lod = lod; k.x = x; k.y = y; k.z = z;
  std::lock_guard<std::mutex> g(w->mu);
  w->s.insert(k, std::move(t));
  return 0;
}

int vmw_remove(vmw_world* w, uint8_t lod, int32_t x, int32_t y, int32_t z) {
  Key k; k.lod = lod; k.x = x; k.y = y; k.z = z;
  std::lock_guard<std::mutex> g(w->mu);
  return w->s.remove(k) ? 0 : 1;
}

int vmw_set_fade(vmw_world* w, uint8_t lod, int32_t x, int32_t y, int32_t z, float fade) {
  Key k; k.lod = lod; k.x = x; k.y = y; k.z = z;
  if (!(fade >= -1.0f && fade <= 1.0f) || fade == 0.0f) return 2;
  std::lock_guard<std::mutex> g(w->mu);
  return w->s.set_fade(k, fade) ? 0 : 1;
}

uint32_t vmw_get_block(const vmw_world* w, int32_t x, int32_t y, int32_t z) { return w->s.block(x, y, z); }

int vmw_get_chunk_info(const vmw_world* wc, uint8_t lod, int32_t x, int32_t y, int32_t z, vmw_chunk_info* out) {
  vmw_world* w = const_cast<vmw_world*>(wc);
  std::lock_guard<std::mutex> g(w->mu);
  w->s.pack();
  Key k; k.lod = lod; k.x = x; k.y = y; k.z = z;
  const Entry* e = w->s.find(k);
  if (!e) return 1;
  const vm_tree_info& t = e->tree.info;
  memset(out, 0, sizeof *out);
  memcpy(out->root, e->place.root, sizeof out->root);
  out->attr_uniform = e->place.attr_uniform;
  out->attr_value = e->place.attr_base;
  for (int i = 0; i < 3; ++i) { out->aabb_min[i] = t.aabb_min[i]; out->aabb_max[i] = t.aabb_max[i]; }
  out->solid_count = t.solid_count;
  out->leaf_count = t.leaf_count;
  out->dry_mask = t.dry_mask;
  out->has_water = (t.flags & VM_TREE_WATER) != 0;
  out->has_foliage = (t.flags & VM_TREE_FOLIAGE) != 0;
  out->has_cutout = (t.flags & VM_TREE_CUTOUT) != 0;
  out->has_glass = (t.flags & VM_TREE_GLASS) != 0;
  out->has_emitter = (t.flags & VM_TREE_EMITTER) != 0;
  return 0;
}

void vmw_pool_stats(const vmw_world* wc, vmw_pool_stats_t* s) {
  vmw_world* w = const_cast<vmw_world*>(wc);
  std::lock_guard<std::mutex> g(w->mu);
  w->s.pack();
  memset(s, 0, sizeof *s);
  s->n_inners = w->s.inners().size() / 4;
  s->n_leaves = w->s.leaves().size() / 2;
  s->n_bricks = w->s.words().size();
  s->live_inners = s->n_inners;
  s->live_leaves = s->n_leaves;
  s->referenced_inners = w->s.inner_refs();
  s->referenced_leaves = w->s.leaf_refs();
  s->used_words = s->n_bricks;
  s->n_chunks = w->s.size();
}

const uint32_t* vmw_inners(const vmw_world* w) { const_cast<vmw_world*>(w)->s.pack(); return w->s.inners().data(); }
const uint32_t* vmw_leaves(const vmw_world* w) { const_cast<vmw_world*>(w)->s.pack(); return w->s.leaves().data(); }
const uint32_t* vmw_bricks(const vmw_world* w) { const_cast<vmw_world*>(w)->s.pack(); return w->s.words().data(); }

int vmw_generate(vmw_world* w, const vmw_recipe* r) {
  if (!w || !r) return 1;
  for (int i = 0; i < 3; ++i) if (r->size[i] == 0 || r->size[i] % 64 != 0) return 2;
  const vmr::Heights hs = vmr::make_heights(*r);
  const int32_t nx = r->size[0] / 64, ny = r->size[1] / 64, nz = r->size[2] / 64;
  const int64_t total = (int64_t)nx * ny * nz;
  std::vector<vms::Tree> trees((size_t)total);
#pragma omp parallel
  {
    std::vector<uint16_t> dense(64 * 64 * 64);
#pragma omp for schedule(dynamic, 1)
    for (int64_t i = 0; i < total; ++i) {
      vmr::fill_chunk(*r, hs, (int32_t)(i % nx), (int32_t)((i / nx) % ny), (int32_t)(i / ((int64_t)nx * ny)),
                      dense.data());
      vms::encode_host(dense.data(), trees[i]);
    }
  }
  std::lock_guard<std::mutex> g(w->mu);
  for (int64_t i = 0; i < total; ++i) {
    Key k; k.x = (int32_t)(i % nx); k.y = (int32_t)((i / nx) % ny); k.z = (int32_t)(i / ((int64_t)nx * ny));
    w->s.insert(k, std::move(trees[i]));
  }
  return 0;
}

int vmw_recipe_dense_all(const vmw_recipe* r, uint16_t* dense) {
  if (!r || !dense) return 1;
  for (int i = 0; i < 3; ++i) if (r->size[i] == 0 || r->size[i] % 64 != 0) return 2;
  const vmr::Heights hs = vmr::make_heights(*r);
  const int32_t nx = r->size[0] / 64, ny = r->size[1] / 64, nz = r->size[2] / 64;
  const int64_t total = (int64_t)nx * ny * nz;
#pragma omp parallel for schedule(dynamic, 1)
  for (int64_t i = 0; i < total; ++i)
    vmr::fill_chunk(*r, hs, (int32_t)(i % nx), (int32_t)((i / nx) % ny), (int32_t)(i / ((int64_t)nx * ny)),
                    dense + (size_t)i * 64 * 64 * 64);
  return 0;
}

int vmw_recipe_dense(const vmw_recipe* r, int32_t cx, int32_t cy, int32_t cz, uint16_t* dense) {
  if (!r || !dense) return 1;
  vmr::fill_chunk(*r, vmr::make_heights(*r), cx, cy, cz, dense);
  return 0;
}

int vmw_recipe_dense_lod(const vmw_recipe* r, uint32_t lod, int32_t cx, int32_t cy, int32_t cz, uint16_t* dense) {
  if (!r || !dense || lod > 4) return 1;
  vmr::fill_chunk_lod(*r, lod, cx, cy, cz, dense);
  return 0;
}

int32_t vmw_recipe_height(const vmw_recipe* r, int32_t x, int32_t z) {
  return (int32_t)floorf(r->base + r->amplitude * vmr::fbm((float)x, (float)z, *r));
}

// Camera basis: look_dir (src/player.rs:122-126) and the right / up vectors of
// src/scene.rs:334-339.
void vmw_camera_basis(float yaw, float pitch, float* fwd, float* right, float* up) {
  const float sy = sinf(yaw), cy = cosf(yaw), sp = sinf(pitch), cp = cosf(pitch);
  const V3 f = unit_or(V3{cy * cp, sp, sy * cp}, V3{0, 0, 0});
  const V3 r = unit_or(cross(f, V3{0, 1, 0}), V3{1, 0, 0});
  const V3 u = unit_or(cross(r, f), V3{0, 1, 0});
  const V3* src[3] = {&f, &r, &u};
  float* dst[3] = {fwd, right, up};
  for (int i = 0; i < 3; ++i) { dst[i][0] = src[i]->x; dst[i][1] = src[i]->y; dst[i][2] = src[i]->z; }
}

// pairs_for (src/render/mod.rs:27-30): the pair list's capacity
uint32_t vmw_pairs_for(uint32_t tiles_x, uint32_t tiles_y) {
  const uint64_t want = std::max<uint64_t>((uint64_t)tiles_x * tiles_y * VM_PAIRS_PER_TILE, VM_MAX_PAIRS_FLOOR);
  return (uint32_t)std::min<uint64_t>(want, (uint64_t)UINT32_MAX / 2);
}

// build_chunk_list + partition_for_grid (src/render/mod.rs:109-138,1447-1564)
// and the GpuFrame fill (1640-1707) for one view.
int vmw_build_view(const vmw_world* wc, const vmw_camera* cam, vm_frame* frame, vm_chunk* out, uint32_t cap,
                   uint32_t* n_out, uint32_t* grid) {
  vmw_world* w = const_cast<vmw_world*>(wc);
  std::lock_guard<std::mutex> g(w->mu);
  w->s.pack();
  V3 fwd, right, up;
  if (cam->use_basis) {
    fwd = ld(cam->fwd); right = ld(cam->right); up = ld(cam->up);
  } else {
    float f[3], r[3], u[3];
    vmw_camera_basis(cam->yaw, cam->pitch, f, r, u);
    fwd = ld(f); right = ld(r); up = ld(u);
  }
  const V3 pos = ld(cam->pos);
  const float tan_half = tanf(cam->fov_y * 0.5f), aspect = (float)cam->width / (float)cam->height;
  uint32_t gdim[3] = {VM_GRID_X, VM_GRID_Y, VM_GRID_Z};
  if (cam->grid_dim[0]) memcpy(gdim, cam->grid_dim, sizeof gdim);
  int32_t gmin[3] = {(int32_t)floorf(pos.x / 64.0f) - (int32_t)gdim[0] / 2, 0,
                     (int32_t)floorf(pos.z / 64.0f) - (int32_t)gdim[2] / 2};
  if (cam->grid_min_set) memcpy(gmin, cam->grid_min, sizeof gmin);
  const Frustum fr(pos, fwd, right, up, tan_half, aspect, cam->far_);

  // the render set: every non-empty chunk, in insertion order, split into
  // the frustum's chunks and the off-screen ones the shadow grid covers, each
  // sorted by box distance (stable)
  struct Item { const Entry* e; Key key; float dist; float lo[3], hi[3]; };
  std::vector<Item> on, off;
  for (const Entry* e : w->s.ordered()) {
    const Key& k = e->key;
    if (e->tree.info.solid_count == 0) continue;
    Item it;
    it.e = e;
    it.key = k;
    const float vs = (float)(1 << k.lod);
    const float o[3] = {(float)(k.x * k.size()), (float)(k.y * k.size()), (float)(k.z * k.size())};
    for (int i = 0; i < 3; ++i) {
      it.lo[i] = o[i] + (float)e->tree.info.aabb_min[i] * vs;
      it.hi[i] = o[i] + (float)e->tree.info.aabb_max[i] * vs;
    }
    const V3 dd{std::max(std::max(it.lo[0] - pos.x, pos.x - it.hi[0]), 0.0f),
                std::max(std::max(it.lo[1] - pos.y, pos.y - it.hi[1]), 0.0f),
                std::max(std::max(it.lo[2] - pos.z, pos.z - it.hi[2]), 0.0f)};
    it.dist = sqrtf(dot(dd, dd));
    int32_t clo[3], chi[3];
    if (fr.holds(it.lo, it.hi)) on.push_back(it);
    else if (cam->offscreen_shadows && cells_of(k, gmin, gdim, clo, chi)) off.push_back(it);
  }
  const auto nearer = [](const Item& a, const Item& b) { return a.dist < b.dist; };
  const uint32_t max_chunks = cam->max_chunks ? cam->max_chunks : VM_MAX_CHUNKS;
  std::stable_sort(on.begin(), on.end(), nearer);
  if (on.size() > max_chunks) on.resize(max_chunks);
  std::stable_sort(off.begin(), off.end(), nearer);
  if (off.size() > max_chunks - on.size()) off.resize(max_chunks - on.size());
  const uint32_t n = (uint32_t)(on.size() + off.size());
  *n_out = n;
  if (n > cap) return 3;

  std::vector<const Item*> list;
  list.reserve(n);
  for (const Item& it : on) list.push_back(&it);
  for (const Item& it : off) list.push_back(&it);
  uint32_t camera_chunk = VM_NO_CHUNK;
  for (uint32_t i = 0; i < n; ++i) {
    const Item& it = *list[i];
    const vms::Placement& pl = it.e->place;
    const vm_tree_info& t = it.e->tree.info;
    if (i < on.size() && camera_chunk == VM_NO_CHUNK && pos.x >= it.lo[0] && pos.y >= it.lo[1] &&
        pos.z >= it.lo[2] && pos.x <= it.hi[0] && pos.y <= it.hi[1] && pos.z <= it.hi[2])
      camera_chunk = i;
    vm_chunk& c = out[i];
    memset(&c, 0, sizeof c);
    memcpy(c.aabb_min, it.lo, sizeof it.lo);
    memcpy(c.aabb_max, it.hi, sizeof it.hi);
    c.voxel_size = (float)(1 << it.key.lod);
    c.lod = it.key.lod;
    c.origin[0] = (float)(it.key.x * it.key.size());
    c.origin[1] = (float)(it.key.y * it.key.size());
    c.origin[2] = (float)(it.key.z * it.key.size());
    c.fade = it.e->fade;
    memcpy(c.root, pl.root, sizeof c.root);
    c.attr_base = pl.attr_base;
    c.attr_flags = (pl.attr_uniform ? VM_ATTR_UNIFORM : 0u) | ((t.flags & VM_TREE_WATER) ? VM_ATTR_HAS_WATER : 0u) |
                   ((t.flags & VM_TREE_FOLIAGE) ? VM_ATTR_HAS_FOLIAGE : 0u) |
                   ((t.flags & VM_TREE_CUTOUT) ? VM_ATTR_HAS_CUTOUT : 0u) |
                   ((t.flags & VM_TREE_EMITTER) ? VM_ATTR_HAS_EMITTER : 0u) |
                   ((t.flags & VM_TREE_GLASS) ? VM_ATTR_HAS_GLASS : 0u);
    c.light_base = 0xF000u;
    c.light_flags = 1u;
    c.dry_mask[0] = (uint32_t)t.dry_mask;
    c.dry_mask[1] = (uint32_t)(t.dry_mask >> 32);
  }
  // the grid: NO_CHUNK, then every listed chunk's cells, lowest share first
  // and, at equal share, coarser levels first, so the finest fully shown
  // chunk of a cell is the one left in it (share: fade, or 1 + fade for the
  // fading-out parent of a cross-fade, src/lod.rs:69-75)
  const uint64_t cells = (uint64_t)gdim[0] * gdim[1] * gdim[2];
  std::fill(grid, grid + cells, VM_NO_CHUNK);
  std::vector<uint32_t> order(n);
  for (uint32_t i = 0; i < n; ++i) order[i] = i;
  const auto share = [&](uint32_t i) { const float f = list[i]->e->fade; return f >= 0.0f ? f : 1.0f + f; };
  std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) {
    const float sa = share(a), sb = share(b);
    if (sa != sb) return sa < sb;
    return list[a]->key.lod > list[b]->key.lod;
  });
  for (uint32_t i : order) {
    int32_t lo[3], hi[3];
    if (!cells_of(list[i]->key, gmin, gdim, lo, hi)) continue;
    for (int32_t z = lo[2]; z < hi[2]; ++z)
      for (int32_t y = lo[1]; y < hi[1]; ++y)
        for (int32_t x = lo[0]; x < hi[0]; ++x)
          grid[(uint64_t)x + (uint64_t)y * gdim[0] + (uint64_t)z * gdim[0] * gdim[1]] = i;
  }

  memset(frame, 0, sizeof *frame);
  memcpy(frame->cam_pos, cam->pos, sizeof frame->cam_pos);
  const V3* basis[3] = {&fwd, &right, &up};
  float* dst[3] = {frame->cam_fwd, frame->cam_right, frame->cam_up};
  for (int i = 0; i < 3; ++i) { dst[i][0] = basis[i]->x; dst[i][1] = basis[i]->y; dst[i][2] = basis[i]->z; }
  frame->tan_half_fov = tan_half;
  frame->aspect = aspect;
  frame->far_ = cam->far_;
  memcpy(frame->sun_dir, cam->sun_dir, sizeof frame->sun_dir);
  frame->daylight = cam->daylight;
  frame->res[0] = cam->width; frame->res[1] = cam->height;
  frame->tiles[0] = (cam->width + VM_TILE - 1) / VM_TILE;
  frame->tiles[1] = (cam->height + VM_TILE - 1) / VM_TILE;
  frame->chunk_count = (uint32_t)on.size();
  frame->camera_chunk = camera_chunk;
  frame->flags = cam->flags;
  frame->max_pairs = vmw_pairs_for(frame->tiles[0], frame->tiles[1]);
  frame->shadow_dist = 220.0f;
  frame->ambient = 1.0f;
  for (int i = 0; i < 3; ++i) { frame->grid_min[i] = gmin[i]; frame->grid_dim[i] = gdim[i]; }
  frame->sea_level = cam->sea_level;
  frame->water_absorb = 1.0f;
  memcpy(frame->jitter, cam->jitter, sizeof frame->jitter);
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

// Halton(2,3) sub-pixel jitter of frame `index` (src/math.rs:119-134)
void vmw_halton_jitter(uint64_t index, float* out2) {
  const auto radical = [](uint32_t i, uint32_t base) {
    float f = 1.0f, r = 0.0f;
    for (; i > 0; i /= base) { f /= (float)base; r += f * (float)(i % base); }
    return r;
  };
  const uint32_t i = (uint32_t)(index % 8u) + 1u;
  out2[0] = radical(i, 2) - 0.5f;
  out2[1] = radical(i, 3) - 0.5f;
}

}  // extern "C"
