/* Host-side world store behind the march ABI.
 *
 * The engine builds its march inputs on the CPU in Rust: the dense -> 64-tree
 * encoder and the run / word pools (src/voxel/tree.rs:89-204,
 * src/voxel/world.rs:63-175, src/voxel/geometry.rs:64-219,
 * src/voxel/attributes.rs:6-139) and, per frame, the chunk list and chunk grid
 * (src/render/mod.rs:88-138,1447-1564).  An engine that keeps its own Rust
 * world only needs include/voxmarch.h; this header is the same host work in
 * C++ for callers without it (the tests, the benchmarks and the smoke check),
 * producing byte-identical buffers.
 */
#ifndef VOXMARCH_WORLD_H
#define VOXMARCH_WORLD_H
#include <stdint.h>
#include "../voxelcraft_menu_b200/csrc/vm_types.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct vmw_world vmw_world;

/* Synthetic terrain recipe: heightfield = base + amplitude * fbm(value noise,
 * `octaves` octaves from base_freq, lacunarity 2, gain 0.5); GRASS top, DIRT 3
 * below, STONE under; WATER fills air below water_level (<0: none); trees on
 * tree_permille of dry surface columns (5-tall LOG + 5x5x3 LEAVES blob);
 * GLASS replaces glass_permille of the top two surface layers; island_permille
 * > 0 keeps terrain only where a coarse mask noise is below it (sparse worlds,
 * with a water sheet water_depth thick). */
typedef struct vmw_recipe {
  uint32_t size[3];
  uint32_t octaves;
  uint32_t seed;
  float base;
  float amplitude;
  float base_freq;
  int32_t water_level;
  int32_t water_depth;
  uint32_t tree_permille;
  uint32_t glass_permille;
  uint32_t island_permille;
} vmw_recipe;

typedef struct vmw_camera {
  float pos[3];
  float yaw, pitch;          /* radians; ignored when use_basis != 0 */
  uint32_t use_basis;
  float fwd[3], right[3], up[3];
  float fov_y;               /* radians */
  uint32_t width, height;
  float far_;
  float sun_dir[3];
  float daylight;
  uint32_t flags;            /* VM_FLAG_* */
  float jitter[2];
  uint32_t frame_index;
  float sea_level;
  uint32_t offscreen_shadows;
  uint32_t grid_dim[3];      /* 0 = engine default 32x8x32 */
  uint32_t grid_min_set;
  int32_t grid_min[3];
  uint32_t max_chunks;       /* 0 = engine default 8191 */
} vmw_camera;

typedef struct vmw_chunk_info {
  uint32_t root[4];
  uint32_t attr_uniform, attr_value;
  int32_t aabb_min[3], aabb_max[3];
  uint32_t solid_count, leaf_count;
  uint64_t dry_mask;
  uint32_t has_water, has_foliage, has_cutout, has_glass, has_emitter;
} vmw_chunk_info;

typedef struct vmw_pool_stats_t {
  uint64_t n_inners, n_leaves, n_bricks;
  uint64_t live_inners, live_leaves, referenced_inners, referenced_leaves;
  uint64_t used_words, n_chunks;
} vmw_pool_stats_t;

vmw_world* vmw_create(void);
void vmw_destroy(vmw_world* w);
/* World::insert_local(key, build_local(dense)); dense index x | z<<6 | y<<12 */
int vmw_insert_dense(vmw_world* w, uint8_t lod, int32_t x, int32_t y, int32_t z, const uint16_t* dense);
/* build_local (src/voxel/tree.rs:89-204) of one dense chunk (64^3 block ids,
 * index x | z<<6 | y<<12) into the flat layout that vm_encode_trees writes:
 * info, up to 64 L1 nodes, up to 4096 leaf masks and attribute entries, and
 * up to palette_cap palette words (more sets VM_TREE_PALETTE_OVERFLOW).  The
 * CPU restatement of the engine's encoder: the GPU encoder's parity anchor. */
int vmw_build_tree(const uint16_t* dense, uint32_t palette_cap, vm_tree_info* info, vm_tree_l1* l1,
                   uint64_t* leaves, uint32_t* attrs, uint32_t* palette);
/* World::insert_local (src/voxel/world.rs:63-175) of a chunk in that flat
 * layout, e.g. from vm_encode_trees: the run / word pools dedup it exactly as
 * vmw_insert_dense does.  Rejects an overflowed or inconsistent tree (1). */
int vmw_insert_tree(vmw_world* w, uint8_t lod, int32_t x, int32_t y, int32_t z, const vm_tree_info* info,
                    const vm_tree_l1* l1, const uint64_t* leaves, const uint32_t* attrs, const uint32_t* palette);
int vmw_remove(vmw_world* w, uint8_t lod, int32_t x, int32_t y, int32_t z);
/* World::get_block (src/voxel/world.rs:258-277) */
uint32_t vmw_get_block(const vmw_world* w, int32_t x, int32_t y, int32_t z);
int vmw_get_chunk_info(const vmw_world* w, uint8_t lod, int32_t x, int32_t y, int32_t z, vmw_chunk_info* out);
/* World::l1_node (src/voxel/world.rs:225-234): 1 found, 0 absent, -1 no chunk */
int vmw_l1_node(const vmw_world* w, uint8_t lod, int32_t x, int32_t y, int32_t z, uint32_t l1b, uint32_t* out4);
void vmw_pool_stats(const vmw_world* w, vmw_pool_stats_t* s);
const uint32_t* vmw_inners(const vmw_world* w);   /* n_inners x vec4<u32> */
const uint32_t* vmw_leaves(const vmw_world* w);   /* n_leaves x vec2<u32> */
const uint32_t* vmw_bricks(const vmw_world* w);   /* n_bricks x u32 */
int vmw_generate(vmw_world* w, const vmw_recipe* r);
int vmw_recipe_dense(const vmw_recipe* r, int32_t cx, int32_t cy, int32_t cz, uint16_t* dense);
/* Every chunk of the recipe's world, chunk i = cx + nx (cy + ny cz) at
 * dense + i * 64^3 (the order vmw_generate inserts them in). */
int vmw_recipe_dense_all(const vmw_recipe* r, uint16_t* dense);
int32_t vmw_recipe_height(const vmw_recipe* r, int32_t x, int32_t z);
void vmw_camera_basis(float yaw, float pitch, float* fwd, float* right, float* up);
uint32_t vmw_pairs_for(uint32_t tiles_x, uint32_t tiles_y);
int vmw_build_view(const vmw_world* w, const vmw_camera* cam, vm_frame* frame, vm_chunk* chunks_out,
                   uint32_t cap, uint32_t* n_chunks_out, uint32_t* grid_out);
void vmw_halton_jitter(uint64_t index, float* out2);

#ifdef __cplusplus
}
#endif
#endif
