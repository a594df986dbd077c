/* Host-side world store behind the march ABI.
 *
 * The engine builds its march inputs on the CPU in Rust: the dense -> 64-tree
 * encoder and the run / word pools (src/voxel/tree.rs:89-204,
 * src/voxel/world.rs:63-175, src/voxel/geometry.rs:64-219,
 * src/voxel/attributes.rs:6-139) and, per frame, the chunk list and chunk grid
 * (src/render/mod.rs:88-138,1447-1564).  An engine that keeps its own Rust
 * world only needs include/voxmarch.h.  This header is a world store for
 * callers without one (the tests, the benchmarks and the smoke check): the
 * same encoded chunk format and pool node formats, the same chunk list and
 * grid, and march outputs identical to those over the engine's pools.  The
 * pools' offsets are its own: chunks are kept encoded and the pools are
 * packed from them, in insertion order with identical leaf-mask and
 * inner-node runs shared, whenever a view or a pool is asked for after an
 * edit (no reference counts, no free lists).
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
  uint32_t tuft_permille;    /* foliage tufts (TALL_GRASS, GRASS_TALL, REEDS) on dry surface columns without a tree */
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
/* Insert (or replace) the chunk of level lod at chunk cell (x, y, z), encoded
 * from dense 64^3 block ids, index x | z<<6 | y<<12 (World::insert_local of
 * build_local, src/voxel/world.rs:63, src/voxel/tree.rs:89).  The chunk
 * becomes the last of the render set, with fade 1. */
int vmw_insert_dense(vmw_world* w, uint8_t lod, int32_t x, int32_t y, int32_t z, const uint16_t* dense);
/* The encoder on the host (build_local, src/voxel/tree.rs:89-204, with
 * encode_leaf src/voxel/attributes.rs:90-139) for one dense chunk, in the flat
 * layout that vm_encode_trees writes, by the same passes: info, up to 64 L1
 * nodes, up to 4096 leaf masks and attribute entries, and up to palette_cap
 * palette words (more sets VM_TREE_PALETTE_OVERFLOW). */
int vmw_build_tree(const uint16_t* dense, uint32_t palette_cap, vm_tree_info* info, vm_tree_l1* l1,
                   uint64_t* leaves, uint32_t* attrs, uint32_t* palette);
/* Insert a chunk given in that flat layout, e.g. from vm_encode_trees, as
 * vmw_insert_dense does.  Rejects an overflowed or inconsistent tree (1): a
 * leaf run, attribute range or palette offset outside its arrays. */
int vmw_insert_tree(vmw_world* w, uint8_t lod, int32_t x, int32_t y, int32_t z, const vm_tree_info* info,
                    const vm_tree_l1* l1, const uint64_t* leaves, const uint32_t* attrs, const uint32_t* palette);
int vmw_remove(vmw_world* w, uint8_t lod, int32_t x, int32_t y, int32_t z);
/* The chunk's LOD cross-fade as the engine's render item carries it
 * (RenderItem::fade, src/lod.rs:56-80): 1 solid, f in (0, 1) a fading-in
 * finer chunk, -f its fading-out coarser parent.  It goes into GpuChunk.fade
 * (the march's dither, common.wgsl:370-385) and orders the grid fill by share
 * (src/render/mod.rs:1536-1552).  1 no such chunk, 2 fade outside [-1, 1] or 0. */
int vmw_set_fade(vmw_world* w, uint8_t lod, int32_t x, int32_t y, int32_t z, float fade);
/* World::get_block (src/voxel/world.rs:258-277): the block of lod-0 chunks */
uint32_t vmw_get_block(const vmw_world* w, int32_t x, int32_t y, int32_t z);
int vmw_get_chunk_info(const vmw_world* w, uint8_t lod, int32_t x, int32_t y, int32_t z, vmw_chunk_info* out);
/* Pool sizes after packing; live_* equal n_* (packed pools hold no free
 * space) and referenced_* count the elements all chunks refer to, so
 * referenced - live is what run sharing saved. */
void vmw_pool_stats(const vmw_world* w, vmw_pool_stats_t* s);
const uint32_t* vmw_inners(const vmw_world* w);   /* n_inners x vec4<u32> */
const uint32_t* vmw_leaves(const vmw_world* w);   /* n_leaves x vec2<u32> */
const uint32_t* vmw_bricks(const vmw_world* w);   /* n_bricks x u32 */
int vmw_generate(vmw_world* w, const vmw_recipe* r);
int vmw_recipe_dense(const vmw_recipe* r, int32_t cx, int32_t cy, int32_t cz, uint16_t* dense);
/* A chunk of level lod (voxels of 1 << lod blocks, lod <= 4) at chunk cell
 * (cx, cy, cz) of that level, sampled from the recipe's heightfield: each
 * voxel column takes the height at its first block, each voxel the layer
 * block of its top block inside the terrain (no trees, no glass). */
int vmw_recipe_dense_lod(const vmw_recipe* r, uint32_t lod, int32_t cx, int32_t cy, int32_t cz, uint16_t* dense);
/* Every chunk of the recipe's world, chunk i = cx + nx (cy + ny cz) at
 * dense + i * 64^3 (the order vmw_generate inserts them in). */
int vmw_recipe_dense_all(const vmw_recipe* r, uint16_t* dense);
int32_t vmw_recipe_height(const vmw_recipe* r, int32_t x, int32_t z);
void vmw_camera_basis(float yaw, float pitch, float* fwd, float* right, float* up);
uint32_t vmw_pairs_for(uint32_t tiles_x, uint32_t tiles_y);
int vmw_build_view(const vmw_world* w, const vmw_camera* cam, vm_frame* frame, vm_chunk* chunks_out,
                   uint32_t cap, uint32_t* n_chunks_out, uint32_t* grid_out);
void vmw_halton_jitter(uint64_t index, float* out2);

/* Material inputs of the resolve (vm_upload_atlas, vm_upload_block_faces,
 * vm_upload_probes, vm_upload_shaft) for callers without the engine's own.
 * vmw_build_atlas: a procedural atlas of this library's own design in the
 * engine's format (VM_TEX_COUNT Rgba8UnormSrgb layers of 16x16, mips 16, 8, 4,
 * 2 in sequence, vmw_atlas_bytes(VM_TEX_COUNT) bytes; mips box-filtered in
 * linear light; alpha = the tint mask of grass / leaves / meadow faces and the
 * coverage of tufts).  vmw_block_faces: the engine's face table
 * (src/block.rs:265-276: 8 words per block id, layer | perm class << 16; n >=
 * 8 * VM_BLOCK_COUNT).  vmw_probe_field: a 128 x 768 x 128 RGBA16F field of
 * values in [0.55, 1].  vmw_shaft_envelope: the terrain sun envelope of a
 * recipe on the 512 x 512 texel window at `origin` (x, z) with `texel`
 * blocks per texel.  vmw_look_defaults: the engine's default fog, cloud, god
 * ray, tint (seed = the world seed) and shaft parameters of a frame, the
 * shaft window centred on the frame's camera. */
uint64_t vmw_atlas_bytes(uint32_t layers);
int vmw_build_atlas(uint32_t seed, uint8_t* out);
int vmw_block_faces(uint32_t* out, uint32_t n);
int vmw_probe_field(uint32_t seed, uint16_t* out);
int vmw_shaft_envelope(const vmw_recipe* r, const float* sun_dir, const float* origin, float texel, float* out);
void vmw_look_defaults(vm_frame* f, int32_t seed);

#ifdef __cplusplus
}
#endif
#endif
