// Buffer layouts and constants of the sparse-voxel-tree march, shared by the
// host code, the CUDA kernels and the CPU oracle.
//
// Every struct here is byte-for-byte the layout the engine uploads to its
// wgpu compute pass, so a caller can hand the engine's own buffers over
// unchanged:
//   vm_frame  == GpuFrame  (src/render/mod.rs:399-459, asserts at 458-466;
//                           WGSL side src/render/shaders/common.wgsl:1-78)
//   vm_chunk  == GpuChunk  (src/render/mod.rs:469-488;
//                           WGSL side common.wgsl:80-96)
//   inner pool  = array<vec4<u32>>  (common.wgsl:100; Inner, src/voxel/geometry.rs:11-18)
//   leaf pool   = array<vec2<u32>>  (common.wgsl:101; u64 leaf masks)
//   brick pool  = array<u32>        (common.wgsl:102; src/voxel/attributes.rs)
//   grid        = array<u32>        (common.wgsl:121; src/render/mod.rs:82-86)
//   vis         = array<u64>        (common.wgsl:115; key packing common.wgsl:1320-1330)
#pragma once
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct vm_frame {
  float cam_pos[3];
  float time;
  float cam_fwd[3];
  float tan_half_fov;
  float cam_right[3];
  float aspect;
  float cam_up[3];
  float far_;          /* `far` in the reference; renamed because of <windows.h> */
  float sun_dir[3];
  float daylight;
  uint32_t res[2];
  uint32_t tiles[2];
  uint32_t chunk_count;
  uint32_t camera_chunk;
  uint32_t flags;
  uint32_t max_pairs;
  float fog_density;
  float fog_falloff;
  float shadow_dist;
  float ambient;
  float fog_scatter;
  float fog_g;
  float fog_height;
  float mip_bias;
  int32_t grid_min[3];
  float sea_level;
  uint32_t grid_dim[3];
  float water_absorb;
  float jitter[2];
  float taa_feedback;
  uint32_t frame_index;
  float cloud_cover;
  float cloud_height;
  float cloud_scale;
  float cloud_speed;
  float godray_strength;
  uint32_t godray_steps;
  float godray_dist;
  float cloud_shadow;
  float tint_strength;
  int32_t tint_seed;
  float tint_freq_t;
  float tint_freq_h;
  float wave_amp;
  float wave_scale;
  float wave_speed;
  float wave_reflect_slope;
  float shaft_origin[2];
  float shaft_texel;
  float shaft_soft;
  float cloud_patch;
  float cloud_relief;
  float haze_warm;
  float zenith_deep;
  float prev_view_proj[16];
} vm_frame;

typedef struct vm_chunk {
  float aabb_min[3];
  float voxel_size;
  float aabb_max[3];
  uint32_t lod;
  float origin[3];
  float fade;
  uint32_t root[4];     /* Inner: mask lo, mask hi, run_ptr (bit31 FULL), leaf_prefix */
  uint32_t attr_base;
  uint32_t attr_flags;
  uint32_t light_base;
  uint32_t light_flags;
  uint32_t dry_mask[2];
  uint32_t reserved[2];
} vm_chunk;

#ifdef __cplusplus
}  /* extern "C" */
#include <cstddef>
static_assert(sizeof(vm_frame) == 352, "GpuFrame is 352 bytes (src/render/mod.rs:458)");
static_assert(offsetof(vm_frame, res) == 80, "res offset");
static_assert(offsetof(vm_frame, grid_min) == 144, "grid_min offset");
static_assert(offsetof(vm_frame, grid_dim) == 160, "grid_dim offset");
static_assert(offsetof(vm_frame, jitter) == 176, "jitter offset");
static_assert(offsetof(vm_frame, cloud_cover) == 192, "src/render/mod.rs:460");
static_assert(offsetof(vm_frame, godray_strength) == 208, "src/render/mod.rs:461");
static_assert(offsetof(vm_frame, tint_strength) == 224, "src/render/mod.rs:462");
static_assert(offsetof(vm_frame, wave_amp) == 240, "src/render/mod.rs:463");
static_assert(offsetof(vm_frame, shaft_origin) == 256, "src/render/mod.rs:464");
static_assert(offsetof(vm_frame, cloud_patch) == 272, "src/render/mod.rs:465");
static_assert(offsetof(vm_frame, prev_view_proj) == 288, "src/render/mod.rs:466");
static_assert(sizeof(vm_chunk) == 96, "GpuChunk is 96 bytes");
static_assert(offsetof(vm_chunk, root) == 48, "root offset");
static_assert(offsetof(vm_chunk, attr_base) == 64, "attr_base offset");
static_assert(offsetof(vm_chunk, dry_mask) == 80, "dry_mask offset");
#endif

/* ---- constants (common.wgsl:138-263, src/render/mod.rs:20-39,82-86) ---- */
#define VM_TILE 8u                    /* src/render/mod.rs:20 */
#define VM_MAX_CHUNKS 8191u           /* src/render/mod.rs:21, 13-bit chunk field */
#define VM_MAX_PAIRS_FLOOR (1u << 20) /* src/render/mod.rs:23 */
#define VM_PAIRS_PER_TILE 16u         /* src/render/mod.rs:25 */
#define VM_TILE_ID_BITS 19u           /* src/render/mod.rs:32 */
#define VM_MAX_TILES (1u << 19)
#define VM_GRID_X 32u                 /* src/render/mod.rs:82-84 */
#define VM_GRID_Y 8u
#define VM_GRID_Z 32u
#define VM_NO_CHUNK 0xFFFFFFFFu
#define VM_FULL_BIT 0x80000000u
#define VM_PTR_MASK 0x7FFFFFFFu
#define VM_UNIFORM_BIT 0x80000000u

/* One chunk encoded into the 64-tree (build_local, src/voxel/tree.rs:89-204),
 * flat: the LocalTree fields, its L1 nodes and its variable-length arrays
 * (leaf masks, attribute entries, palette words) in the encoder's order. */
#define VM_TREE_LEAVES 4096u          /* leaf masks / attribute entries per chunk at most */
#define VM_TREE_L1 64u
#define VM_TREE_WATER 1u
#define VM_TREE_FOLIAGE 2u
#define VM_TREE_CUTOUT 4u
#define VM_TREE_GLASS 8u
#define VM_TREE_EMITTER 16u
#define VM_TREE_PALETTE_OVERFLOW 0x80000000u   /* n_palette words needed > palette_cap; palette truncated */
typedef struct vm_tree_info {
  uint64_t root_mask, dry_mask;
  int32_t uniform;               /* the block id when every solid voxel has it, else -1 */
  uint32_t flags;                /* VM_TREE_* */
  uint32_t emitters, solid_count, leaf_count;
  uint32_t n_l1, n_leaves, n_attrs, n_palette;
  uint8_t aabb_min[3], aabb_max[3];
  uint8_t pad[6];
} vm_tree_info;
typedef struct vm_tree_l1 {     /* LocalL1, src/voxel/tree.rs:37-46 */
  uint64_t mask;
  uint32_t leaf_start, leaf_prefix;
  uint8_t full, water_line;
  uint8_t pad[6];
} vm_tree_l1;
#ifdef __cplusplus
static_assert(sizeof(vm_tree_info) == 64, "vm_tree_info layout");
static_assert(sizeof(vm_tree_l1) == 24, "vm_tree_l1 layout");
#endif
#define VM_PREFIX_MASK 0x0FFFFFFFu
#define VM_MAX_ITERS 512u             /* common.wgsl:163 */

#define VM_FLAG_HIZ 1u
#define VM_FLAG_HEATMAP 2u
#define VM_FLAG_SHADOWS 4u
#define VM_FLAG_WATER_REFLECT 16u
#define VM_FLAG_WATER_REFRACT 32u
#define VM_FLAG_UNDERWATER 64u
#define VM_FLAG_WAVES 512u
#define VM_FLAG_WAVE_ANISO 1024u
#define VM_FLAG_WAVE_SHOAL 2048u
#define VM_FLAG_WAVE_FILL 4096u
#define VM_FLAG_WATER_FAR 2097152u
#define VM_FLAG_WATER_DARK 4194304u
/* the rest of the engine's frame flags word (src/render/mod.rs:140-262), read
 * by the resolve */
#define VM_FLAG_AO 8u
#define VM_FLAG_TINT 128u
#define VM_FLAG_FOLIAGE 256u
#define VM_FLAG_TERRAIN_SHAFTS 8192u
#define VM_FLAG_FLAT_SECONDARY 1048576u
#define VM_FLAG_TEX_VARIATION 16384u
#define VM_FLAG_DISTANT_SHADOWS 32768u
#define VM_FLAG_PROBE_TAP 16777216u
#define VM_FLAG_PROBE_AMBIENT 33554432u
#define VM_FLAG_PROBE_CUBE 67108864u
#define VM_FLAG_PROBE_BOUNCE 134217728u
#define VM_FLAG_LIGHT_RGB 268435456u
#define VM_FLAG_PROBE_SUN 536870912u
#define VM_FLAG_PROBE_SUN_HIGH 1073741824u
#define VM_FLAG_SKY_TINT 2147483648u
/* the resolve's material inputs (src/textures.rs:3-4, src/render/mod.rs:2240-2246,
 * src/shaft.rs:3, common.wgsl:174-178) */
#define VM_TEX_COUNT 27u              /* atlas layers (src/block.rs:37-65) */
#define VM_ATLAS_SIZE 16u
#define VM_ATLAS_MIPS 4u
#define VM_PROBE_NX 128u
#define VM_PROBE_NY 768u             /* 6 slabs (one per face normal) of 128 */
#define VM_PROBE_NZ 128u
#define VM_SHAFT_DIM 512u
/* Soft sun shadows (an extension; the engine filters one blocker distance
 * instead, shadow.wgsl:49-116): VM_SOFT_SAMPLES rays per lit-facing hit, the
 * sun direction offset inside a 0.02 rad disk, and the shadow buffer holds the
 * blocked fraction (VM_SPEC_SOFT_RAYS). */

#define VM_SOFT_SAMPLES 4u
#define VM_SOFT_ROTATIONS 16u
/* Offsets in the sun's tangent plane (radians, radius 0.02): 16 rotations of
 * a 4-point pattern (radii 0.02 sqrt((s + 1/2) / 4), golden-angle spacing),
 * one rotation per pixel and frame.  Float literals, so the CUDA kernels and
 * the CPU restatement use the same values. */
#define VM_SOFT_DISK_INIT {\
  {{0.007071067579090595f, 0.0f}, {-0.009030887857079506f, 0.008273032493889332f}, {0.0013823220506310463f, -0.01575084775686264f}, {0.01138284895569086f, 0.01484691072255373f}},\
  {{0.00653281481936574f, 0.002705980557948351f}, {-0.011509404517710209f, 0.00418731477111578f}, {0.0073046875186264515f, -0.014022893272340298f}, {0.004834714345633984f, 0.018072783946990967f}},\
  {{0.004999999888241291f, 0.004999999888241291f}, {-0.012235719710588455f, -0.0005358842317946255f}, {0.01211498025804758f, -0.010160081088542938f}, {-0.002449461491778493f, 0.018547240644693375f}},\
  {{0.002705980557948351f, 0.00653281481936574f}, {-0.011099256575107574f, -0.0051774997264146805f}, {0.015080876648426056f, -0.004750489257276058f}, {-0.009360728785395622f, 0.01619804836809635f}},\
  {{4.329780239674731e-19f, 0.007071067579090595f}, {-0.008273032493889332f, -0.009030887857079506f}, {0.01575084775686264f, 0.0013823220506310463f}, {-0.01484691072255373f, 0.01138284895569086f}},\
  {{-0.002705980557948351f, 0.00653281481936574f}, {-0.00418731477111578f, -0.011509404517710209f}, {0.014022893272340298f, 0.0073046875186264515f}, {-0.018072783946990967f, 0.004834714345633984f}},\
  {{-0.004999999888241291f, 0.004999999888241291f}, {0.0005358842317946255f, -0.012235719710588455f}, {0.010160081088542938f, 0.01211498025804758f}, {-0.018547240644693375f, -0.002449461491778493f}},\
  {{-0.00653281481936574f, 0.002705980557948351f}, {0.0051774997264146805f, -0.011099256575107574f}, {0.004750489257276058f, 0.015080876648426056f}, {-0.01619804836809635f, -0.009360728785395622f}},\
  {{-0.007071067579090595f, 8.659560479349462e-19f}, {0.009030887857079506f, -0.008273032493889332f}, {-0.0013823220506310463f, 0.01575084775686264f}, {-0.01138284895569086f, -0.01484691072255373f}},\
  {{-0.00653281481936574f, -0.002705980557948351f}, {0.011509404517710209f, -0.00418731477111578f}, {-0.0073046875186264515f, 0.014022893272340298f}, {-0.004834714345633984f, -0.018072783946990967f}},\
  {{-0.004999999888241291f, -0.004999999888241291f}, {0.012235719710588455f, 0.0005358842317946255f}, {-0.01211498025804758f, 0.010160081088542938f}, {0.002449461491778493f, -0.018547240644693375f}},\
  {{-0.002705980557948351f, -0.00653281481936574f}, {0.011099256575107574f, 0.0051774997264146805f}, {-0.015080876648426056f, 0.004750489257276058f}, {0.009360728785395622f, -0.01619804836809635f}},\
  {{-1.2989341236012077e-18f, -0.007071067579090595f}, {0.008273032493889332f, 0.009030887857079506f}, {-0.01575084775686264f, -0.0013823220506310463f}, {0.01484691072255373f, -0.01138284895569086f}},\
  {{0.002705980557948351f, -0.00653281481936574f}, {0.00418731477111578f, 0.011509404517710209f}, {-0.014022893272340298f, -0.0073046875186264515f}, {0.018072783946990967f, -0.004834714345633984f}},\
  {{0.004999999888241291f, -0.004999999888241291f}, {-0.0005358842317946255f, 0.012235719710588455f}, {-0.010160081088542938f, -0.01211498025804758f}, {0.018547240644693375f, 0.002449461491778493f}},\
  {{0.00653281481936574f, -0.002705980557948351f}, {-0.0051774997264146805f, 0.011099256575107574f}, {-0.004750489257276058f, -0.015080876648426056f}, {0.01619804836809635f, 0.009360728785395622f}}}

#define VM_ATTR_UNIFORM 1u
#define VM_ATTR_HAS_WATER 2u
#define VM_ATTR_HAS_FOLIAGE 4u
#define VM_ATTR_HAS_CUTOUT 8u
#define VM_ATTR_HAS_GLASS 16u
#define VM_ATTR_HAS_EMITTER 32u

/* block ids (src/block.rs:3-35) */
#define VM_AIR 0u
#define VM_STONE 1u
#define VM_DIRT 2u
#define VM_GRASS 3u
#define VM_SAND 4u
#define VM_GRAVEL 5u
#define VM_LOG 6u
#define VM_LEAVES 7u
#define VM_PLANKS 8u
#define VM_GLASS 10u
#define VM_GLOWSTONE 11u
#define VM_BEDROCK 12u
#define VM_WATER 13u
#define VM_PINE_LEAVES 16u
#define VM_TALL_GRASS 18u
#define VM_MEADOW 19u
#define VM_AMBER_LAMP 20u
#define VM_AZURE_LAMP 21u
#define VM_VERDANT_LAMP 22u
#define VM_GRASS_TALL 24u
#define VM_REEDS 25u
#define VM_BLOCK_COUNT 26u

/* WGSL override defaults that reach the march (common.wgsl:180-263) */
#define VM_LEAF_FILL 0.62f
#define VM_LEAF_FILL_PRE43 0.72f    /* SPEC_LEAF_FILL without FLAG_LEAF_THIN (src/render/mod.rs:321-323,2500-2506) */

/* Pipeline specialisations of the march (the engine's override constants,
 * make_spec src/render/mod.rs:2355-2689, common.wgsl:180-262), set per
 * context with vm_set_spec.  VM_SPEC_DEFAULT is the engine's default
 * configuration (src/config.rs:305-348). */
#define VM_SPEC_FULL_MARCH 1u       /* SPEC_FULL_MARCH: march full roots (else the full-root shortcut, common.wgsl:677-686) */
#define VM_SPEC_WATER_REPAIR 2u     /* SPEC_WATER_REPAIR: the water-interface repair (common.wgsl:666) */
#define VM_SPEC_LEAF_CUTOUT 4u      /* SPEC_LEAF_CUTOUT: micro-voxel leaves (common.wgsl:643-649) */
#define VM_SPEC_GLASS 8u            /* SPEC_GLASS: glass transparent to shadow / secondary rays, its own legs */
#define VM_SPEC_EMITTER_GATHER 16u  /* SPEC_EMITTER_GATHER: emitters cast no sun shadow (common.wgsl:664) */
#define VM_SPEC_FOLIAGE 32u         /* SPEC_FOLIAGE: tuft blocks are foliage (else plain solid cubes) */
#define VM_SPEC_SNELL_BEND 64u      /* SPEC_SNELL_BEND: bent primary rays from underwater (march.wgsl:23-44) */
#define VM_SPEC_LEAF_THIN 128u      /* FLAG_LEAF_THIN: SPEC_LEAF_FILL = 0.62, else 0.72 */
#define VM_SPEC_DEFAULT (VM_SPEC_FULL_MARCH | VM_SPEC_WATER_REPAIR | VM_SPEC_LEAF_CUTOUT | VM_SPEC_GLASS | \
                         VM_SPEC_EMITTER_GATHER | VM_SPEC_FOLIAGE | VM_SPEC_LEAF_THIN)
#define VM_SPEC_ALL 255u
/* Extension, outside the engine's spec set: soft shadows, VM_SOFT_SAMPLES jittered
 * sun rays per lit-facing hit whose shadow buffer entry is the blocked fraction.
 * Every bit of the engine's frame flags word is taken, so the switch is a
 * specialisation of the context, not a frame flag. */
#define VM_SPEC_SOFT_RAYS 256u
/* SPEC_WIND_SWAY (FLAG_HI_WIND_SWAY, src/render/mod.rs:232): tuft quads sheared by the wind
 * (common.wgsl:419-423, 433-447); off in the engine's default configuration. */
#define VM_SPEC_WIND_SWAY 512u
#define VM_SURFACE_EPS 0.02f          /* common.wgsl:1258 */
#define VM_WATER_IOR 1.333f           /* common.wgsl:1256 */
#define VM_WATER_REFRACT_DIST 96.0f   /* resolve.wgsl:879 */
#define VM_WATER_REFRACT_NEAR 96.0f   /* resolve.wgsl:873 */
#define VM_WATER_REFRACT_FAR 192.0f   /* resolve.wgsl:874 */
#define VM_GLASS_TRANSMIT_DIST 192.0f /* resolve.wgsl:886 */
#define VM_WATER_REFLECT_NEAR 512.0f  /* resolve.wgsl:876 */
#define VM_WATER_REFLECT_FAR 1024.0f  /* resolve.wgsl:877 */
#define VM_WATER_REFLECT_DIST 768.0f  /* resolve.wgsl:880 */
#define VM_WATER_FAR_DIST 128.0f      /* common.wgsl:165 */
#define VM_WATER_DARK_DEPTH 15.0f     /* common.wgsl:167 */
#define VM_WATER_DARK_DIST 64.0f      /* common.wgsl:172 */

/* normal ids (common.wgsl:387-398) */
#define VM_NORMAL_PY 3u
#define VM_NORMAL_CROSS_A 6u
#define VM_NORMAL_CROSS_B 7u
