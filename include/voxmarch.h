/* voxmarch: the sparse-voxel-tree ray march of the voxel engine
 * Vuk03-boop/voxelcraft-menu, as CUDA kernels for one B200 (sm_100a) behind a
 * flat C ABI.
 *
 * The engine runs this path as wgpu compute passes inside Renderer::render
 * (src/render/mod.rs:1593-1919).  Every call below replaces one piece of that
 * host code, keeps the engine's buffer layouts byte for byte (vm_frame ==
 * GpuFrame, vm_chunk == GpuChunk, inner / leaf / brick pools, chunk grid,
 * 64-bit visibility keys) and is stream-ordered on the context's stream.
 *
 * Conventions
 *  - Every call returns a vm_status; on error vm_last_error() has the text.
 *  - Host arrays are read (or written) only during the call.  The context owns
 *    all device buffers; vm_device_buffers() exposes them for zero-copy use.
 *  - One context per host thread; no internal threads.
 *  - Read calls synchronise the context's stream; all others only enqueue.
 */
#ifndef VOXMARCH_H
#define VOXMARCH_H
#include <stddef.h>
#include <stdint.h>
#include "../voxelcraft_menu_b200/csrc/vm_types.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef enum vm_status {
  VM_OK = 0,
  VM_E_INVALID = 1,        /* bad argument or malformed buffer */
  VM_E_CAPACITY = 2,       /* pair list truncated: the engine's TRUNCATION_MARK (src/render/mod.rs:37,1957-1975) */
  VM_E_TILE_OVERFLOW = 3,  /* tile index does not fit the 19-bit pair field: OVERSIZE_MARK (src/render/mod.rs:39,2047-2060) */
  VM_E_ITER_CAP = 4,       /* informational: some march hit MAX_ITERS (common.wgsl:698-701); counted, not fatal */
  VM_E_TIMEOUT = 5,        /* a bounded device wait gave up */
  VM_E_CUDA = 6,           /* CUDA runtime error */
  VM_E_NOT_READY = 7,      /* call order: e.g. march before world / frame */
  VM_E_TOO_LARGE = 8       /* the frame exceeds a fixed limit of vm_render_static (nothing was run) */
} vm_status;

typedef struct vm_ctx vm_ctx;

typedef struct vm_caps {
  uint32_t max_width, max_height;   /* largest frame this context renders */
  uint32_t max_chunks;              /* largest chunk list (<= 8191 for the 13-bit field) */
  uint32_t max_views;               /* largest batch (vm_batch_*) */
  uint64_t max_batch_pixels;        /* total pixels of a batch */
} vm_caps;

/* Renderer::new (src/render/mod.rs:851): device buffers for one renderer. */
int vm_create(int device_ordinal, const vm_caps* caps, vm_ctx** out);
void vm_destroy(vm_ctx* ctx);
const char* vm_last_error(const vm_ctx* ctx);
/* Run on a caller stream (cudaStream_t as void*); NULL restores the context's own. */
int vm_set_stream(vm_ctx* ctx, void* cuda_stream);

/* Renderer::sync_world (src/render/mod.rs:1355-1396): replace the three pools.
 * inners: n_inners x vec4<u32> (common.wgsl:100); leaves: n_leaves x vec2<u32>
 * (common.wgsl:101); bricks: n_bricks x u32 (common.wgsl:102). */
int vm_upload_world(vm_ctx* ctx, const uint32_t* inners, uint64_t n_inners, const uint32_t* leaves,
                    uint64_t n_leaves, const uint32_t* bricks, uint64_t n_bricks);
/* GpuMirror dirty-range upload (src/render/pools.rs): pool 0 inners, 1 leaves,
 * 2 bricks; offset and count in that pool's elements; the pool grows if needed. */
int vm_update_pool(vm_ctx* ctx, int pool, uint64_t offset, const uint32_t* data, uint64_t count);
/* build_chunk_list's uploads (src/render/mod.rs:1555-1562): the chunk list
 * (visible chunks first, then shadow-only ones) and the chunk grid. */
int vm_upload_chunks(vm_ctx* ctx, const vm_chunk* chunks, uint32_t n_chunks, const uint32_t* grid, uint64_t grid_len);
/* queue.write_buffer of GpuFrame (src/render/mod.rs:1707).  A sun_dir with a
 * zero component is accepted (the engine's sun(t), src/scene.rs:10-14, has
 * dir.y == 0 at t = 0.25 with shadows on): as in shadow_ray_t
 * (common.wgsl:1157) the reciprocal is then an IEEE infinity and the shadow
 * DDA runs on IEEE arithmetic (NaN comparisons false, NaN -> 0 conversions,
 * wrapping i32 subtraction), the same operations as the oracle's. */
int vm_set_frame(vm_ctx* ctx, const vm_frame* frame);

/* The engine's passes, one call per group of dispatches (src/render/mod.rs:1716-1851):
 * vm_select   = clear vis / counters (hiz too unless FLAG_HIZ) + tile_select + finalize (1716-1749)
 * vm_march    = march; with FLAG_HIZ also build_hiz, finalize_deferred,
 *               recover_select, finalize_recover and the second march (1751-1794)
 * vm_primary_shadow = primary_shadow (1824-1841), blocker distance per pixel
 * vm_secondary      = one water-refraction / glass-transmission ray per hit
 *                     (water_refract_leg resolve.wgsl:1029, shade_glass resolve.wgsl:1261) */
int vm_select(vm_ctx* ctx);
int vm_march(vm_ctx* ctx);
int vm_primary_shadow(vm_ctx* ctx);
int vm_secondary(vm_ctx* ctx);

/* shadow_horizontal + shadow_vertical (src/render/shaders/shadow.wgsl:62-116,
 * stages 1 and 2 of src/render/mod.rs:1827-1840) with SPEC_SOFT_SHADOWS on: the
 * bilateral reconstruction of the sun shadow from the frame's blocker
 * distances (the vis and shadow buffers of vm_render or vm_march +
 * vm_primary_shadow), guided by shadow_guide (shadow.wgsl:7-31).
 * radius_limit = SHADOW_RADIUS_LIMIT (1..8; the engine uses 4, or 8 with
 * FLAG_HI_SOFT_HQ, src/render/mod.rs:2660), penumbra = SOFT_PENUMBRA (1.0,
 * 1.5 or 3.0, src/render/mod.rs:2664).  The distances are read as the engine's
 * r16float target stores them and the horizontal pass is rounded as its
 * rg16float target stores it.  Output (vm_read_shadow_mask): per pixel the
 * shadow mask clamp(1 - occlusion, 0, 1) as a float, the value the engine
 * quantises into its r8unorm target; 1 = lit.  A context with
 * VM_SPEC_SOFT_RAYS (jittered rays, whose shadow buffer holds blocked
 * fractions) is rejected with VM_E_INVALID. */
int vm_soften_shadows(vm_ctx* ctx, uint32_t radius_limit, float penumbra);

/* The same frame as vm_select + vm_march + vm_primary_shadow + vm_secondary
 * as a warp-independent wavefront pipeline (per-tile cull, front-to-back
 * primary march with an exact early out, queued shadow and secondary rays);
 * identical vis / shadow / secondary output.  hiz receives the final
 * visibility's per-8x8-tile minimum. */
int vm_render(vm_ctx* ctx);

/* Tuning of vm_render and vm_batch_run's primary-ray kernel: warps per block
 * (4 or 8), register budget as the resident warps per SM it must allow
 * (0 unconstrained, 1 24 warps ~80 registers, 2 32 warps 64 registers,
 * 3 20 warps ~100 registers, 4 16 warps 128 registers) and resident blocks
 * per SM (0 = occupancy maximum). */
int vm_set_tuning(vm_ctx* ctx, int warps_per_block, int reg_level, int ctas_per_sm);
/* Packet size of the same kernel: pixels each lane marches (1: a warp takes
 * 8x4-pixel items, half an 8x8 tile; 2: whole 8x8 tiles, a lane starting its
 * second pixel as soon as its first is done).  Output is identical; no
 * counterpart in the engine, which runs one 64-thread group per (tile, chunk)
 * pair (march.wgsl:1-55). */
int vm_set_packet(vm_ctx* ctx, int pixels_per_lane);
/* The engine's pipeline specialisations of the march (make_spec,
 * src/render/mod.rs:2355-2689): VM_SPEC_* bits (vm_types.h), VM_SPEC_DEFAULT
 * on creation.  They select the full-root shortcut (--no-full-march), the
 * water-interface repair (--legacy-water), leaf cutouts (--no-leaf-cutout),
 * glass as its own surface, emitters without sun shadow, tufts as foliage, the
 * Snell bend of underwater primary rays (--snell-bend) and the leaf fill
 * (--no-leaf-thin).  VM_SPEC_SOFT_RAYS (an extension, no engine counterpart)
 * traces VM_SOFT_SAMPLES jittered sun rays per lit-facing hit and stores the
 * blocked fraction in the shadow buffer.  Unknown bits: VM_E_INVALID. */
int vm_set_spec(vm_ctx* ctx, uint32_t spec);

/* Read-backs (synchronise the context's stream). */
int vm_read_vis(vm_ctx* ctx, uint64_t* out);                 /* res.x*res.y keys (common.wgsl:1324) */
int vm_read_hiz(vm_ctx* ctx, uint32_t* out);                 /* tiles.x*tiles.y */
int vm_read_shadow(vm_ctx* ctx, float* out);                 /* blocker distance, 0 = lit */
int vm_read_secondary(vm_ctx* ctx, uint64_t* key, float* t); /* see below */
int vm_read_heatmap(vm_ctx* ctx, uint32_t* out);             /* FLAG_HEATMAP iteration sums (march.wgsl:51-53) */
int vm_read_shadow_mask(vm_ctx* ctx, float* out);            /* vm_soften_shadows output (shadow.wgsl:115) */
/* The reflect leg of every water hit (water_reflect_leg, resolve.wgsl:1044-1058,
 * traced per hit as the refract leg is) of the last vm_render / vm_secondary
 * frame with FLAG_WATER_REFLECT: key as vm_read_secondary's (bit 61 clear) and
 * t; key 0 where the pixel has none (no water, or reflect_detail 0 beyond
 * 1024 voxels).  The leg leaves along water_ctx's mirror_t: the face normal's
 * reflection, on a waved +Y face (FLAG_WAVES) the wave normal's
 * (resolve.wgsl:1107-1163, with FLAG_WAVE_ANISO / _SHOAL / _FILL, the frame's
 * time and wave_* fields).  The first such frame grows the
 * context's buffers (12 bytes per pixel, and a secondary queue of 2 items per
 * pixel); VM_E_NOT_READY after a frame without the flag. */
int vm_read_reflection(vm_ctx* ctx, uint64_t* key, float* t);
/* The engine's schedule of the water legs (water_sec, resolve.wgsl:1468-1535,
 * WATER_SEC_SHIFT = 1), over the visibility of the last frame: for every
 * (1 << shift)^2 pixel block (shift 0..3), its water pixel nearest the camera
 * (smallest hit_t; the first in x-major order on a tie) traces the refract leg
 * (FLAG_WATER_REFRACT, water_refract_leg) and the reflect leg
 * (FLAG_WATER_REFLECT, water_reflect_leg, along water_ctx's mirror_t,
 * waved surfaces included).  vm_read_water_sec then returns
 * ceil(res.x / 2^shift) * ceil(res.y / 2^shift) cells, row-major: keys as
 * vm_read_secondary's (0 = no leg) and the legs' hit distances.  Any pointer
 * may be NULL.  The cell buffers are allocated by the first call. */
int vm_water_sec(vm_ctx* ctx, uint32_t shift);
int vm_read_water_sec(vm_ctx* ctx, uint64_t* refr_key, float* refr_t, uint64_t* refl_key, float* refl_t);

/* The resolve: the engine's resolve pass (src/render/shaders/resolve.wgsl:
 * 1378-1466, its three lanes).  Opaque surfaces: shade_hit_legacy_cached
 * (resolve.wgsl:1537-1788: atlas texel with texture variation, biome tint,
 * shore wetting, smooth light with AO from the light bricks, the frame's sun
 * visibility, distant terrain shadow, cloud shadow, probe field, sky
 * specular).  Water: water_ctx and water_compose (resolve.wgsl:1078-1221:
 * body colour, wave normals, foam, glint, the refract leg through the water
 * medium and the reflect leg, each leg's hit shaded with a traced sun test),
 * the legs from the half-resolution water_sec pass (FLAG_HI_WATER_SEC: a
 * 2x2 block's nearest water pixel, through the engine's rgba16float targets;
 * blocks that are not one flat water plane trace their own legs) or per
 * pixel.  Glass: shade_glass (resolve.wgsl:1261-1319: transmission, the
 * reflection, FLAG_HI_GLASS_REFLECT).  Then the fog blend toward sky_base
 * with the sun shafts; sky pixels get sky_color with clouds.
 *
 * Material inputs, set once (the engine's own buffers):
 *   vm_upload_atlas        the block atlas as make_atlas uploads it
 *                          (src/render/mod.rs:2159-2222): Rgba8UnormSrgb,
 *                          layers x 16 x 16, mips 16, 8, 4, 2 one after the
 *                          other (each [layer][y][x][rgba]); decoded to
 *                          linear float here.  Replaces textureSampleLevel on
 *                          `atlas` (mag nearest, min / mipmap linear, clamp).
 *   vm_upload_block_faces  block_faces (src/block.rs:265-276 face_table): 8
 *                          words per block id, layer | perm class << 16.
 *   vm_upload_probes       the probe field (src/render/mod.rs:2248-2300):
 *                          RGBA16F, 128 x 768 x 128; NULL: the engine's
 *                          initial fill of 1.0.
 *   vm_upload_shaft        the shaft pass's envelope (the SHAFT_RESULT slice
 *                          of `shaft`, common.wgsl:174-178): 512 x 512 f32;
 *                          NULL: no terrain shadow (shade 1).
 * vm_resolve(ctx, spec_hi): after vm_render (and vm_soften_shadows when the
 * engine's SPEC_SOFT_SHADOWS is on: its mask is then the sun visibility, as
 * the engine's primary_sun texture), spec_hi = the engine's FLAG_HI_* word
 * (src/render/mod.rs:196-300; SKY_SPECULAR, SHORE_WET, SHORE_FOAM,
 * WATER_SEC, CAUSTICS, GLASS_REFLECT, TINT_BALANCE, SKY_LOOK, SKY_COOL,
 * FOLIAGE_RICH, CANOPY_RELIEF, LEGACY_LIGHTING are read; COMPACT_SHADE_HIT
 * is accepted and gives the same colours (the compact shade_hit reorders the
 * legacy one's statements); WATER_LOOK and the surface debug views
 * (DEBUG_A..C, SURFACE_DEBUG = spec_hi >> 23 & 7) are read; a FLAG_HEATMAP
 * frame resolves to the heat map of the
 * iteration counts of vm_select / vm_march, VM_E_NOT_READY without them).
 * The frame flags give the rest
 * (AO, TINT, TEX_VARIATION, DISTANT_SHADOWS, TERRAIN_SHAFTS, FLAT_SECONDARY,
 * WAVES..., PROBE_CUBE / BOUNCE / SUN / SUN_HIGH / TAP / AMBIENT, LIGHT_RGB,
 * SKY_TINT, WATER_REFRACT / REFLECT, UNDERWATER, SNELL), as make_spec
 * derives them; WATER_SEC_SHIFT is 1 (the engine's water_sec_scale 2).
 * vm_resolve issues its work on the context's stream (vm_set_stream); the
 * water and glass lanes run on three streams of the context forked from it
 * with events and joined back before the call returns, so the call can be
 * recorded into a stream capture of the caller's stream.
 * vm_read_color: res.x * res.y RGBA float (alpha 1), the value the engine
 * stores into its rgba16float target. */
int vm_upload_atlas(vm_ctx* ctx, const uint8_t* rgba, uint32_t layers, uint32_t size, uint32_t mips);
int vm_upload_block_faces(vm_ctx* ctx, const uint32_t* words, uint32_t n);
int vm_upload_probes(vm_ctx* ctx, const uint16_t* rgba16f, uint32_t nx, uint32_t ny, uint32_t nz);
int vm_upload_shaft(vm_ctx* ctx, const float* envelope, uint32_t dim);
int vm_resolve(vm_ctx* ctx, uint32_t spec_hi);
int vm_read_color(vm_ctx* ctx, float* rgba);
/* Expanded visibility: voxel index X*(Z*y + z) + x over the world box
 * [origin, origin + dims), face = normal id (common.wgsl:387), t = hit_t
 * (common.wgsl:1300).  Misses: voxel 0xFFFFFFFF, face 0xFF, t 0. */
int vm_read_expanded(vm_ctx* ctx, const int32_t origin[3], const uint32_t dims[3], uint32_t* voxel, uint8_t* face,
                     float* t);
/* The visibility and shadow buffers copied to host memory without waiting:
 * the copies are enqueued on the context's stream, and the host buffers hold
 * the frame once that stream is synchronised (vm_sync or an event).  With
 * page-locked host buffers the copy overlaps other work, e.g. the next frame
 * of a second context.  Either pointer may be NULL. */
int vm_read_async(vm_ctx* ctx, uint64_t* vis, float* shadow);
/* vm_read_async with the blocker distances in the engine's own shadow target
 * format: shadow_dist_tex is texture_storage_2d<r16float> (shadow.wgsl:1),
 * so shadow receives res.x*res.y binary16 values (IEEE half, rounded to
 * nearest even from the float blocker distances): 10 bytes per pixel cross
 * the host link instead of 12.  Either pointer may be NULL. */
int vm_read_async_r16f(vm_ctx* ctx, uint64_t* vis, uint16_t* shadow);
/* Frames in flight over several contexts on one device: work enqueued on ctx
 * after this call waits until other's last vm_render has finished its
 * kernels, but not for other's read-back.  A caller that alternates two
 * contexts and calls this before each vm_render runs the frames' kernels
 * one after another, each on the whole GPU, while the previous frame's
 * read-back crosses the host link.  No counterpart in the engine, which keeps
 * its frames in flight inside wgpu's queue.  No-op if other has not rendered. */
int vm_wait_render(vm_ctx* ctx, vm_ctx* other);
/* Hi-Z input of the next FLAG_HIZ frame (the engine keeps last frame's buffer). */
int vm_write_hiz(vm_ctx* ctx, const uint32_t* hiz);

/* secondary key: 0 = no secondary ray for the pixel; else bit 63 traced,
 * bit 62 hit, bit 61 glass (else water), bits 37-39 normal, 24-36 chunk,
 * 0-23 voxel (x<<16 | y<<8 | z); t = distance along the ray, max on a miss. */

/* Renderer::pair_demand / march_stats (src/render/mod.rs:1948-2045). */
typedef struct vm_stats {
  uint32_t counters[8];     /* the engine's counters[0..5] after the last vm_march */
  uint32_t pairs_selected, pairs_deferred, pairs_recovered, max_pairs;
  uint32_t truncated;       /* 1 if any list exceeded max_pairs */
  uint32_t device_error;    /* nonzero: a pool index was out of range (bit set per pool) */
} vm_stats;
int vm_stats_read(vm_ctx* ctx, vm_stats* out);

/* Traffic counted by the instrumented fused kernel (one extra launch):
 * chunk records, L1 / leaf / attribute fetches, palette decodes, grid
 * lookups, DDA iterations, and rays of each kind. */
typedef struct vm_traffic {
  uint64_t chunk_records, l1_fetches, leaf_fetches, attr_fetches, palette_decodes, grid_lookups, iters;
  uint64_t rays_primary, rays_shadow, rays_secondary;
  uint64_t list_entries;    /* tile-list entries the primary rays examined */
  uint64_t stage_iters[3];  /* DDA steps of the primary, shadow and secondary rays */
  uint64_t stage_chunks[3]; /* chunk marches of the primary, shadow and secondary rays */
  uint64_t stage_bytes[3];  /* algorithmic bytes of each stage's traversal: 96 per chunk record, 16 per L1
                               node, 8 per leaf mask, 4 per attribute word, 12 per palette decode, 4 per
                               grid lookup */
} vm_traffic;
int vm_render_counted(vm_ctx* ctx, vm_traffic* out);

/* vm_render that also records five caller-created CUDA events (cudaEvent_t
 * as void*) on the context's stream: at the start, after the tile cull, and
 * after the primary, shadow and secondary kernels, so a caller can time each
 * stage.  No counterpart in the engine, which times whole passes with
 * timestamp queries (src/render/mod.rs:1593-1919). */
int vm_render_events(vm_ctx* ctx, void* const* events);

/* Batched views: many frames (each with its own chunk list and grid) marched
 * by one persistent work-stealing launch (VM_BATCH_PERSISTENT, replayed from
 * a CUDA graph) or by one launch sequence per view (VM_BATCH_PER_VIEW, the
 * baseline), optionally | VM_BATCH_SECONDARY to also trace the water / glass
 * rays (needed by vm_shade_gbuffer).  Views are packed in order; their
 * outputs are concatenated in the batch buffers.  The engine renders one
 * view per Renderer::render (src/render/mod.rs:1593); its probe and lookbook
 * views are separate dispatches, which VM_BATCH_PER_VIEW reproduces. */
#define VM_BATCH_PERSISTENT 0
#define VM_BATCH_PER_VIEW 1
#define VM_BATCH_SECONDARY 2
int vm_batch_set(vm_ctx* ctx, uint32_t n_views, const vm_frame* frames, const vm_chunk* chunks,
                 const uint32_t* chunk_counts, const uint32_t* grids, const uint32_t* grid_lens);
int vm_batch_run(vm_ctx* ctx, int mode);
int vm_batch_read(vm_ctx* ctx, uint64_t* vis, float* shadow);
/* One instrumented run of the whole batch (as VM_BATCH_PERSISTENT, with the
 * secondary rays when secondary != 0): same outputs, plus its traffic. */
int vm_batch_counted(vm_ctx* ctx, int secondary, vm_traffic* out);
/* the secondary rays' keys and distances of the last VM_BATCH_SECONDARY run */
int vm_batch_read_secondary(vm_ctx* ctx, uint64_t* key, float* t);
uint64_t vm_batch_pixels(const vm_ctx* ctx);

/* Differentiable shading over a fixed visibility buffer.  The engine has no
 * such stage: its shading lives in resolve.wgsl:1379-1466.  This pair restates
 * the terms sun N.L with the shadow verdict, sky ambient, height fog
 * (common.wgsl:1332-1341) and Beer-Lambert water absorption
 * (common.wgsl:1262-1265) as a smooth function of VM_SHADE_NPARAMS floats:
 * [0,768) albedo table 256 x 3, [768,771) sun direction (normalised inside),
 * [771,774) sky ambient RGB, 774 fog density, [775,778) water absorption RGB.
 *
 * vm_shade_gbuffer writes one vm_shade_gbuf per pixel of the last batch
 * (vm_batch_run with VM_BATCH_SECONDARY).  The fog's optical length per unit
 * density (e * path of transmittance_from) depends on the geometry and the
 * fog falloff / height only, so it is computed there once.  vm_shade_forward
 * writes RGB per pixel (and/or adds the L2 loss against d_target into
 * *d_loss); vm_shade_backward adds dL/dparams into d_grad_params (FP64) for
 * dL/dcolour = d_grad_color, or for the L2 loss against d_target when
 * d_grad_color is NULL, in which case it also adds that loss into *d_loss when
 * d_loss is not NULL (forward and backward fused).  All pointers are device
 * pointers on the current device; work is enqueued on cuda_stream. */
#define VM_SHADE_NPARAMS 778
#define VM_SHADE_GBUF_BYTES 16
typedef struct vm_shade_consts {
  float sun_rgb[3];        /* sun colour times the engine's 0.78 gain */
  float fog_falloff, fog_height;
} vm_shade_consts;
typedef struct vm_shade_gbuf {
  uint32_t code;           /* id | face << 8 | HIT 1<<11 | LIT 1<<12 | TRACED 1<<13 | HIT2 1<<14 | FLIP 1<<15
                              | id2 << 16 | face2 << 24 (id2 / face2: the refracted ray's hit)
                              | blocked soft-shadow rays << 27 | SOFT 1<<30 (VM_SPEC_SOFT_RAYS) */
  float t;                 /* primary hit distance (0 for sky) */
  float d;                 /* water refraction leg length */
  float fog;               /* fog optical length per unit density (0 for sky) */
} vm_shade_gbuf;
int vm_shade_gbuffer(vm_ctx* ctx, const vm_shade_consts* consts, void* d_gbuf);
int vm_shade_forward(const void* d_gbuf, uint64_t n_pixels, const float* d_params, const vm_shade_consts* consts,
                     float* d_color, const float* d_target, double* d_loss, void* cuda_stream);
int vm_shade_backward(const void* d_gbuf, uint64_t n_pixels, const float* d_params, const vm_shade_consts* consts,
                      const float* d_grad_color, const float* d_target, double* d_grad_params, double* d_loss,
                      void* cuda_stream);

/* The engine's dense -> 64-tree encoder (build_local, src/voxel/tree.rs:89-204,
 * with encode_leaf src/voxel/attributes.rs:90-139) for n_chunks dense chunks
 * at once, on the GPU; the engine runs it per chunk on the CPU (its
 * --bench-terrain "tree build").  Device pointers, enqueued on cuda_stream:
 * d_dense n_chunks x 64^3 block ids (index x | z<<6 | y<<12 within a chunk);
 * per chunk c: d_info[c], d_l1[64 c ..], d_leaves[4096 c ..],
 * d_attrs[4096 c ..], d_palette[palette_cap c ..] in the layout of
 * vm_tree_info (vm_types.h).  A chunk whose palette needs more than
 * palette_cap words has VM_TREE_PALETTE_OVERFLOW set, n_palette = the words
 * needed and its first palette_cap words written.  The output equals vmw_build_tree's (the CPU restatement) and
 * vmw_insert_tree puts it into a world.  No context, no allocation. */
int vm_encode_trees(const uint16_t* d_dense, uint32_t n_chunks, uint32_t palette_cap, vm_tree_info* d_info,
                    vm_tree_l1* d_l1, uint64_t* d_leaves, uint32_t* d_attrs, uint32_t* d_palette, void* cuda_stream);

/* Device pointers of the context's buffers (valid until the next upload that
 * grows them), for zero-copy callers such as a torch binding. */
typedef struct vm_device_ptrs {
  void* vis; void* shadow; void* sec_key; void* sec_t; void* hiz;
  void* batch_vis; void* batch_shadow;
  void* stream;
} vm_device_ptrs;
int vm_device_buffers(vm_ctx* ctx, vm_device_ptrs* out);

/* Synchronise the context's stream. */
int vm_sync(vm_ctx* ctx);

/* Frame march that allocates nothing (this entry point has no counterpart in
 * the reference).  For callers that cannot call cudaMalloc: code inside a
 * stream capture it does not own, engines that hand out all device memory
 * from their own arenas, allocation-free real-time paths.  The caller passes
 * every input and output as device pointers (pools, chunk list, grid, vis,
 * shadow, a zeroed u32 error word) on the current device and stream; the
 * pipeline's scratch is one static device array of 8,650,900 bytes (8.25 MiB)
 * per GPU.  Primary and shadow rays only; at most 262144 pixels and 8192 8x8
 * tiles per frame (larger frames return VM_E_TOO_LARGE and run nothing).  The first call on a device
 * looks the array up and must come before any stream capture.  Every call
 * shares the array: calls that overlap on the GPU race.
 * vm_static_last_error() describes the last failure of this thread. */
int vm_render_static(const vm_frame* frame, const vm_chunk* d_chunks, uint32_t n_chunks, const uint32_t* d_grid,
                     uint64_t grid_len, const uint32_t* d_inners, uint64_t n_inners, const uint32_t* d_leaves,
                     uint64_t n_leaves, const uint32_t* d_bricks, uint64_t n_bricks, uint64_t* d_vis,
                     float* d_shadow, uint32_t* d_error, void* cuda_stream);
const char* vm_static_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
