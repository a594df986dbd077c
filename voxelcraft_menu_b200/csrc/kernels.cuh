// Kernel declarations and launch helpers shared by the ABI layer.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "vm_types.h"
#include "march_device.cuh"

namespace vmd { struct Look; }

namespace vmk {

// One view of a (possibly batched) frame pipeline.  Views own consecutive
// ranges of chunks, grid cells, 8x8 tiles and pixels in the batch buffers.
struct ViewDesc {
  uint32_t chunk_off;     // first chunk of this view in the concatenated chunk list
  uint32_t n_chunks;      // chunks of this view (visible + shadow-only)
  uint64_t grid_off;      // first grid cell of this view
  uint32_t grid_len;
  uint32_t tile_begin;    // first 8x8 tile of this view (also its hiz offset)
  uint32_t tiles_x, tiles_y;   // 8x8 tiles of this view (the engine's tile grid)
  uint64_t pix_off;       // first pixel of this view in the output buffers
  uint32_t super_begin;   // first 32x32-pixel super-tile of this view (4x4 tiles)
  uint32_t pad;
};
static_assert(sizeof(ViewDesc) == 48, "ViewDesc layout");

struct Traffic64 {
  unsigned long long chunk, l1, leaf, attr, pal, grid, iters, rays_primary, rays_shadow, rays_secondary, entries;
};

// Queued secondary work, written by the primary kernel and consumed densely.
struct ShadowItem { uint32_t view, pix; float o[3]; uint32_t pad; };                 // 24 B
// kind: SEC_GLASS, SEC_REFRACT (water refract leg) or SEC_REFLECT (water reflect leg)
enum : uint32_t { SEC_GLASS = 0u, SEC_REFRACT = 1u, SEC_REFLECT = 2u };
struct SecItem { uint32_t view, pix; float o[3], d[3]; float max_dist; uint32_t kind; };  // 40 B

// Pipeline counters (zeroed before each frame)
// Cost order of the primary kernel's work.  Consecutive launches over the
// same tiles (the next frame, a replayed batch) see nearly the same rays, so
// the primary kernel records each item's duration (SM cycles) and the next
// launch takes the tiles in decreasing order of that cost: the few items
// whose rays run long (up to the 512-step cap in a chunk, or through tree
// canopies) start first instead of last, where they would hold the frame's
// tail.  The order only decides when an item starts, never what it computes.
constexpr uint32_t N_COST_BUCKETS = 16;
__device__ __forceinline__ uint32_t cost_bucket(uint32_t cycles) {
  // log2 buckets, 0 the most expensive (>= 2^20 cycles, about 0.5 ms)
  const uint32_t lg = cycles ? 31u - (uint32_t)__clz(cycles) : 0u;
  return lg >= 20u ? 0u : (lg <= 5u ? N_COST_BUCKETS - 1u : 20u - lg);
}

enum : int { W_PRIMARY = 0, W_SHADOW_N = 1, W_SEC_N = 2, W_SHADOW_TAKE = 3, W_HIST = 4, W_FILL = W_HIST + (int)N_COST_BUCKETS,
             W_SEC_TAKE = W_FILL + (int)N_COST_BUCKETS, W_WORDS = W_SEC_TAKE + 1 };

struct PipeArgs {
  const vm_frame* frames;      // one per view; nullptr: single view in frame0 / view0
  const ViewDesc* views;
  uint32_t n_views;
  uint32_t total_tiles;        // 8x8 tiles over all views
  const vm_chunk* chunks;      // concatenated per-view chunk lists
  const uint32_t* grids;       // concatenated per-view grids
  const uint4* inners; uint64_t n_inners;
  const uint2* leaves; uint64_t n_leaves;
  const uint32_t* bricks; uint64_t n_bricks;
  uint32_t* dkmax;             // per chunk: best depth key a hit in it can have
  uint32_t* sufmax;            // suffix maximum of dkmax over the view's list
  uint16_t* tile_list;         // per 8x8 tile: culled chunk indices, ascending
  uint32_t* tile_count;        // per 8x8 tile: list length (may exceed list_cap)
  uint16_t* super_list;        // per 32x32 super-tile: chunks its frustum cannot rule out (cap list_cap)
  uint32_t* super_count;       // per super-tile: their number (above list_cap: no list, test all)
  uint32_t total_supers;
  uint32_t list_cap;
  unsigned long long* vis;
  float* shadow;
  unsigned long long* sec_key;
  float* sec_t;
  unsigned long long* refl_key;  // reflect legs of water hits (do_reflect)
  float* refl_t;
  uint32_t* hiz;               // per 8x8 tile: min depth key of the final visibility
  ShadowItem* shadow_q;
  SecItem* sec_q;
  uint32_t* work;              // W_* counters
  uint32_t* item_cost;         // per primary item (2 per tile): SM cycles it took in the last launch
  uint32_t* tile_order;        // per tile: tiles in decreasing order of that cost
  uint32_t* err;
  Traffic64* traffic;          // counting kernels only
  uint32_t do_shadow, do_secondary;
  uint32_t spec;               // VM_SPEC_* pipeline specialisations
  const float* atlas_alpha;    // the tuft quads' atlas alpha (DevWorld), or null
  uint32_t atlas_layers;
  uint32_t tuft_layer[3];
  uint32_t tufts;              // trace tuft cross quads: the chunks hold tufts and atlas_alpha is set
  uint32_t do_reflect;         // with do_secondary: also queue the reflect leg of water hits
                               // (sec_q then holds up to 2 items per pixel)
  vm_frame frame0;
  ViewDesc view0;
};

// launchers of the engine's pass sequence (return cudaError_t of the launch)
cudaError_t launch_tile_select(const vm_frame& f, const vmd::DevWorld& w, const uint32_t* hiz, uint32_t* pairs,
                               uint32_t* counters, cudaStream_t s);
cudaError_t launch_finalize(const vm_frame& f, uint32_t* counters, bool recover, cudaStream_t s);
cudaError_t launch_march_pairs(const vm_frame& f, const vmd::DevWorld& w, const uint32_t* pairs,
                               const uint32_t* counters, unsigned long long* vis, uint32_t* dbg, int sms,
                               cudaStream_t s);
cudaError_t launch_build_hiz(const vm_frame& f, const unsigned long long* vis, uint32_t* hiz, cudaStream_t s);
cudaError_t launch_recover(const vm_frame& f, const vmd::DevWorld& w, uint32_t* pairs, uint32_t* counters,
                           const uint32_t* hiz, int sms, cudaStream_t s);
cudaError_t launch_primary_shadow(const vm_frame& f, const vmd::DevWorld& w, const unsigned long long* vis,
                                  float* out, cudaStream_t s);
// refl_key / refl_t (may be null): the reflect leg of water hits as well
cudaError_t launch_secondary(const vm_frame& f, const vmd::DevWorld& w, const unsigned long long* vis,
                             unsigned long long* sec_key, float* sec_t, unsigned long long* refl_key, float* refl_t,
                             cudaStream_t s);
// water_sec (resolve.wgsl:1468-1535): refract and reflect legs of each
// (1 << shift)^2 block's nearest water pixel, ceil(res / (1 << shift)) cells
cudaError_t launch_water_sec(const vm_frame& f, const vmd::DevWorld& w, const unsigned long long* vis, uint32_t shift,
                             unsigned long long* refr_key, float* refr_t, unsigned long long* refl_key,
                             float* refl_t, cudaStream_t s);
// n blocker distances as binary16 (the engine's R16F shadow target), rounded
// to nearest even; in and out 16-byte / 8-byte aligned
cudaError_t launch_to_r16f(const float* in, uint16_t* out, uint64_t n, int sms, cudaStream_t s);
// shadow_horizontal + shadow_vertical (shadow.wgsl:62-116), fused: the shadow
// mask (clamp(1 - occlusion, 0, 1)) of the frame's blocker distances.
// limit = SHADOW_RADIUS_LIMIT (1..SOFTEN_MAX_LIMIT), penumbra = SOFT_PENUMBRA.
constexpr uint32_t SOFTEN_MAX_LIMIT = 8;
cudaError_t launch_soften(const vm_frame& f, const vmd::DevWorld& w, const unsigned long long* vis, const float* dist,
                          float* mask, uint32_t limit, float penumbra, cudaStream_t s);
// the resolve (resolve.wgsl:1378-1466, all three lanes): RGBA colour of every
// pixel.  mask: the soft shadow mask of this frame, or null (visibility from
// the blocker distances, or from the blocked fractions when soft rays traced
// them).  leg_refr / leg_refl: the water_sec targets (4 halves per
// (2^shift)^2 block; null: every water pixel traces its own legs).
// lane: one byte per pixel, each pixel's lane (sky, opaque, water, glass,
// water with its own legs).  lists: 2 x pixels + 2 words, the compact lists
// of the glass pixels and of the water pixels with their own legs, and their
// counts.  fog: one float4 per pixel, the fog terms of the water and glass
// pixels (sky colour behind, opacity), blended after their lanes.
// light_ao: one float per pixel, the opaque lane's AO between its light stage
// and its shading (null: one kernel does both).  The water lane (legs, then
// the pixels that share them), the glass lane and the water pixels with
// their own legs (the last two over their lists, on sms x 8 resident blocks)
// run on lane_stream[0] / [1] / [2], forked from s at
// lane_event[0] and joined back into s at lane_event[1..3]; s orders
// everything after the call.
cudaError_t launch_resolve(const vm_frame& f, const vmd::DevWorld& w, const vmd::Look& L, const unsigned long long* vis,
                           const float* mask, const float* dist, bool soft_rays, uint32_t water_sec_shift,
                           uint16_t* leg_refr, uint16_t* leg_refl, uint8_t* lane, uint32_t* lists, float* light_ao,
                           float4* fog, float4* out, int sms, cudaStream_t s, const cudaStream_t lane_stream[3],
                           const cudaEvent_t lane_event[4]);
// the heat map of a FLAG_HEATMAP frame (resolve.wgsl:36-44,1389-1394) from
// the iteration counts the engine passes' march summed per pixel
cudaError_t launch_resolve_heat(const vm_frame& f, const uint32_t* dbg, float4* out, cudaStream_t s);
cudaError_t launch_expand(const vm_frame& f, const vmd::DevWorld& w, const unsigned long long* vis,
                          int32_t wx, int32_t wy, int32_t wz, uint32_t dx, uint32_t dy, uint32_t dz,
                          uint32_t* voxel, uint8_t* face, float* t, cudaStream_t s);

// The wavefront frame pipeline (pipeline.cu): chunk bounds -> per-tile cull
// -> primary march (+ queue shadow / secondary rays) -> shadow -> secondary.
struct PipeTuning {
  int primary_warps;     // warps per block of the primary kernel (4, 8)
  int reg_level;         // register budget (resident warps per SM): 0 unconstrained, 1 24, 2 32, 3 20, 4 16
  int ctas_per_sm;       // resident blocks per SM of the persistent primary kernel; 0 = occupancy max
  int px_per_lane;       // pixels per lane (1: 8x4-pixel items, 2: 8x8-pixel items)
};
// ev (optional): five events recorded at the start, after the cull, after the
// primary, shadow and secondary kernels.
cudaError_t launch_pipeline(const PipeArgs& a, const PipeTuning& t, bool underwater, bool count, int sms,
                            cudaStream_t s, const cudaEvent_t* ev = nullptr);
int primary_max_ctas_per_sm(const PipeTuning& t, bool underwater, bool count, bool reflect = false,
                            bool single = true, bool tufts = false);

}  // namespace vmk
