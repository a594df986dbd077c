// Kernel declarations and launch helpers shared by the ABI layer.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "vm_types.h"
#include "march_device.cuh"

namespace vmk {

// One view of a (possibly batched) fused launch.
struct ViewDesc {
  uint32_t chunk_off;     // first chunk of this view in the concatenated chunk list
  uint32_t n_chunks;      // chunks of this view (visible + shadow-only)
  uint64_t grid_off;      // first grid cell of this view
  uint32_t grid_len;
  uint32_t tile_begin;    // first work item (fused tile) of this view
  uint32_t tiles_x, tiles_y;   // fused tiles of this view
  uint64_t pix_off;       // first pixel of this view in the output buffers
  uint32_t hiz_off;       // first 8x8 tile of this view in the hiz buffer
  uint32_t pad;
};

struct Traffic64 {
  unsigned long long chunk, l1, leaf, attr, pal, grid, iters, rays_primary, rays_shadow, rays_secondary;
};

struct FusedArgs {
  const vm_frame* frames;      // one per view
  const ViewDesc* views;
  uint32_t n_views;
  uint32_t total_tiles;
  const vm_chunk* chunks;      // concatenated per-view chunk lists
  const uint32_t* grids;       // concatenated per-view grids
  const uint4* inners; uint64_t n_inners;
  const uint2* leaves; uint64_t n_leaves;
  const uint32_t* bricks; uint64_t n_bricks;
  const uint32_t* dkmax;       // per chunk (concatenated like chunks)
  const uint32_t* sufmax;
  unsigned long long* vis;
  float* shadow;
  unsigned long long* sec_key;
  float* sec_t;
  uint32_t* hiz;
  uint32_t* work;              // work[0] = next tile counter (zeroed before launch)
  uint32_t* err;
  Traffic64* traffic;          // only with counting kernels
  uint32_t do_shadow, do_secondary;
  // single-view launches carry their frame and view in the parameter space
  // (frames == nullptr), so no host->device copy is needed per frame
  vm_frame frame0;
  ViewDesc view0;
};

enum FusedVariant : int { FUSED_8x8 = 0, FUSED_16x8 = 1, FUSED_16x16 = 2, FUSED_32x16 = 3, FUSED_VARIANTS = 4 };
inline void fused_dims(int v, uint32_t* tw, uint32_t* th) {
  static const uint32_t W[] = {8, 16, 16, 32}, H[] = {8, 8, 16, 16};
  *tw = W[v]; *th = H[v];
}

// launchers (return cudaError_t of the launch)
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
cudaError_t launch_secondary(const vm_frame& f, const vmd::DevWorld& w, const unsigned long long* vis,
                             unsigned long long* sec_key, float* sec_t, cudaStream_t s);
cudaError_t launch_expand(const vm_frame& f, const vmd::DevWorld& w, const unsigned long long* vis,
                          int32_t wx, int32_t wy, int32_t wz, uint32_t dx, uint32_t dy, uint32_t dz,
                          uint32_t* voxel, uint8_t* face, float* t, cudaStream_t s);
// frames == nullptr: one view given by value (f0, v0)
cudaError_t launch_chunk_bounds(const vm_frame* frames, const ViewDesc* views, uint32_t n_views,
                                const vm_frame& f0, const ViewDesc& v0, const vm_chunk* chunks, uint32_t* dkmax,
                                uint32_t* sufmax, cudaStream_t s);
// underwater: the frame's FLAG_UNDERWATER (uniform over a launch; every view of
// a batched launch must agree).  count: traffic-counting instantiation.
cudaError_t launch_fused(const FusedArgs& a, int variant, bool underwater, bool count, uint32_t grid_ctas,
                         cudaStream_t s);
int fused_max_ctas_per_sm(int variant, bool underwater, bool count);

}  // namespace vmk
