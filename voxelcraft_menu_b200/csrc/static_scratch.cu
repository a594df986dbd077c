// vm_render_static: the frame pipeline with no device allocation at all.
//
// Who needs it: callers that must not call cudaMalloc -- code running inside a
// CUDA stream capture they do not own (allocation is not capturable), engines
// that hand out all device memory from their own fixed arenas and forbid other
// allocations, and allocation-free real-time paths.  They pass every input and
// output buffer; the pipeline's scratch (tile lists, chunk depth bounds, the
// shadow-ray queue, counters) lives in one file-scope __device__ array instead.
//
// Limits and sharing rules:
//  * at most STATIC_MAX_PIXELS pixels and STATIC_MAX_TILES 8x8 tiles per frame
//    (larger frames are rejected with VM_E_TOO_LARGE); 8,650,900 bytes (8.25 MiB)
//    of device memory that every GPU loading this library keeps until the
//    process exits (checked by a static_assert below);
//  * primary and shadow rays only (no secondary rays, no Hi-Z output);
//  * the scratch is shared by every call on a device and keeps the last call's
//    contents; calls whose work overlaps on the GPU (different streams, or
//    other threads) race on it and must be serialised by the caller;
//  * the first call on each device looks the array's address up
//    (cudaGetSymbolAddress): make that first call before any stream capture.
#include <cuda_runtime.h>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "../../include/voxmarch.h"
#include "kernels.cuh"

namespace {

constexpr uint32_t STATIC_MAX_PIXELS = 512u * 512u;
constexpr uint32_t STATIC_MAX_TILES = 8192u;
constexpr uint32_t STATIC_LIST_CAP = 64u;   // chunks per tile kept; longer lists are rescanned

struct StaticScratch {
  uint32_t work[vmk::W_WORDS];
  uint32_t dkmax[VM_MAX_CHUNKS + 1];
  uint32_t sufmax[VM_MAX_CHUNKS + 1];
  uint32_t tile_count[STATIC_MAX_TILES];
  uint32_t item_cost[2 * STATIC_MAX_TILES];
  uint32_t tile_order[STATIC_MAX_TILES];
  uint32_t hiz[STATIC_MAX_TILES];
  uint16_t tile_list[STATIC_MAX_TILES * STATIC_LIST_CAP];
  uint16_t super_list[STATIC_MAX_TILES * STATIC_LIST_CAP];   // super-tiles never outnumber tiles
  uint32_t super_count[STATIC_MAX_TILES];
  vmk::ShadowItem shadow_q[STATIC_MAX_PIXELS];
};
static_assert(sizeof(StaticScratch) == 8650900, "the documented size of the static scratch");

__device__ __align__(256) StaticScratch g_static_scratch;

std::mutex g_mu;
StaticScratch* g_addr[64] = {nullptr};   // device address of g_static_scratch, per device
thread_local char g_err[256];

int fail(int code, const char* msg) {
  snprintf(g_err, sizeof g_err, "%s", msg);
  return code;
}

}  // namespace

extern "C" const char* vm_static_last_error(void) { return g_err; }

extern "C" int vm_render_static(const vm_frame* frame, const vm_chunk* d_chunks, uint32_t n_chunks,
                                const uint32_t* d_grid, uint64_t grid_len, const uint32_t* d_inners,
                                uint64_t n_inners, const uint32_t* d_leaves, uint64_t n_leaves,
                                const uint32_t* d_bricks, uint64_t n_bricks, uint64_t* d_vis, float* d_shadow,
                                uint32_t* d_error, void* stream) {
  g_err[0] = 0;
  if (!frame || !d_chunks || !d_grid || !d_inners || !d_leaves || !d_bricks || !d_vis || !d_shadow || !d_error)
    return fail(VM_E_INVALID, "null argument");
  const vm_frame& f = *frame;
  const uint64_t npix = (uint64_t)f.res[0] * f.res[1];
  const uint64_t tiles = (uint64_t)f.tiles[0] * f.tiles[1];
  if (npix == 0) return fail(VM_E_INVALID, "empty resolution");
  if (f.tiles[0] != (f.res[0] + 7) / 8 || f.tiles[1] != (f.res[1] + 7) / 8)
    return fail(VM_E_INVALID, "tiles do not match the resolution in 8x8 tiles");
  if (npix > STATIC_MAX_PIXELS || tiles > STATIC_MAX_TILES)
    return fail(VM_E_TOO_LARGE, "frame exceeds the static scratch: at most 262144 pixels and 8192 8x8 tiles");
  if (n_chunks > VM_MAX_CHUNKS || f.chunk_count > n_chunks)
    return fail(VM_E_INVALID, "chunk_count must not exceed the chunk list, which must not exceed 8191");
  if (f.camera_chunk != VM_NO_CHUNK && f.camera_chunk >= f.chunk_count)
    return fail(VM_E_INVALID, "camera_chunk outside the visible list");
  if ((uint64_t)f.grid_dim[0] * f.grid_dim[1] * f.grid_dim[2] > grid_len)
    return fail(VM_E_INVALID, "grid_dim product exceeds the grid");
  if (!(f.far_ > 0.0f)) return fail(VM_E_INVALID, "far must be positive");

  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return fail(VM_E_CUDA, "no current CUDA device");
  StaticScratch* s = nullptr;
  {
    std::lock_guard<std::mutex> g(g_mu);
    if (!g_addr[dev]) {
      // set-up, once per device, with that device current
      void* p = nullptr;
      const cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
      if (e != cudaSuccess) return fail(VM_E_CUDA, cudaGetErrorString(e));
      g_addr[dev] = static_cast<StaticScratch*>(p);
    }
    s = g_addr[dev];
  }
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);

  vmk::ViewDesc v;
  memset(&v, 0, sizeof v);
  v.n_chunks = n_chunks;
  v.grid_len = (uint32_t)grid_len;
  v.tiles_x = f.tiles[0];
  v.tiles_y = f.tiles[1];
  vmk::PipeArgs a;
  memset(&a, 0, sizeof a);
  a.frames = nullptr;
  a.views = nullptr;
  a.n_views = 1;
  a.total_tiles = (uint32_t)tiles;
  a.chunks = d_chunks;
  a.grids = d_grid;
  a.inners = reinterpret_cast<const uint4*>(d_inners); a.n_inners = n_inners;
  a.leaves = reinterpret_cast<const uint2*>(d_leaves); a.n_leaves = n_leaves;
  a.bricks = d_bricks; a.n_bricks = n_bricks;
  a.dkmax = s->dkmax;
  a.sufmax = s->sufmax;
  a.tile_list = s->tile_list;
  a.tile_count = s->tile_count;
  a.super_list = s->super_list;
  a.super_count = s->super_count;
  a.total_supers = ((f.tiles[0] + 3) / 4) * ((f.tiles[1] + 3) / 4);
  a.item_cost = s->item_cost;
  a.tile_order = s->tile_order;
  a.list_cap = STATIC_LIST_CAP;
  a.vis = reinterpret_cast<unsigned long long*>(d_vis);
  a.shadow = d_shadow;
  a.hiz = s->hiz;
  a.shadow_q = s->shadow_q;
  a.work = s->work;
  a.err = d_error;
  a.do_shadow = 1;
  a.spec = VM_SPEC_DEFAULT;
  a.do_secondary = 0;
  a.frame0 = f;
  a.view0 = v;
  const vmk::PipeTuning t{4, 1, 0, 1};
  const cudaError_t e = vmk::launch_pipeline(a, t, (f.flags & VM_FLAG_UNDERWATER) != 0u, false, sms,
                                             static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) return fail(VM_E_CUDA, cudaGetErrorString(e));
  return VM_OK;
}
