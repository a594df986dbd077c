// The C ABI of include/voxmarch.h: one context = one renderer's device state.
#include <cuda_runtime.h>
#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/voxmarch.h"
#include "kernels.cuh"
#include "resolve.cuh"

using vmk::ViewDesc;

namespace {

struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
};

}  // namespace

struct vm_ctx {
  int device = 0;
  int sms = 148;
  cudaStream_t own = nullptr, stream = nullptr;
  cudaEvent_t rendered = nullptr;   // recorded after each vm_render's kernels (vm_wait_render)
  bool have_rendered = false;
  vm_caps caps{};
  // world pools
  DevBuf inners, leaves, bricks;
  uint64_t n_inners = 0, n_leaves = 0, n_bricks = 0;
  bool have_world = false;
  // per-frame inputs
  DevBuf chunks, grid;
  uint32_t n_chunks = 0;
  uint64_t grid_len = 0;
  bool have_chunks = false;
  vm_frame frame{};
  bool have_frame = false;
  // per-frame outputs and scratch
  DevBuf vis, shadow, sec_key, sec_t, hiz, dbg, pairs, counters, err, work, dkmax, sufmax, traffic, expand;
  DevBuf shadow_mask;   // vm_soften_shadows output, sized on first use
  bool mask_valid = false;   // the mask belongs to the last rendered frame
  // the resolve's material inputs and output (vm_upload_atlas ... vm_resolve)
  DevBuf atlas, faces, probes, shaft, grad, color, leg_refr, leg_refl, light_ao, lane, lane_lists, fog;
  uint32_t atlas_layers = 0, n_faces = 0;
  DevBuf atlas_alpha;          // the atlas's alpha channel for the tuft quads of the march
  uint32_t tuft_layer[3] = {0, 0, 0};
  bool chunks_foliage = false;   // a chunk of the uploaded list holds tufts (VM_ATTR_HAS_FOLIAGE)
  bool batch_foliage = false;    // the same for the batch's chunk lists
  bool have_probes = false, have_shaft = false, color_done = false;
  bool heat_valid = false;   // dbg holds the iteration counts of this frame's vm_select / vm_march
  // the resolve's water and glass lanes run beside the sky / opaque lanes:
  // three streams forked from the context's stream and joined back by events
  cudaStream_t lane_stream[3] = {nullptr, nullptr, nullptr};
  cudaEvent_t lane_event[4] = {nullptr, nullptr, nullptr, nullptr};
  DevBuf shadow16;      // vm_read_async_r16f staging, sized on first use
  DevBuf refl_key, refl_t;   // reflect legs of water hits, sized by the first FLAG_WATER_REFLECT frame
  DevBuf ws_refr_key, ws_refr_t, ws_refl_key, ws_refl_t;   // vm_water_sec cells, sized by its first call
  uint32_t ws_shift = 0, ws_cells = 0;
  bool ws_done = false;
  bool refl_frame = false;   // the last frame traced them
  DevBuf tile_list, tile_count, shadow_q, sec_q, item_cost, tile_order, super_list, super_count;
  // batch
  DevBuf b_frames, b_views, b_views1, b_chunks, b_grids, b_vis, b_shadow, b_seck, b_sect, b_hiz, b_dkmax, b_sufmax;
  DevBuf b_tile_list, b_tile_count, b_shadow_q, b_sec_q, b_item_cost, b_tile_order, b_super_list, b_super_count;
  std::vector<vm_frame> bh_frames;
  std::vector<ViewDesc> bh_views;
  uint32_t b_n_views = 0, b_total_tiles = 0, b_n_chunks = 0, b_list_cap = 1, b_total_supers = 0;
  uint64_t b_pixels = 0, b_grid_total = 0;
  bool b_underwater = false;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t graph_exec = nullptr;
  bool graph_secondary = false;   // the cached graph also traces the secondary rays
  // tuning of the primary kernel
  vmk::PipeTuning tuning{4, 0, 0, 1};
  uint32_t spec = VM_SPEC_DEFAULT;   // VM_SPEC_* pipeline specialisations
  std::string err_text;
};

namespace {

int fail(vm_ctx* c, int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  if (c) c->err_text = buf;
  return code;
}

int cuda_fail(vm_ctx* c, cudaError_t e, const char* what) {
  return fail(c, VM_E_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

#define CK(call)                                         \
  do {                                                   \
    cudaError_t e_ = (call);                             \
    if (e_ != cudaSuccess) return cuda_fail(ctx, e_, #call); \
  } while (0)

// grow a device buffer; keep_bytes of the old contents are copied over
int ensure(vm_ctx* ctx, DevBuf& b, size_t bytes, size_t keep_bytes = 0) {
  if (bytes <= b.bytes && b.p) return VM_OK;
  size_t cap = std::max<size_t>(bytes, 256);
  if (b.bytes) cap = std::max(cap, b.bytes + b.bytes / 2);
  void* p = nullptr;
  cudaError_t e = cudaMalloc(&p, cap);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaMalloc");
  if (b.p) {
    if (keep_bytes) {
      e = cudaMemcpyAsync(p, b.p, std::min(keep_bytes, b.bytes), cudaMemcpyDeviceToDevice, ctx->stream);
      if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaMemcpyAsync");
    }
    cudaStreamSynchronize(ctx->stream);
    cudaFree(b.p);
  }
  b.p = p;
  b.bytes = cap;
  return VM_OK;
}

void release(DevBuf& b) {
  if (b.p) cudaFree(b.p);
  b.p = nullptr;
  b.bytes = 0;
}

void drop_graph(vm_ctx* ctx) {
  if (ctx->graph_exec) cudaGraphExecDestroy(ctx->graph_exec);
  if (ctx->graph) cudaGraphDestroy(ctx->graph);
  ctx->graph_exec = nullptr;
  ctx->graph = nullptr;
}

vmd::DevWorld dev_world(vm_ctx* ctx) {
  vmd::DevWorld w;
  w.chunks = (const vm_chunk*)ctx->chunks.p; w.n_chunks = ctx->n_chunks;
  w.inners = (const uint4*)ctx->inners.p; w.n_inners = ctx->n_inners;
  w.leaves = (const uint2*)ctx->leaves.p; w.n_leaves = ctx->n_leaves;
  w.bricks = (const uint32_t*)ctx->bricks.p; w.n_bricks = ctx->n_bricks;
  w.grid = (const uint32_t*)ctx->grid.p; w.n_grid = ctx->grid_len;
  w.err = (uint32_t*)ctx->err.p;
  w.spec = ctx->spec;
  const bool tufts = ctx->atlas_layers && ctx->n_faces;   // the march reads the atlas once both are in
  w.atlas_alpha = tufts ? (const float*)ctx->atlas_alpha.p : nullptr;
  w.atlas_layers = ctx->atlas_layers;
  for (int i = 0; i < 3; ++i) w.tuft_layer[i] = ctx->tuft_layer[i];
  return w;
}

// Checks shared by every frame entry point.
int check_frame(vm_ctx* ctx, const vm_frame& f, uint32_t n_chunks, uint64_t grid_len) {
  if (f.res[0] == 0 || f.res[1] == 0) return fail(ctx, VM_E_INVALID, "empty resolution");
  if (f.tiles[0] != (f.res[0] + 7) / 8 || f.tiles[1] != (f.res[1] + 7) / 8)
    return fail(ctx, VM_E_INVALID, "tiles (%u,%u) do not match res (%u,%u) in 8x8 tiles", f.tiles[0], f.tiles[1],
                f.res[0], f.res[1]);
  if ((uint64_t)f.tiles[0] * f.tiles[1] > VM_MAX_TILES)
    return fail(ctx, VM_E_TILE_OVERFLOW, "tile index overflows the pair word: %u x %u tiles > %u", f.tiles[0],
                f.tiles[1], VM_MAX_TILES);
  if (f.chunk_count > n_chunks) return fail(ctx, VM_E_INVALID, "chunk_count %u > uploaded chunks %u", f.chunk_count, n_chunks);
  if (n_chunks > VM_MAX_CHUNKS) return fail(ctx, VM_E_INVALID, "%u chunks exceed the 13-bit chunk field", n_chunks);
  if (f.camera_chunk != VM_NO_CHUNK && f.camera_chunk >= f.chunk_count)
    return fail(ctx, VM_E_INVALID, "camera_chunk %u outside the visible list", f.camera_chunk);
  if ((uint64_t)f.grid_dim[0] * f.grid_dim[1] * f.grid_dim[2] > grid_len)
    return fail(ctx, VM_E_INVALID, "grid_dim product exceeds the uploaded grid");
  if (!(f.far_ > 0.0f)) return fail(ctx, VM_E_INVALID, "far must be positive");
  if (f.max_pairs == 0 || f.max_pairs > 0x7FFFFFFFu) return fail(ctx, VM_E_INVALID, "max_pairs out of range");
  return VM_OK;
}

int check_ready(vm_ctx* ctx) {
  if (!ctx->have_world) return fail(ctx, VM_E_NOT_READY, "no world uploaded");
  if (!ctx->have_chunks) return fail(ctx, VM_E_NOT_READY, "no chunk list uploaded");
  if (!ctx->have_frame) return fail(ctx, VM_E_NOT_READY, "no frame set");
  const vm_frame& f = ctx->frame;
  if (f.res[0] > ctx->caps.max_width || f.res[1] > ctx->caps.max_height)
    return fail(ctx, VM_E_INVALID, "frame %ux%u exceeds the context's %ux%u", f.res[0], f.res[1], ctx->caps.max_width,
                ctx->caps.max_height);
  return check_frame(ctx, f, ctx->n_chunks, ctx->grid_len);
}

constexpr uint32_t LIST_CAP_MAX = 256;   // chunks stored per 8x8 tile before the march rescans

vmk::PipeArgs base_args(vm_ctx* ctx) {
  vmk::PipeArgs a;
  memset(&a, 0, sizeof a);
  a.inners = (const uint4*)ctx->inners.p; a.n_inners = ctx->n_inners;
  a.leaves = (const uint2*)ctx->leaves.p; a.n_leaves = ctx->n_leaves;
  a.bricks = (const uint32_t*)ctx->bricks.p; a.n_bricks = ctx->n_bricks;
  a.err = (uint32_t*)ctx->err.p;
  a.work = (uint32_t*)ctx->work.p;
  a.item_cost = (uint32_t*)ctx->item_cost.p;
  a.tile_order = (uint32_t*)ctx->tile_order.p;
  a.traffic = (vmk::Traffic64*)ctx->traffic.p;
  a.do_shadow = 1;
  a.spec = ctx->spec;
  const bool tufts = ctx->atlas_layers && ctx->n_faces;
  a.atlas_alpha = tufts ? (const float*)ctx->atlas_alpha.p : nullptr;
  a.atlas_layers = ctx->atlas_layers;
  for (int i = 0; i < 3; ++i) a.tuft_layer[i] = ctx->tuft_layer[i];
  // the tuft kernels: the single view's chunks (the batch paths set their own)
  a.tufts = tufts && (ctx->spec & VM_SPEC_FOLIAGE) != 0u && ctx->chunks_foliage ? 1u : 0u;
  a.do_secondary = 1;
  return a;
}

// Buffers of the reflect legs when the frame asks for them
// (FLAG_WATER_REFLECT): one key + t per pixel, and a secondary queue of two
// items per pixel (a water hit queues its refract and its reflect leg).
// Allocated by the first such frame and kept.
int prepare_reflect(vm_ctx* ctx) {
  const vm_frame& f = ctx->frame;
  ctx->refl_frame = (f.flags & VM_FLAG_WATER_REFLECT) != 0u;
  if (!ctx->refl_frame) return VM_OK;
  const size_t npix = (size_t)f.res[0] * f.res[1];
  int rc;
  if ((rc = ensure(ctx, ctx->refl_key, npix * 8))) return rc;
  if ((rc = ensure(ctx, ctx->refl_t, npix * 4))) return rc;
  return ensure(ctx, ctx->sec_q, 2 * npix * sizeof(vmk::SecItem));
}

// The single-view pipeline (frame and view descriptor by value).
int enqueue_render(vm_ctx* ctx, bool count, const cudaEvent_t* ev = nullptr) {
  ctx->mask_valid = false;
  ctx->color_done = false;
  ctx->heat_valid = false;
  const vm_frame& f = ctx->frame;
  // buffers are grown before any of their pointers is taken below
  int rc;
  if ((rc = prepare_reflect(ctx))) return rc;
  ViewDesc v;
  memset(&v, 0, sizeof v);
  v.n_chunks = ctx->n_chunks;
  v.grid_len = (uint32_t)ctx->grid_len;
  v.tiles_x = f.tiles[0];
  v.tiles_y = f.tiles[1];
  vmk::PipeArgs a = base_args(ctx);
  a.frames = nullptr;
  a.views = nullptr;
  a.n_views = 1;
  a.total_tiles = v.tiles_x * v.tiles_y;
  a.chunks = (const vm_chunk*)ctx->chunks.p;
  a.grids = (const uint32_t*)ctx->grid.p;
  a.dkmax = (uint32_t*)ctx->dkmax.p;
  a.sufmax = (uint32_t*)ctx->sufmax.p;
  a.tile_list = (uint16_t*)ctx->tile_list.p;
  a.tile_count = (uint32_t*)ctx->tile_count.p;
  a.super_list = (uint16_t*)ctx->super_list.p;
  a.super_count = (uint32_t*)ctx->super_count.p;
  a.total_supers = ((v.tiles_x + 3) / 4) * ((v.tiles_y + 3) / 4);
  a.list_cap = std::max(1u, std::min(f.chunk_count, LIST_CAP_MAX));
  a.vis = (unsigned long long*)ctx->vis.p;
  a.shadow = (float*)ctx->shadow.p;
  a.sec_key = (unsigned long long*)ctx->sec_key.p;
  a.sec_t = (float*)ctx->sec_t.p;
  a.hiz = (uint32_t*)ctx->hiz.p;
  a.shadow_q = (vmk::ShadowItem*)ctx->shadow_q.p;
  a.sec_q = (vmk::SecItem*)ctx->sec_q.p;
  a.frame0 = f;
  a.view0 = v;
  if (ctx->refl_frame) {
    a.refl_key = (unsigned long long*)ctx->refl_key.p;
    a.refl_t = (float*)ctx->refl_t.p;
    a.do_reflect = 1;
  }
  const bool uw = (f.flags & VM_FLAG_UNDERWATER) != 0u;
  CK(vmk::launch_pipeline(a, ctx->tuning, uw, count, ctx->sms, ctx->stream, ev));
  return VM_OK;
}

}  // namespace

extern "C" {

int vm_create(int device_ordinal, const vm_caps* caps, vm_ctx** out) {
  if (!out || !caps) return VM_E_INVALID;
  *out = nullptr;
  if (caps->max_width == 0 || caps->max_height == 0) return VM_E_INVALID;
  vm_ctx* ctx = new vm_ctx();
  ctx->device = device_ordinal;
  ctx->caps = *caps;
  if (ctx->caps.max_chunks == 0) ctx->caps.max_chunks = VM_MAX_CHUNKS;
  cudaError_t e = cudaSetDevice(device_ordinal);
  if (e != cudaSuccess) { delete ctx; return VM_E_CUDA; }
  cudaDeviceGetAttribute(&ctx->sms, cudaDevAttrMultiProcessorCount, device_ordinal);
  e = cudaStreamCreateWithFlags(&ctx->own, cudaStreamNonBlocking);
  if (e != cudaSuccess) { delete ctx; return VM_E_CUDA; }
  ctx->stream = ctx->own;
  const uint64_t npix = (uint64_t)caps->max_width * caps->max_height;
  const uint64_t tiles = (uint64_t)((caps->max_width + 7) / 8) * ((caps->max_height + 7) / 8);
  int rc = VM_OK;
  rc |= ensure(ctx, ctx->vis, npix * 8);
  rc |= ensure(ctx, ctx->shadow, npix * 4);
  rc |= ensure(ctx, ctx->sec_key, npix * 8);
  rc |= ensure(ctx, ctx->sec_t, npix * 4);
  rc |= ensure(ctx, ctx->dbg, npix * 4);
  rc |= ensure(ctx, ctx->expand, npix * 9);
  rc |= ensure(ctx, ctx->hiz, tiles * 4);
  rc |= ensure(ctx, ctx->counters, 64);
  rc |= ensure(ctx, ctx->err, 64);
  rc |= ensure(ctx, ctx->work, vmk::W_WORDS * sizeof(uint32_t));
  rc |= ensure(ctx, ctx->item_cost, tiles * 8);
  rc |= ensure(ctx, ctx->tile_order, tiles * 4);
  rc |= ensure(ctx, ctx->traffic, 3 * sizeof(vmk::Traffic64));
  rc |= ensure(ctx, ctx->dkmax, (size_t)ctx->caps.max_chunks * 4);
  rc |= ensure(ctx, ctx->sufmax, (size_t)ctx->caps.max_chunks * 4);
  rc |= ensure(ctx, ctx->tile_list, tiles * LIST_CAP_MAX * 2);
  rc |= ensure(ctx, ctx->tile_count, tiles * 4);
  const uint64_t supers = (uint64_t)((caps->max_width + 31) / 32) * ((caps->max_height + 31) / 32);
  rc |= ensure(ctx, ctx->super_list, supers * LIST_CAP_MAX * 2);
  rc |= ensure(ctx, ctx->super_count, supers * 4);
  rc |= ensure(ctx, ctx->shadow_q, npix * sizeof(vmk::ShadowItem));
  rc |= ensure(ctx, ctx->sec_q, npix * sizeof(vmk::SecItem));
  if (rc != VM_OK) { vm_destroy(ctx); return VM_E_CUDA; }
  cudaMemsetAsync(ctx->hiz.p, 0, tiles * 4, ctx->stream);
  cudaMemsetAsync(ctx->item_cost.p, 0, tiles * 8, ctx->stream);
  cudaMemsetAsync(ctx->err.p, 0, 64, ctx->stream);
  cudaMemsetAsync(ctx->counters.p, 0, 64, ctx->stream);
  cudaStreamSynchronize(ctx->stream);
  *out = ctx;
  return VM_OK;
}

void vm_destroy(vm_ctx* ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  drop_graph(ctx);
  DevBuf* all[] = {&ctx->inners, &ctx->leaves, &ctx->bricks, &ctx->chunks, &ctx->grid, &ctx->vis, &ctx->shadow,
                   &ctx->sec_key, &ctx->sec_t, &ctx->hiz, &ctx->dbg, &ctx->pairs, &ctx->counters, &ctx->err,
                   &ctx->work, &ctx->dkmax, &ctx->sufmax, &ctx->traffic, &ctx->expand, &ctx->b_frames,
                   &ctx->b_views, &ctx->b_views1, &ctx->b_chunks, &ctx->b_grids, &ctx->b_vis, &ctx->b_shadow,
                   &ctx->b_seck, &ctx->b_sect, &ctx->b_hiz, &ctx->b_dkmax, &ctx->b_sufmax, &ctx->tile_list,
                   &ctx->tile_count, &ctx->shadow_q, &ctx->sec_q, &ctx->b_tile_list, &ctx->b_tile_count,
                   &ctx->b_shadow_q, &ctx->b_sec_q, &ctx->item_cost, &ctx->tile_order, &ctx->b_item_cost,
                   &ctx->b_tile_order, &ctx->super_list, &ctx->super_count, &ctx->b_super_list,
                   &ctx->b_super_count, &ctx->shadow_mask, &ctx->refl_key, &ctx->refl_t,
                   &ctx->shadow16, &ctx->ws_refr_key, &ctx->ws_refr_t, &ctx->ws_refl_key, &ctx->ws_refl_t,
                   &ctx->atlas, &ctx->faces, &ctx->probes, &ctx->shaft, &ctx->grad, &ctx->color,
                   &ctx->atlas_alpha, &ctx->leg_refr, &ctx->leg_refl, &ctx->light_ao, &ctx->lane,
                   &ctx->lane_lists, &ctx->fog};
  for (DevBuf* b : all) release(*b);
  if (ctx->rendered) cudaEventDestroy(ctx->rendered);
  for (cudaEvent_t e : ctx->lane_event)
    if (e) cudaEventDestroy(e);
  for (cudaStream_t ls : ctx->lane_stream)
    if (ls) cudaStreamDestroy(ls);
  if (ctx->own) cudaStreamDestroy(ctx->own);
  delete ctx;
}

const char* vm_last_error(const vm_ctx* ctx) { return ctx ? ctx->err_text.c_str() : "null context"; }

int vm_set_stream(vm_ctx* ctx, void* s) {
  if (!ctx) return VM_E_INVALID;
  ctx->stream = s ? (cudaStream_t)s : ctx->own;
  drop_graph(ctx);
  return VM_OK;
}

int vm_upload_world(vm_ctx* ctx, const uint32_t* inners, uint64_t n_inners, const uint32_t* leaves, uint64_t n_leaves,
                    const uint32_t* bricks, uint64_t n_bricks) {
  if (!ctx) return VM_E_INVALID;
  if ((n_inners && !inners) || (n_leaves && !leaves) || (n_bricks && !bricks))
    return fail(ctx, VM_E_INVALID, "null pool with nonzero size");
  CK(cudaSetDevice(ctx->device));
  int rc;
  if ((rc = ensure(ctx, ctx->inners, std::max<uint64_t>(n_inners, 1) * 16))) return rc;
  if ((rc = ensure(ctx, ctx->leaves, std::max<uint64_t>(n_leaves, 1) * 8))) return rc;
  if ((rc = ensure(ctx, ctx->bricks, std::max<uint64_t>(n_bricks, 1) * 4))) return rc;
  if (n_inners) CK(cudaMemcpyAsync(ctx->inners.p, inners, n_inners * 16, cudaMemcpyHostToDevice, ctx->stream));
  if (n_leaves) CK(cudaMemcpyAsync(ctx->leaves.p, leaves, n_leaves * 8, cudaMemcpyHostToDevice, ctx->stream));
  if (n_bricks) CK(cudaMemcpyAsync(ctx->bricks.p, bricks, n_bricks * 4, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  ctx->n_inners = n_inners;
  ctx->n_leaves = n_leaves;
  ctx->n_bricks = n_bricks;
  ctx->have_world = true;
  drop_graph(ctx);
  return VM_OK;
}

int vm_update_pool(vm_ctx* ctx, int pool, uint64_t offset, const uint32_t* data, uint64_t count) {
  if (!ctx || !data || pool < 0 || pool > 2) return VM_E_INVALID;
  CK(cudaSetDevice(ctx->device));
  DevBuf* b = pool == 0 ? &ctx->inners : pool == 1 ? &ctx->leaves : &ctx->bricks;
  uint64_t* n = pool == 0 ? &ctx->n_inners : pool == 1 ? &ctx->n_leaves : &ctx->n_bricks;
  const size_t esz = pool == 0 ? 16 : pool == 1 ? 8 : 4;
  const uint64_t end = offset + count;
  int rc;
  if ((rc = ensure(ctx, *b, end * esz, *n * esz))) return rc;
  CK(cudaMemcpyAsync((char*)b->p + offset * esz, data, count * esz, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  *n = std::max(*n, end);
  ctx->have_world = true;
  drop_graph(ctx);
  return VM_OK;
}

int vm_upload_chunks(vm_ctx* ctx, const vm_chunk* chunks, uint32_t n_chunks, const uint32_t* grid, uint64_t grid_len) {
  if (!ctx || (n_chunks && !chunks) || !grid || grid_len == 0) return VM_E_INVALID;
  if (n_chunks > ctx->caps.max_chunks || n_chunks > VM_MAX_CHUNKS)
    return fail(ctx, VM_E_INVALID, "%u chunks exceed the context capacity %u", n_chunks, ctx->caps.max_chunks);
  CK(cudaSetDevice(ctx->device));
  int rc;
  if ((rc = ensure(ctx, ctx->chunks, std::max<uint32_t>(n_chunks, 1) * sizeof(vm_chunk)))) return rc;
  if ((rc = ensure(ctx, ctx->grid, grid_len * 4))) return rc;
  if (n_chunks) CK(cudaMemcpyAsync(ctx->chunks.p, chunks, (size_t)n_chunks * sizeof(vm_chunk), cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(ctx->grid.p, grid, grid_len * 4, cudaMemcpyHostToDevice, ctx->stream));
  ctx->n_chunks = n_chunks;
  ctx->grid_len = grid_len;
  ctx->have_chunks = true;
  ctx->chunks_foliage = false;
  for (uint32_t i = 0; i < n_chunks && !ctx->chunks_foliage; ++i)
    ctx->chunks_foliage = (chunks[i].attr_flags & VM_ATTR_HAS_FOLIAGE) != 0u;
  return VM_OK;
}

int vm_set_frame(vm_ctx* ctx, const vm_frame* frame) {
  if (!ctx || !frame) return VM_E_INVALID;
  ctx->frame = *frame;
  ctx->have_frame = true;
  ctx->heat_valid = false;
  return VM_OK;
}

int vm_set_tuning(vm_ctx* ctx, int warps_per_block, int reg_level, int ctas_per_sm) {
  if (!ctx) return VM_E_INVALID;
  if (!(warps_per_block == 4 || warps_per_block == 8) || reg_level < 0 || reg_level > 4 || ctas_per_sm < 0)
    return fail(ctx, VM_E_INVALID, "warps per block must be 4 or 8, register level 0..4, CTAs per SM >= 0");
  if (warps_per_block != ctx->tuning.primary_warps || reg_level != ctx->tuning.reg_level ||
      ctas_per_sm != ctx->tuning.ctas_per_sm)
    drop_graph(ctx);
  ctx->tuning.primary_warps = warps_per_block;
  ctx->tuning.reg_level = reg_level;
  ctx->tuning.ctas_per_sm = ctas_per_sm;
  return VM_OK;
}

int vm_set_spec(vm_ctx* ctx, uint32_t spec) {
  if (!ctx) return VM_E_INVALID;
  const uint32_t known = VM_SPEC_ALL | VM_SPEC_SOFT_RAYS | VM_SPEC_WIND_SWAY;
  if ((spec & ~known) != 0u) return fail(ctx, VM_E_INVALID, "unknown VM_SPEC bits 0x%x", spec & ~known);
  if (spec != ctx->spec) drop_graph(ctx);
  ctx->spec = spec;
  return VM_OK;
}

int vm_set_packet(vm_ctx* ctx, int pixels_per_lane) {
  if (!ctx) return VM_E_INVALID;
  if (pixels_per_lane != 1 && pixels_per_lane != 2)
    return fail(ctx, VM_E_INVALID, "pixels per lane must be 1 (8x4-pixel items) or 2 (8x8-pixel items)");
  if (pixels_per_lane != ctx->tuning.px_per_lane) drop_graph(ctx);
  ctx->tuning.px_per_lane = pixels_per_lane;
  return VM_OK;
}

int vm_select(vm_ctx* ctx) {
  if (!ctx) return VM_E_INVALID;
  int rc = check_ready(ctx);
  if (rc) return rc;
  CK(cudaSetDevice(ctx->device));
  const vm_frame& f = ctx->frame;
  const uint64_t npix = (uint64_t)f.res[0] * f.res[1];
  const uint64_t tiles = (uint64_t)f.tiles[0] * f.tiles[1];
  if ((rc = ensure(ctx, ctx->pairs, (size_t)f.max_pairs * 2 * 4))) return rc;
  CK(cudaMemsetAsync(ctx->vis.p, 0, npix * 8, ctx->stream));
  CK(cudaMemsetAsync(ctx->counters.p, 0, 32, ctx->stream));
  ctx->heat_valid = false;
  if (f.flags & VM_FLAG_HEATMAP) CK(cudaMemsetAsync(ctx->dbg.p, 0, npix * 4, ctx->stream));
  if (!(f.flags & VM_FLAG_HIZ)) CK(cudaMemsetAsync(ctx->hiz.p, 0, tiles * 4, ctx->stream));
  const vmd::DevWorld w = dev_world(ctx);
  CK(vmk::launch_tile_select(f, w, (const uint32_t*)ctx->hiz.p, (uint32_t*)ctx->pairs.p, (uint32_t*)ctx->counters.p,
                             ctx->stream));
  CK(vmk::launch_finalize(f, (uint32_t*)ctx->counters.p, false, ctx->stream));
  return VM_OK;
}

int vm_march(vm_ctx* ctx) {
  if (!ctx) return VM_E_INVALID;
  int rc = check_ready(ctx);
  if (rc) return rc;
  if (!ctx->pairs.p) return fail(ctx, VM_E_NOT_READY, "vm_march before vm_select");
  CK(cudaSetDevice(ctx->device));
  const vm_frame& f = ctx->frame;
  const vmd::DevWorld w = dev_world(ctx);
  uint32_t* pairs = (uint32_t*)ctx->pairs.p;
  uint32_t* ctr = (uint32_t*)ctx->counters.p;
  unsigned long long* vis = (unsigned long long*)ctx->vis.p;
  uint32_t* dbg = (f.flags & VM_FLAG_HEATMAP) ? (uint32_t*)ctx->dbg.p : nullptr;
  CK(vmk::launch_march_pairs(f, w, pairs, ctr, vis, dbg, ctx->sms, ctx->stream));
  if (f.flags & VM_FLAG_HIZ) {
    CK(vmk::launch_build_hiz(f, vis, (uint32_t*)ctx->hiz.p, ctx->stream));
    CK(vmk::launch_recover(f, w, pairs, ctr, (const uint32_t*)ctx->hiz.p, ctx->sms, ctx->stream));
    CK(vmk::launch_finalize(f, ctr, true, ctx->stream));
    CK(vmk::launch_march_pairs(f, w, pairs, ctr, vis, dbg, ctx->sms, ctx->stream));
  }
  ctx->heat_valid = dbg != nullptr;
  return VM_OK;
}

int vm_primary_shadow(vm_ctx* ctx) {
  if (ctx) {
    ctx->mask_valid = false;
    ctx->color_done = false;
  }
  if (!ctx) return VM_E_INVALID;
  int rc = check_ready(ctx);
  if (rc) return rc;
  CK(cudaSetDevice(ctx->device));
  CK(vmk::launch_primary_shadow(ctx->frame, dev_world(ctx), (const unsigned long long*)ctx->vis.p, (float*)ctx->shadow.p,
                                ctx->stream));
  return VM_OK;
}

int vm_soften_shadows(vm_ctx* ctx, uint32_t radius_limit, float penumbra) {
  if (!ctx) return VM_E_INVALID;
  int rc = check_ready(ctx);
  if (rc) return rc;
  if (radius_limit < 1u || radius_limit > vmk::SOFTEN_MAX_LIMIT)
    return fail(ctx, VM_E_INVALID, "radius limit %u outside 1..%u", radius_limit, vmk::SOFTEN_MAX_LIMIT);
  if (!(penumbra > 0.0f) || !(penumbra < 1e30f))
    return fail(ctx, VM_E_INVALID, "penumbra must be positive and finite");
  if (ctx->spec & VM_SPEC_SOFT_RAYS)
    return fail(ctx, VM_E_INVALID, "the filter reads blocker distances; this frame's shadow buffer holds the "
                                   "blocked fractions of jittered rays");
  CK(cudaSetDevice(ctx->device));
  const vm_frame& f = ctx->frame;
  if ((rc = ensure(ctx, ctx->shadow_mask, (size_t)f.res[0] * f.res[1] * 4))) return rc;
  CK(vmk::launch_soften(f, dev_world(ctx), (const unsigned long long*)ctx->vis.p, (const float*)ctx->shadow.p,
                        (float*)ctx->shadow_mask.p, radius_limit, penumbra, ctx->stream));
  ctx->mask_valid = true;
  return VM_OK;
}

int vm_secondary(vm_ctx* ctx) {
  if (!ctx) return VM_E_INVALID;
  int rc = check_ready(ctx);
  if (rc) return rc;
  CK(cudaSetDevice(ctx->device));
  if ((rc = prepare_reflect(ctx))) return rc;
  CK(vmk::launch_secondary(ctx->frame, dev_world(ctx), (const unsigned long long*)ctx->vis.p,
                           (unsigned long long*)ctx->sec_key.p, (float*)ctx->sec_t.p,
                           ctx->refl_frame ? (unsigned long long*)ctx->refl_key.p : nullptr,
                           ctx->refl_frame ? (float*)ctx->refl_t.p : nullptr, ctx->stream));
  return VM_OK;
}

int vm_water_sec(vm_ctx* ctx, uint32_t shift) {
  if (!ctx) return VM_E_INVALID;
  int rc = check_ready(ctx);
  if (rc) return rc;
  if (shift > 3) return fail(ctx, VM_E_INVALID, "water_sec shift %u outside 0..3", shift);
  CK(cudaSetDevice(ctx->device));
  const vm_frame& f = ctx->frame;
  const uint32_t span = 1u << shift;
  const size_t cells = (size_t)((f.res[0] + span - 1) >> shift) * ((f.res[1] + span - 1) >> shift);
  if ((rc = ensure(ctx, ctx->ws_refr_key, cells * 8)) || (rc = ensure(ctx, ctx->ws_refr_t, cells * 4)) ||
      (rc = ensure(ctx, ctx->ws_refl_key, cells * 8)) || (rc = ensure(ctx, ctx->ws_refl_t, cells * 4)))
    return rc;
  CK(vmk::launch_water_sec(f, dev_world(ctx), (const unsigned long long*)ctx->vis.p, shift,
                           (unsigned long long*)ctx->ws_refr_key.p, (float*)ctx->ws_refr_t.p,
                           (unsigned long long*)ctx->ws_refl_key.p, (float*)ctx->ws_refl_t.p, ctx->stream));
  ctx->ws_shift = shift;
  ctx->ws_cells = (uint32_t)cells;
  ctx->ws_done = true;
  return VM_OK;
}

static int read_dev(vm_ctx* ctx, void* dst, const void* src, size_t bytes);

int vm_read_water_sec(vm_ctx* ctx, uint64_t* refr_key, float* refr_t, uint64_t* refl_key, float* refl_t) {
  if (!ctx || !ctx->ws_done) return ctx ? fail(ctx, VM_E_NOT_READY, "no vm_water_sec yet") : VM_E_INVALID;
  const size_t n = ctx->ws_cells;
  int rc = VM_OK;
  if (refr_key && (rc = read_dev(ctx, refr_key, ctx->ws_refr_key.p, n * 8))) return rc;
  if (refr_t && (rc = read_dev(ctx, refr_t, ctx->ws_refr_t.p, n * 4))) return rc;
  if (refl_key && (rc = read_dev(ctx, refl_key, ctx->ws_refl_key.p, n * 8))) return rc;
  if (refl_t && (rc = read_dev(ctx, refl_t, ctx->ws_refl_t.p, n * 4))) return rc;
  return VM_OK;
}

int vm_render(vm_ctx* ctx) {
  if (!ctx) return VM_E_INVALID;
  int rc = check_ready(ctx);
  if (rc) return rc;
  CK(cudaSetDevice(ctx->device));
  if ((rc = enqueue_render(ctx, false))) return rc;
  if (!ctx->rendered) CK(cudaEventCreateWithFlags(&ctx->rendered, cudaEventDisableTiming));
  CK(cudaEventRecord(ctx->rendered, ctx->stream));
  ctx->have_rendered = true;
  return VM_OK;
}

int vm_wait_render(vm_ctx* ctx, vm_ctx* other) {
  if (!ctx || !other) return VM_E_INVALID;
  if (!other->have_rendered) return VM_OK;
  CK(cudaSetDevice(ctx->device));
  CK(cudaStreamWaitEvent(ctx->stream, other->rendered, 0));
  return VM_OK;
}

static int read_traffic(vm_ctx* ctx, vm_traffic* out);

int vm_render_events(vm_ctx* ctx, void* const* events) {
  if (!ctx || !events) return VM_E_INVALID;
  for (int i = 0; i < 5; ++i)
    if (!events[i]) return fail(ctx, VM_E_INVALID, "event %d is null", i);
  int rc = check_ready(ctx);
  if (rc) return rc;
  CK(cudaSetDevice(ctx->device));
  return enqueue_render(ctx, false, (const cudaEvent_t*)events);
}

int vm_render_counted(vm_ctx* ctx, vm_traffic* out) {
  if (!ctx || !out) return VM_E_INVALID;
  int rc = check_ready(ctx);
  if (rc) return rc;
  CK(cudaSetDevice(ctx->device));
  CK(cudaMemsetAsync(ctx->traffic.p, 0, 3 * sizeof(vmk::Traffic64), ctx->stream));
  if ((rc = enqueue_render(ctx, true))) return rc;
  return read_traffic(ctx, out);
}

static int read_traffic(vm_ctx* ctx, vm_traffic* out) {
  vmk::Traffic64 st[3];
  CK(cudaMemcpyAsync(st, ctx->traffic.p, sizeof st, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  memset(out, 0, sizeof *out);
  for (const vmk::Traffic64& t : st) {
    out->chunk_records += t.chunk; out->l1_fetches += t.l1; out->leaf_fetches += t.leaf; out->attr_fetches += t.attr;
    out->palette_decodes += t.pal; out->grid_lookups += t.grid; out->iters += t.iters;
    out->rays_primary += t.rays_primary; out->rays_shadow += t.rays_shadow; out->rays_secondary += t.rays_secondary;
    out->list_entries += t.entries;
  }
  for (int s = 0; s < 3; ++s) {
    out->stage_iters[s] = st[s].iters;
    out->stage_chunks[s] = st[s].chunk;
    // algorithmic bytes: the layout's element sizes times the fetches counted
    out->stage_bytes[s] = 96ull * st[s].chunk + 16ull * st[s].l1 + 8ull * st[s].leaf + 4ull * st[s].attr +
                          12ull * st[s].pal + 4ull * st[s].grid;
  }
  return VM_OK;
}

static int read_dev(vm_ctx* ctx, void* dst, const void* src, size_t bytes) {
  if (!dst) return fail(ctx, VM_E_INVALID, "null output");
  CK(cudaSetDevice(ctx->device));
  CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return VM_OK;
}

int vm_read_async(vm_ctx* ctx, uint64_t* vis, float* shadow) {
  if (!ctx || !ctx->have_frame) return VM_E_NOT_READY;
  CK(cudaSetDevice(ctx->device));
  const size_t npix = (size_t)ctx->frame.res[0] * ctx->frame.res[1];
  if (vis) CK(cudaMemcpyAsync(vis, ctx->vis.p, npix * 8, cudaMemcpyDeviceToHost, ctx->stream));
  if (shadow) CK(cudaMemcpyAsync(shadow, ctx->shadow.p, npix * 4, cudaMemcpyDeviceToHost, ctx->stream));
  return VM_OK;
}

int vm_read_async_r16f(vm_ctx* ctx, uint64_t* vis, uint16_t* shadow) {
  if (!ctx || !ctx->have_frame) return VM_E_NOT_READY;
  CK(cudaSetDevice(ctx->device));
  const size_t npix = (size_t)ctx->frame.res[0] * ctx->frame.res[1];
  if (vis) CK(cudaMemcpyAsync(vis, ctx->vis.p, npix * 8, cudaMemcpyDeviceToHost, ctx->stream));
  if (shadow) {
    int rc;
    if ((rc = ensure(ctx, ctx->shadow16, npix * 2))) return rc;
    CK(vmk::launch_to_r16f((const float*)ctx->shadow.p, (uint16_t*)ctx->shadow16.p, npix, ctx->sms, ctx->stream));
    CK(cudaMemcpyAsync(shadow, ctx->shadow16.p, npix * 2, cudaMemcpyDeviceToHost, ctx->stream));
  }
  return VM_OK;
}

int vm_read_vis(vm_ctx* ctx, uint64_t* out) {
  if (!ctx || !ctx->have_frame) return VM_E_NOT_READY;
  return read_dev(ctx, out, ctx->vis.p, (size_t)ctx->frame.res[0] * ctx->frame.res[1] * 8);
}
int vm_read_hiz(vm_ctx* ctx, uint32_t* out) {
  if (!ctx || !ctx->have_frame) return VM_E_NOT_READY;
  return read_dev(ctx, out, ctx->hiz.p, (size_t)ctx->frame.tiles[0] * ctx->frame.tiles[1] * 4);
}
int vm_write_hiz(vm_ctx* ctx, const uint32_t* hiz) {
  if (!ctx || !ctx->have_frame || !hiz) return VM_E_NOT_READY;
  CK(cudaSetDevice(ctx->device));
  CK(cudaMemcpyAsync(ctx->hiz.p, hiz, (size_t)ctx->frame.tiles[0] * ctx->frame.tiles[1] * 4, cudaMemcpyHostToDevice,
                     ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return VM_OK;
}
int vm_read_shadow(vm_ctx* ctx, float* out) {
  if (!ctx || !ctx->have_frame) return VM_E_NOT_READY;
  return read_dev(ctx, out, ctx->shadow.p, (size_t)ctx->frame.res[0] * ctx->frame.res[1] * 4);
}
int vm_read_shadow_mask(vm_ctx* ctx, float* out) {
  if (!ctx || !ctx->have_frame) return VM_E_NOT_READY;
  const size_t bytes = (size_t)ctx->frame.res[0] * ctx->frame.res[1] * 4;
  if (!ctx->shadow_mask.p || ctx->shadow_mask.bytes < bytes)
    return fail(ctx, VM_E_NOT_READY, "no shadow mask: call vm_soften_shadows first");
  return read_dev(ctx, out, ctx->shadow_mask.p, bytes);
}
int vm_read_secondary(vm_ctx* ctx, uint64_t* key, float* t) {
  if (!ctx || !ctx->have_frame) return VM_E_NOT_READY;
  const size_t n = (size_t)ctx->frame.res[0] * ctx->frame.res[1];
  int rc = read_dev(ctx, key, ctx->sec_key.p, n * 8);
  if (rc) return rc;
  return read_dev(ctx, t, ctx->sec_t.p, n * 4);
}
int vm_read_reflection(vm_ctx* ctx, uint64_t* key, float* t) {
  if (!ctx || !ctx->have_frame) return VM_E_NOT_READY;
  if (!ctx->refl_frame) return fail(ctx, VM_E_NOT_READY, "the last frame had no FLAG_WATER_REFLECT");
  const size_t n = (size_t)ctx->frame.res[0] * ctx->frame.res[1];
  int rc = read_dev(ctx, key, ctx->refl_key.p, n * 8);
  if (rc) return rc;
  return read_dev(ctx, t, ctx->refl_t.p, n * 4);
}
int vm_read_heatmap(vm_ctx* ctx, uint32_t* out) {
  if (!ctx || !ctx->have_frame) return VM_E_NOT_READY;
  return read_dev(ctx, out, ctx->dbg.p, (size_t)ctx->frame.res[0] * ctx->frame.res[1] * 4);
}

int vm_read_expanded(vm_ctx* ctx, const int32_t origin[3], const uint32_t dims[3], uint32_t* voxel, uint8_t* face,
                     float* t) {
  if (!ctx) return VM_E_INVALID;
  int rc = check_ready(ctx);
  if (rc) return rc;
  if (!origin || !dims || !voxel || !face || !t) return fail(ctx, VM_E_INVALID, "null argument");
  CK(cudaSetDevice(ctx->device));
  const vm_frame& f = ctx->frame;
  const size_t n = (size_t)f.res[0] * f.res[1];
  uint32_t* dv = (uint32_t*)ctx->expand.p;
  float* dt = (float*)((char*)ctx->expand.p + n * 4);
  uint8_t* df = (uint8_t*)((char*)ctx->expand.p + n * 8);
  CK(vmk::launch_expand(f, dev_world(ctx), (const unsigned long long*)ctx->vis.p, origin[0], origin[1], origin[2], dims[0],
                        dims[1], dims[2], dv, df, dt, ctx->stream));
  CK(cudaMemcpyAsync(voxel, dv, n * 4, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaMemcpyAsync(t, dt, n * 4, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaMemcpyAsync(face, df, n, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return VM_OK;
}

int vm_stats_read(vm_ctx* ctx, vm_stats* out) {
  if (!ctx || !out) return VM_E_INVALID;
  CK(cudaSetDevice(ctx->device));
  memset(out, 0, sizeof *out);
  uint32_t c[8] = {0}, e = 0;
  CK(cudaMemcpyAsync(c, ctx->counters.p, 32, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaMemcpyAsync(&e, ctx->err.p, 4, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  memcpy(out->counters, c, sizeof c);
  out->pairs_selected = c[4];
  out->pairs_deferred = c[1];
  out->pairs_recovered = c[5];
  out->max_pairs = ctx->frame.max_pairs;
  out->truncated = (c[4] > out->max_pairs || c[1] > out->max_pairs || c[5] > out->max_pairs) ? 1u : 0u;
  out->device_error = e;
  return VM_OK;
}

// ---------------------------------------------------------------------------
// batches
// ---------------------------------------------------------------------------
int vm_batch_set(vm_ctx* ctx, uint32_t n_views, const vm_frame* frames, const vm_chunk* chunks,
                 const uint32_t* chunk_counts, const uint32_t* grids, const uint32_t* grid_lens) {
  if (!ctx || n_views == 0 || !frames || !chunks || !chunk_counts || !grids || !grid_lens) return VM_E_INVALID;
  if (!ctx->have_world) return fail(ctx, VM_E_NOT_READY, "no world uploaded");
  if (ctx->caps.max_views && n_views > ctx->caps.max_views)
    return fail(ctx, VM_E_INVALID, "%u views exceed the context capacity %u", n_views, ctx->caps.max_views);
  CK(cudaSetDevice(ctx->device));
  ctx->bh_frames.assign(frames, frames + n_views);
  ctx->bh_views.assign(n_views, ViewDesc{});
  std::vector<ViewDesc> single(n_views);
  uint64_t chunk_total = 0, grid_total = 0, pix = 0, tiles = 0, supers = 0;
  uint32_t max_vis = 1;
  const bool uw = (frames[0].flags & VM_FLAG_UNDERWATER) != 0u;
  for (uint32_t v = 0; v < n_views; ++v) {
    const vm_frame& f = frames[v];
    int rc = check_frame(ctx, f, chunk_counts[v], grid_lens[v]);
    if (rc) return fail(ctx, rc, "view %u: %s", v, ctx->err_text.c_str());
    if (((f.flags & VM_FLAG_UNDERWATER) != 0u) != uw)
      return fail(ctx, VM_E_INVALID, "views of one batch must agree on FLAG_UNDERWATER");
    ViewDesc& d = ctx->bh_views[v];
    d.chunk_off = (uint32_t)chunk_total;
    d.n_chunks = chunk_counts[v];
    d.grid_off = grid_total;
    d.grid_len = grid_lens[v];
    d.pix_off = pix;
    d.tile_begin = (uint32_t)tiles;
    d.super_begin = (uint32_t)supers;
    d.tiles_x = f.tiles[0];
    d.tiles_y = f.tiles[1];
    single[v] = d;
    single[v].tile_begin = 0;   // per-view launches index their own tile scratch from 0
    single[v].super_begin = 0;
    chunk_total += chunk_counts[v];
    grid_total += grid_lens[v];
    pix += (uint64_t)f.res[0] * f.res[1];
    tiles += (uint64_t)f.tiles[0] * f.tiles[1];
    supers += (uint64_t)((f.tiles[0] + 3) / 4) * ((f.tiles[1] + 3) / 4);
    max_vis = std::max(max_vis, std::min(f.chunk_count, chunk_counts[v]));
  }
  if (ctx->caps.max_batch_pixels && pix > ctx->caps.max_batch_pixels)
    return fail(ctx, VM_E_INVALID, "batch of %llu pixels exceeds the context capacity", (unsigned long long)pix);
  if (tiles > 0xFFFFFFFFull) return fail(ctx, VM_E_INVALID, "too many tiles in one batch");
  const uint32_t cap = std::min(max_vis, LIST_CAP_MAX);
  int rc = 0;
  rc |= ensure(ctx, ctx->b_frames, n_views * sizeof(vm_frame));
  rc |= ensure(ctx, ctx->b_views, n_views * sizeof(ViewDesc));
  rc |= ensure(ctx, ctx->b_views1, n_views * sizeof(ViewDesc));
  rc |= ensure(ctx, ctx->b_chunks, std::max<uint64_t>(chunk_total, 1) * sizeof(vm_chunk));
  rc |= ensure(ctx, ctx->b_grids, grid_total * 4);
  rc |= ensure(ctx, ctx->b_vis, pix * 8);
  rc |= ensure(ctx, ctx->b_shadow, pix * 4);
  rc |= ensure(ctx, ctx->b_seck, pix * 8);
  rc |= ensure(ctx, ctx->b_sect, pix * 4);
  rc |= ensure(ctx, ctx->b_hiz, tiles * 4);
  rc |= ensure(ctx, ctx->b_dkmax, std::max<uint64_t>(chunk_total, 1) * 4);
  rc |= ensure(ctx, ctx->b_sufmax, std::max<uint64_t>(chunk_total, 1) * 4);
  rc |= ensure(ctx, ctx->b_tile_list, tiles * cap * 2);
  rc |= ensure(ctx, ctx->b_tile_count, tiles * 4);
  rc |= ensure(ctx, ctx->b_super_list, std::max<uint64_t>(supers, 1) * cap * 2);
  rc |= ensure(ctx, ctx->b_super_count, std::max<uint64_t>(supers, 1) * 4);
  rc |= ensure(ctx, ctx->b_shadow_q, pix * sizeof(vmk::ShadowItem));
  rc |= ensure(ctx, ctx->b_sec_q, pix * sizeof(vmk::SecItem));
  rc |= ensure(ctx, ctx->b_item_cost, tiles * 8);
  rc |= ensure(ctx, ctx->b_tile_order, tiles * 4);
  if (rc) return VM_E_CUDA;
  CK(cudaMemsetAsync(ctx->b_item_cost.p, 0, tiles * 8, ctx->stream));   // a new batch: no costs yet
  CK(cudaMemcpyAsync(ctx->b_frames.p, frames, n_views * sizeof(vm_frame), cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(ctx->b_chunks.p, chunks, chunk_total * sizeof(vm_chunk), cudaMemcpyHostToDevice, ctx->stream));
  ctx->batch_foliage = false;
  for (uint64_t i = 0; i < chunk_total && !ctx->batch_foliage; ++i)
    ctx->batch_foliage = (chunks[i].attr_flags & VM_ATTR_HAS_FOLIAGE) != 0u;
  CK(cudaMemcpyAsync(ctx->b_grids.p, grids, grid_total * 4, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(ctx->b_views.p, ctx->bh_views.data(), n_views * sizeof(ViewDesc), cudaMemcpyHostToDevice,
                     ctx->stream));
  CK(cudaMemcpyAsync(ctx->b_views1.p, single.data(), n_views * sizeof(ViewDesc), cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  ctx->b_n_views = n_views;
  ctx->b_pixels = pix;
  ctx->b_n_chunks = (uint32_t)chunk_total;
  ctx->b_grid_total = grid_total;
  ctx->b_total_tiles = (uint32_t)tiles;
  ctx->b_total_supers = (uint32_t)supers;
  ctx->b_list_cap = cap;
  ctx->b_underwater = uw;
  drop_graph(ctx);
  return VM_OK;
}

static vmk::PipeArgs batch_args(vm_ctx* ctx, bool secondary) {
  vmk::PipeArgs a = base_args(ctx);
  a.tufts = a.atlas_alpha != nullptr && (ctx->spec & VM_SPEC_FOLIAGE) != 0u && ctx->batch_foliage ? 1u : 0u;
  a.frames = (const vm_frame*)ctx->b_frames.p;
  a.views = (const ViewDesc*)ctx->b_views.p;
  a.n_views = ctx->b_n_views;
  a.total_tiles = ctx->b_total_tiles;
  a.chunks = (const vm_chunk*)ctx->b_chunks.p;
  a.grids = (const uint32_t*)ctx->b_grids.p;
  a.dkmax = (uint32_t*)ctx->b_dkmax.p;
  a.sufmax = (uint32_t*)ctx->b_sufmax.p;
  a.tile_list = (uint16_t*)ctx->b_tile_list.p;
  a.tile_count = (uint32_t*)ctx->b_tile_count.p;
  a.super_list = (uint16_t*)ctx->b_super_list.p;
  a.super_count = (uint32_t*)ctx->b_super_count.p;
  a.total_supers = ctx->b_total_supers;
  a.list_cap = ctx->b_list_cap;
  a.vis = (unsigned long long*)ctx->b_vis.p;
  a.shadow = (float*)ctx->b_shadow.p;
  a.sec_key = (unsigned long long*)ctx->b_seck.p;
  a.sec_t = (float*)ctx->b_sect.p;
  a.hiz = (uint32_t*)ctx->b_hiz.p;
  a.shadow_q = (vmk::ShadowItem*)ctx->b_shadow_q.p;
  a.sec_q = (vmk::SecItem*)ctx->b_sec_q.p;
  a.item_cost = (uint32_t*)ctx->b_item_cost.p;
  a.tile_order = (uint32_t*)ctx->b_tile_order.p;
  a.do_secondary = secondary ? 1 : 0;   // batched views: primary + shadow, optionally the water / glass rays
  return a;
}

int vm_batch_run(vm_ctx* ctx, int mode) {
  if (!ctx) return VM_E_INVALID;
  if (ctx->b_n_views == 0) return fail(ctx, VM_E_NOT_READY, "no batch set");
  CK(cudaSetDevice(ctx->device));
  if (mode & ~(VM_BATCH_PER_VIEW | VM_BATCH_SECONDARY)) return fail(ctx, VM_E_INVALID, "unknown batch mode %d", mode);
  const bool secondary = (mode & VM_BATCH_SECONDARY) != 0;
  if ((mode & VM_BATCH_PER_VIEW) == 0) {
    // every view in one pipeline: one launch per stage, replayed from a graph
    if (ctx->graph_exec && ctx->graph_secondary != secondary) drop_graph(ctx);
    if (!ctx->graph_exec) {
      CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
      const vmk::PipeArgs a = batch_args(ctx, secondary);
      const cudaError_t le = vmk::launch_pipeline(a, ctx->tuning, ctx->b_underwater, false, ctx->sms, ctx->stream);
      cudaGraph_t g = nullptr;
      const cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
      if (le != cudaSuccess) { if (g) cudaGraphDestroy(g); return cuda_fail(ctx, le, "launch_pipeline"); }
      if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaStreamEndCapture");
      ctx->graph = g;
      ctx->graph_secondary = secondary;
      CK(cudaGraphInstantiate(&ctx->graph_exec, g, 0));
    }
    CK(cudaGraphLaunch(ctx->graph_exec, ctx->stream));
    return VM_OK;
  }
  {
    // the baseline: one launch sequence per view (same kernels)
    const vmk::PipeArgs base = batch_args(ctx, secondary);
    for (uint32_t v = 0; v < ctx->b_n_views; ++v) {
      vmk::PipeArgs a = base;
      const ViewDesc& d = ctx->bh_views[v];
      a.frames = (const vm_frame*)ctx->b_frames.p + v;
      a.views = (const ViewDesc*)ctx->b_views1.p + v;
      a.n_views = 1;
      a.total_tiles = d.tiles_x * d.tiles_y;
      a.hiz = (uint32_t*)ctx->b_hiz.p + d.tile_begin;
      a.item_cost = (uint32_t*)ctx->b_item_cost.p + 2ull * d.tile_begin;
      a.tile_order = (uint32_t*)ctx->b_tile_order.p + d.tile_begin;
      a.super_list = (uint16_t*)ctx->b_super_list.p + (uint64_t)d.super_begin * ctx->b_list_cap;
      a.super_count = (uint32_t*)ctx->b_super_count.p + d.super_begin;
      a.total_supers = ((d.tiles_x + 3) / 4) * ((d.tiles_y + 3) / 4);
      CK(vmk::launch_pipeline(a, ctx->tuning, ctx->b_underwater, false, ctx->sms, ctx->stream));
    }
    return VM_OK;
  }
}

int vm_batch_counted(vm_ctx* ctx, int secondary, vm_traffic* out) {
  if (!ctx || !out) return VM_E_INVALID;
  if (ctx->b_n_views == 0) return fail(ctx, VM_E_NOT_READY, "no batch set");
  CK(cudaSetDevice(ctx->device));
  CK(cudaMemsetAsync(ctx->traffic.p, 0, 3 * sizeof(vmk::Traffic64), ctx->stream));
  const vmk::PipeArgs a = batch_args(ctx, secondary != 0);
  CK(vmk::launch_pipeline(a, ctx->tuning, ctx->b_underwater, true, ctx->sms, ctx->stream));
  return read_traffic(ctx, out);
}

int vm_batch_read(vm_ctx* ctx, uint64_t* vis, float* shadow) {
  if (!ctx || ctx->b_n_views == 0) return VM_E_NOT_READY;
  int rc = VM_OK;
  if (vis) rc = read_dev(ctx, vis, ctx->b_vis.p, ctx->b_pixels * 8);
  if (rc) return rc;
  if (shadow) rc = read_dev(ctx, shadow, ctx->b_shadow.p, ctx->b_pixels * 4);
  return rc;
}

uint64_t vm_batch_pixels(const vm_ctx* ctx) { return ctx ? ctx->b_pixels : 0; }

int vm_batch_read_secondary(vm_ctx* ctx, uint64_t* key, float* t) {
  if (!ctx || ctx->b_n_views == 0) return VM_E_NOT_READY;
  int rc = VM_OK;
  if (key) rc = read_dev(ctx, key, ctx->b_seck.p, ctx->b_pixels * 8);
  if (rc) return rc;
  if (t) rc = read_dev(ctx, t, ctx->b_sect.p, ctx->b_pixels * 4);
  return rc;
}

int vm_device_buffers(vm_ctx* ctx, vm_device_ptrs* out) {
  if (!ctx || !out) return VM_E_INVALID;
  out->vis = ctx->vis.p; out->shadow = ctx->shadow.p; out->sec_key = ctx->sec_key.p; out->sec_t = ctx->sec_t.p;
  out->hiz = ctx->hiz.p; out->batch_vis = ctx->b_vis.p; out->batch_shadow = ctx->b_shadow.p;
  out->stream = (void*)ctx->stream;
  return VM_OK;
}

int vm_sync(vm_ctx* ctx) {
  if (!ctx) return VM_E_INVALID;
  CK(cudaSetDevice(ctx->device));
  CK(cudaStreamSynchronize(ctx->stream));
  return VM_OK;
}

}  // extern "C"

// The batch's pipeline arguments (with the secondary-ray outputs) and stream,
// for the shading G-buffer pass (gbuffer.cu).
int vm_internal_batch_args(vm_ctx* ctx, vmk::PipeArgs* out, uint64_t* pixels, void** stream) {
  if (!ctx || !out || !pixels || !stream) return VM_E_INVALID;
  if (ctx->b_n_views == 0) return fail(ctx, VM_E_NOT_READY, "no batch set");
  CK(cudaSetDevice(ctx->device));
  *out = batch_args(ctx, true);
  *pixels = ctx->b_pixels;
  *stream = (void*)ctx->stream;
  return VM_OK;
}

// ---------------------------------------------------------------------------
// The resolve of sky and opaque pixels (lane 0 of resolve.wgsl:1378-1466) and
// its material inputs.

namespace {

// the sRGB transfer function (IEC 61966-2-1), as the texture unit applies it
// to an Rgba8UnormSrgb texel before filtering
float srgb_decode(uint8_t u) {
  const float c = (float)u / 255.0f;
  return c <= 0.04045f ? c / 12.92f : powf((c + 0.055f) / 1.055f, 2.4f);
}

// FLAG_HI_COMPACT_SHADE_HIT (131072) is accepted: shade_hit_compact(_cached)
// runs shade_hit_legacy(_cached)'s statements with the material block after
// the light block (the light times face_scale = 1.0, the canopy relief from
// the same n . sun), so its colours are the legacy variant's bit for bit.
constexpr uint32_t HI_WATER_SEC = 32u;
constexpr uint32_t WATER_SEC_SHIFT = 1u;   // WATER_SEC_SHIFT of the engine's default water_sec_scale 2

}  // namespace

int vm_upload_atlas(vm_ctx* ctx, const uint8_t* rgba, uint32_t layers, uint32_t size, uint32_t mips) {
  if (!ctx) return VM_E_INVALID;
  if (!rgba || layers == 0 || layers > 0xFFFFu) return fail(ctx, VM_E_INVALID, "atlas needs 1..65535 layers");
  if (size != VM_ATLAS_SIZE || mips != VM_ATLAS_MIPS)
    return fail(ctx, VM_E_INVALID, "atlas must be %ux%u with %u mips (got %ux%u, %u)", VM_ATLAS_SIZE, VM_ATLAS_SIZE,
                VM_ATLAS_MIPS, size, size, mips);
  size_t texels = 0;
  for (uint32_t m = 0; m < mips; ++m) texels += (size_t)layers * (size >> m) * (size >> m);
  std::vector<float> lin(texels * 4);
  for (size_t i = 0; i < texels; ++i) {
    for (int c = 0; c < 3; ++c) lin[i * 4 + c] = srgb_decode(rgba[i * 4 + c]);
    lin[i * 4 + 3] = (float)rgba[i * 4 + 3] / 255.0f;
  }
  CK(cudaSetDevice(ctx->device));
  int rc;
  if ((rc = ensure(ctx, ctx->atlas, lin.size() * 4))) return rc;
  CK(cudaMemcpyAsync(ctx->atlas.p, lin.data(), lin.size() * 4, cudaMemcpyHostToDevice, ctx->stream));
  std::vector<float> alpha(texels);
  for (size_t i = 0; i < texels; ++i) alpha[i] = lin[i * 4 + 3];
  if ((rc = ensure(ctx, ctx->atlas_alpha, alpha.size() * 4))) return rc;
  CK(cudaMemcpyAsync(ctx->atlas_alpha.p, alpha.data(), alpha.size() * 4, cudaMemcpyHostToDevice, ctx->stream));
  drop_graph(ctx);   // cached launches carry the atlas pointers
  // (cos, sin) of the simplex gradient angles (resolve.wgsl:175-192)
  float grad[64];
  for (uint32_t k = 0; k < 32; ++k) {
    const float a = k < 24 ? 1.4398966328953218f - 0.26179938779914946f * (float)k
                           : 1.1780972450961724f - 0.7853981633974483f * (float)(k - 24);
    grad[2 * k] = cosf(a);
    grad[2 * k + 1] = sinf(a);
  }
  if ((rc = ensure(ctx, ctx->grad, sizeof grad))) return rc;
  CK(cudaMemcpyAsync(ctx->grad.p, grad, sizeof grad, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  ctx->atlas_layers = layers;
  return VM_OK;
}

int vm_upload_block_faces(vm_ctx* ctx, const uint32_t* words, uint32_t n) {
  if (!ctx) return VM_E_INVALID;
  if (!words || n == 0 || n % 8u != 0u) return fail(ctx, VM_E_INVALID, "block faces: 8 words per block id");
  CK(cudaSetDevice(ctx->device));
  int rc;
  if ((rc = ensure(ctx, ctx->faces, (size_t)n * 4))) return rc;
  CK(cudaMemcpyAsync(ctx->faces.p, words, (size_t)n * 4, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  ctx->n_faces = n;
  // the cross-quad layer of each tuft block (block_faces[id * 8 + NORMAL_CROSS_A])
  const uint32_t tufts[3] = {VM_TALL_GRASS, VM_GRASS_TALL, VM_REEDS};
  for (int i = 0; i < 3; ++i) {
    const uint32_t k = tufts[i] * 8u + VM_NORMAL_CROSS_A;
    ctx->tuft_layer[i] = k < n ? (words[k] & 0xFFFFu) : 0u;
  }
  drop_graph(ctx);
  return VM_OK;
}

int vm_upload_probes(vm_ctx* ctx, const uint16_t* rgba16f, uint32_t nx, uint32_t ny, uint32_t nz) {
  if (!ctx) return VM_E_INVALID;
  if (!rgba16f) { ctx->have_probes = false; return VM_OK; }
  if (nx != VM_PROBE_NX || ny != VM_PROBE_NY || nz != VM_PROBE_NZ)
    return fail(ctx, VM_E_INVALID, "probe field must be %ux%ux%u", VM_PROBE_NX, VM_PROBE_NY, VM_PROBE_NZ);
  const size_t bytes = (size_t)nx * ny * nz * 8;
  CK(cudaSetDevice(ctx->device));
  int rc;
  if ((rc = ensure(ctx, ctx->probes, bytes))) return rc;
  CK(cudaMemcpyAsync(ctx->probes.p, rgba16f, bytes, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  ctx->have_probes = true;
  return VM_OK;
}

int vm_upload_shaft(vm_ctx* ctx, const float* envelope, uint32_t dim) {
  if (!ctx) return VM_E_INVALID;
  if (!envelope) { ctx->have_shaft = false; return VM_OK; }
  if (dim != VM_SHAFT_DIM) return fail(ctx, VM_E_INVALID, "shaft envelope must be %ux%u", VM_SHAFT_DIM, VM_SHAFT_DIM);
  const size_t bytes = (size_t)dim * dim * 4;
  CK(cudaSetDevice(ctx->device));
  int rc;
  if ((rc = ensure(ctx, ctx->shaft, bytes))) return rc;
  CK(cudaMemcpyAsync(ctx->shaft.p, envelope, bytes, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  ctx->have_shaft = true;
  return VM_OK;
}

int vm_resolve(vm_ctx* ctx, uint32_t spec_hi) {
  if (!ctx) return VM_E_INVALID;
  int rc = check_ready(ctx);
  if (rc) return rc;
  const vm_frame& f = ctx->frame;
  const size_t npix = (size_t)f.res[0] * f.res[1];
  if (!ctx->vis.p || ctx->vis.bytes < npix * 8 || !ctx->shadow.p)
    return fail(ctx, VM_E_NOT_READY, "no rendered frame to resolve");
  if (f.flags & VM_FLAG_HEATMAP) {
    // the engine's heat-map view (resolve.wgsl:1389-1394): the iteration
    // counts its march summed per pixel, which vm_select / vm_march keep
    if (!ctx->heat_valid)
      return fail(ctx, VM_E_NOT_READY, "a heat-map frame resolves the iteration counts of vm_select / vm_march");
    CK(cudaSetDevice(ctx->device));
    if ((rc = ensure(ctx, ctx->color, npix * 16))) return rc;
    CK(vmk::launch_resolve_heat(f, (const uint32_t*)ctx->dbg.p, (float4*)ctx->color.p, ctx->stream));
    ctx->color_done = true;
    return VM_OK;
  }
  if (!ctx->atlas_layers || !ctx->n_faces) return fail(ctx, VM_E_NOT_READY, "no atlas / block faces uploaded");

  CK(cudaSetDevice(ctx->device));
  if ((rc = ensure(ctx, ctx->color, npix * 16)) || (rc = ensure(ctx, ctx->light_ao, npix * 4)) ||
      (rc = ensure(ctx, ctx->lane, npix)) || (rc = ensure(ctx, ctx->lane_lists, npix * 8 + 8)) ||
      (rc = ensure(ctx, ctx->fog, npix * 16)))
    return rc;
  if (!ctx->lane_stream[0]) {
    // default priority: the lanes' long-latency threads are launched first and
    // fill the SM slots the issue-bound lanes leave (a higher priority for
    // them measured 1.5% slower)
    for (cudaStream_t& ls : ctx->lane_stream) CK(cudaStreamCreateWithFlags(&ls, cudaStreamNonBlocking));
    for (cudaEvent_t& e : ctx->lane_event) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  }
  vmd::Look L;
  L.atlas = (const float4*)ctx->atlas.p; L.atlas_layers = ctx->atlas_layers;
  L.faces = (const uint32_t*)ctx->faces.p; L.n_faces = ctx->n_faces;
  L.probes = ctx->have_probes ? (const ushort4*)ctx->probes.p : nullptr;
  L.shaft = ctx->have_shaft ? (const float*)ctx->shaft.p : nullptr;
  L.grad = (const float2*)ctx->grad.p;
  L.spec_hi = spec_hi;
  const float* mask = ctx->mask_valid ? (const float*)ctx->shadow_mask.p : nullptr;
  uint16_t *refr = nullptr, *refl = nullptr;
  if (spec_hi & HI_WATER_SEC) {
    const uint32_t span = 1u << WATER_SEC_SHIFT;
    const size_t cells = (size_t)((f.res[0] + span - 1) >> WATER_SEC_SHIFT) * ((f.res[1] + span - 1) >> WATER_SEC_SHIFT);
    if ((rc = ensure(ctx, ctx->leg_refr, cells * 8)) || (rc = ensure(ctx, ctx->leg_refl, cells * 8))) return rc;
    refr = (uint16_t*)ctx->leg_refr.p;
    refl = (uint16_t*)ctx->leg_refl.p;
  }
  CK(vmk::launch_resolve(f, dev_world(ctx), L, (const unsigned long long*)ctx->vis.p, mask,
                         (const float*)ctx->shadow.p, (ctx->spec & VM_SPEC_SOFT_RAYS) != 0u, WATER_SEC_SHIFT, refr,
                         refl, (uint8_t*)ctx->lane.p, (uint32_t*)ctx->lane_lists.p, (float*)ctx->light_ao.p,
                         (float4*)ctx->fog.p, (float4*)ctx->color.p, ctx->sms, ctx->stream, ctx->lane_stream,
                         ctx->lane_event));
  ctx->color_done = true;
  return VM_OK;
}

int vm_read_color(vm_ctx* ctx, float* rgba) {
  if (!ctx) return VM_E_INVALID;
  if (!ctx->color_done) return fail(ctx, VM_E_NOT_READY, "no vm_resolve for this frame");
  return read_dev(ctx, rgba, ctx->color.p, (size_t)ctx->frame.res[0] * ctx->frame.res[1] * 16);
}
