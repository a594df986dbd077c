// The frame as a wavefront pipeline of warp-independent kernels, sm_100a.
//
//   k_prepass  blocks [0, views): for every visible chunk, the largest depth
//              key a hit in it can have (from a lower bound on its distance)
//              and the suffix maximum of that bound along the view's
//              front-to-back chunk list; the other blocks: one warp per
//              32x32 super-tile, the chunks its frustum cannot rule out;
//   k_cull     one block per super-tile, one warp per 8x8 tile:
//              tile_select's exact test (tile_select.wgsl:11-92) over the
//              super-tile's survivors, written as the tile's ascending chunk
//              list;
//   k_order    the tiles in decreasing order of the last launch's item cost;
//   k_primary  persistent warps steal 8x4-pixel items in that order; each
//              lane marches its pixel through the tile's list front to back
//              and stops as soon as no remaining chunk can produce a key
//              above the pixel's current one (and a march stops at the
//              distance past which it cannot), so the key equals the engine's
//              atomicMax over all of the tile's pairs; the lane then queues
//              its shadow ray and its water / glass ray, one atomic per warp;
//   k_shadow   persistent lanes step their queued sun ray one chunk march at
//              a time and take the next ray as soon as theirs ends;
//   k_secondary_q the same for the queued water / glass rays (trace_world).
//
// Only the prepass's depth bounds (a block scan), k_cull (its staged boxes)
// and k_order (a block's ranking) synchronise a block; everywhere else warps
// never wait on other warps.
#include "kernels.cuh"
#include "ray_stages.cuh"
#include <cub/block/block_scan.cuh>
#include <algorithm>

namespace vmk {

__device__ __forceinline__ uint32_t find_view(const PipeArgs& a, uint32_t tile) {
  if (a.frames == nullptr) return 0;
  uint32_t lo = 0, hi = a.n_views - 1;
  while (lo < hi) {
    const uint32_t mid = (lo + hi + 1) >> 1;
    if (a.views[mid].tile_begin <= tile) lo = mid; else hi = mid - 1;
  }
  return lo;
}
__device__ __forceinline__ const vm_frame& frame_of(const PipeArgs& a, uint32_t v) {
  return a.frames ? a.frames[v] : a.frame0;
}
__device__ __forceinline__ ViewDesc view_of(const PipeArgs& a, uint32_t v) { return a.frames ? a.views[v] : a.view0; }
__device__ __forceinline__ DevWorld world_of(const PipeArgs& a, const ViewDesc& vd) {
  return {a.chunks + vd.chunk_off, vd.n_chunks, a.inners, a.n_inners, a.leaves, a.n_leaves,
          a.bricks, a.n_bricks, a.grids + vd.grid_off, vd.grid_len, a.err, a.spec, a.atlas_alpha, a.atlas_layers,
          {a.tuft_layer[0], a.tuft_layer[1], a.tuft_layer[2]}};
}

// The same, resolved at compile time when the launch is known to carry one
// view (frames == nullptr): the frame, view and world then come from the
// kernel's parameter space instead of registers.
template <bool SINGLE>
__device__ __forceinline__ uint32_t find_view_t(const PipeArgs& a, uint32_t tile) { return SINGLE ? 0u : find_view(a, tile); }
template <bool SINGLE>
__device__ __forceinline__ const vm_frame& frame_t(const PipeArgs& a, uint32_t v) { return SINGLE ? a.frame0 : a.frames[v]; }
template <bool SINGLE>
__device__ __forceinline__ ViewDesc view_t(const PipeArgs& a, uint32_t v) { return SINGLE ? a.view0 : a.views[v]; }

struct MaxOp {
  __device__ __forceinline__ uint32_t operator()(uint32_t x, uint32_t y) const { return x > y ? x : y; }
};

// A hit in chunk c has t >= dmin * (1 - 1e-5) - 0.05 * vs: the box distance
// and the march's slab / DDA arithmetic differ by float rounding only, far
// below that slack.  dkmax = depth_key of that bound (depth keys fall with t).
constexpr int BOUNDS_THREADS = 256;
__device__ __forceinline__ void bounds_block(const PipeArgs& a, uint32_t v) {
  typedef cub::BlockScan<uint32_t, BOUNDS_THREADS> Scan;
  __shared__ typename Scan::TempStorage tmp;
  // the launch's counters start at zero (the prepass is its first kernel)
  if (v == 0 && threadIdx.x < (uint32_t)W_WORDS) a.work[threadIdx.x] = 0u;
  const vm_frame& f = frame_of(a, v);
  const ViewDesc vd = view_of(a, v);
  const uint32_t n = min(f.chunk_count, vd.n_chunks);
  const F3 cam = ld3(f.cam_pos);
  const uint32_t per = (n + BOUNDS_THREADS - 1) / BOUNDS_THREADS;
  // thread t owns [t*per, t*per+per); threads are taken in reverse so that an
  // exclusive max-scan gives every thread the maximum over later chunks
  const uint32_t t = BOUNDS_THREADS - 1 - threadIdx.x;
  uint32_t* dk = a.dkmax + vd.chunk_off;
  uint32_t* suf = a.sufmax + vd.chunk_off;
  uint32_t local = 0u;
  for (uint32_t k = 0; k < per; ++k) {
    const uint32_t ci = t * per + k;
    if (ci < n) {
      const vm_chunk& c = a.chunks[vd.chunk_off + ci];
      const float dmin = box_distance(cam, ld3(c.aabb_min), ld3(c.aabb_max));
      const float lb = fmaxf(dmin * (1.0f - 1e-5f) - 0.05f * c.voxel_size, 0.0f);
      const uint32_t d = depth_key(f, lb);
      dk[ci] = d;
      local = max(local, d);
    }
  }
  uint32_t run;
  Scan(tmp).ExclusiveScan(local, run, 0u, MaxOp());
  for (int k = (int)per - 1; k >= 0; --k) {
    const uint32_t ci = t * per + (uint32_t)k;
    if (ci < n) {
      run = max(run, dk[ci]);
      suf[ci] = run;
    }
  }
}

// tile_select's per-chunk test (tile_select.wgsl:59-80 without the Hi-Z
// deferral): the camera chunk always, else inside the near plane and the
// tile's four side planes and closer than the reach.
__device__ __forceinline__ bool cull_keep(const vm_frame& f, const TilePlanes& tp, F3 cam, F3 fwd,
                                          const vm_chunk* ch, uint32_t ci) {
  if (ci == f.camera_chunk) return true;
  const float* cp = reinterpret_cast<const float*>(ch + ci);
  const F3 bmin = {__ldg(cp + 0), __ldg(cp + 1), __ldg(cp + 2)};
  const F3 bmax = {__ldg(cp + 4), __ldg(cp + 5), __ldg(cp + 6)};
  if (box_outside(bmin, bmax, fwd, cam) || box_outside(bmin, bmax, tp.n[0], cam) ||
      box_outside(bmin, bmax, tp.n[1], cam) || box_outside(bmin, bmax, tp.n[2], cam) ||
      box_outside(bmin, bmax, tp.n[3], cam))
    return false;
  return box_distance(cam, bmin, bmax) < tp.reach;
}

__device__ __forceinline__ uint32_t find_view_super(const PipeArgs& a, uint32_t s) {
  if (a.frames == nullptr) return 0;
  uint32_t lo = 0, hi = a.n_views - 1;
  while (lo < hi) {
    const uint32_t mid = (lo + hi + 1) >> 1;
    if (a.views[mid].super_begin <= s) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// Coarse cull of a 32x32-pixel super-tile (4x4 of the engine's tiles): a
// chunk is dropped only when it is outside the super-tile's near plane (the
// tiles' own test), beyond far (no tile reaches further), or outside one of
// its four side planes by a margin of 1e-4 of |n| |p - cam| (far above the
// planes' rounding).  Every pixel ray of the super-tile lies inside those
// planes, so a dropped chunk can produce no hit for any of its pixels; the
// tiles then run tile_select's exact test on the survivors only.
__device__ __forceinline__ bool super_keep(const vm_frame& f, const F3* n, F3 cam, F3 fwd, const vm_chunk* ch,
                                           uint32_t ci) {
  if (ci == f.camera_chunk) return true;
  const float* cp = reinterpret_cast<const float*>(ch + ci);
  const F3 bmin = {__ldg(cp + 0), __ldg(cp + 1), __ldg(cp + 2)};
  const F3 bmax = {__ldg(cp + 4), __ldg(cp + 5), __ldg(cp + 6)};
  if (box_outside(bmin, bmax, fwd, cam)) return false;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const F3 p = {n[i].x > 0.0f ? bmax.x : bmin.x, n[i].y > 0.0f ? bmax.y : bmin.y, n[i].z > 0.0f ? bmax.z : bmin.z};
    const F3 q = p - cam;
    if (dot(n[i], q) < -1e-4f * sqrtf(dot(n[i], n[i]) * dot(q, q))) return false;
  }
  return box_distance(cam, bmin, bmax) < f.far_;
}

template <bool SINGLE>
__device__ __forceinline__ void cull_super_blocks(const PipeArgs& a, uint32_t block, uint32_t n_blocks) {
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t n_warps = n_blocks * 8u;
  for (uint32_t s = block * 8u + (threadIdx.x >> 5); s < a.total_supers; s += n_warps) {
    const uint32_t v = SINGLE ? 0u : find_view_super(a, s);
    const vm_frame& f = frame_t<SINGLE>(a, v);
    const ViewDesc vd = view_t<SINGLE>(a, v);
    const uint32_t local = s - vd.super_begin, sxv = (vd.tiles_x + 3u) >> 2;
    F3 d[5], n[4];
    square_dirs_warp(f, (local % sxv) * 32u, (local / sxv) * 32u, 32.0f, lane, d);
    side_planes(d, n);
    const F3 cam = ld3(f.cam_pos), fwd = ld3(f.cam_fwd);
    const uint32_t n_vis = min(f.chunk_count, vd.n_chunks);
    const vm_chunk* ch = a.chunks + vd.chunk_off;
    uint16_t* out = a.super_list + (uint64_t)s * a.list_cap;
    uint32_t cnt = 0;
    for (uint32_t base = 0; base < n_vis; base += 32u) {
      const uint32_t ci = base + lane;
      const bool keep = ci < n_vis && super_keep(f, n, cam, fwd, ch, ci);
      const uint32_t bal = __ballot_sync(FULLMASK, keep);
      if (keep) {
        const uint32_t pos = cnt + __popc(bal & lanemask_lt());
        if (pos < a.list_cap) out[pos] = (uint16_t)ci;
      }
      cnt += __popc(bal);
    }
    if (lane == 0) a.super_count[s] = cnt;
  }
}

// The launch's first kernel: blocks [0, n_views) compute their view's chunk
// depth bounds (and block 0 zeroes the counters), the others run the
// super-tile cull; the two are independent, one launch serves both.
template <bool SINGLE>
__global__ void __launch_bounds__(BOUNDS_THREADS) k_prepass(const __grid_constant__ PipeArgs a) {
  // k_cull, launched behind this kernel with programmatic serialization,
  // traces its tile rays while this kernel runs
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  if (blockIdx.x < a.n_views) bounds_block(a, blockIdx.x);
  else cull_super_blocks<SINGLE>(a, blockIdx.x - a.n_views, gridDim.x - a.n_views);
}

// tile_select's per-chunk test (cull_keep) on a box staged in shared memory
__device__ __forceinline__ bool cull_keep_box(const vm_frame& f, const TilePlanes& tp, F3 cam, F3 fwd, F3 bmin,
                                              F3 bmax, uint32_t ci) {
  if (ci == f.camera_chunk) return true;
  if (box_outside(bmin, bmax, fwd, cam) || box_outside(bmin, bmax, tp.n[0], cam) ||
      box_outside(bmin, bmax, tp.n[1], cam) || box_outside(bmin, bmax, tp.n[2], cam) ||
      box_outside(bmin, bmax, tp.n[3], cam))
    return false;
  return box_distance(cam, bmin, bmax) < tp.reach;
}

// cull_keep_box for a survivor of the super-tile cull (super_keep): it has
// passed the same near-plane test (box_outside with the camera's forward
// axis) and box_distance < far, so only the tile's four side planes remain,
// and the reach when the tile's is shorter than far.
__device__ __forceinline__ bool cull_keep_survivor(const vm_frame& f, const TilePlanes& tp, F3 cam, F3 bmin,
                                                   F3 bmax, uint32_t ci, bool far_reach) {
  if (ci == f.camera_chunk) return true;
  if (box_outside(bmin, bmax, tp.n[0], cam) || box_outside(bmin, bmax, tp.n[1], cam) ||
      box_outside(bmin, bmax, tp.n[2], cam) || box_outside(bmin, bmax, tp.n[3], cam))
    return false;
  return far_reach || box_distance(cam, bmin, bmax) < tp.reach;
}

// One block per 32x32 super-tile, one warp per 8x8 tile of it: the block
// stages its candidates' boxes (the super-tile's survivors, or every chunk
// when it has no list) in shared memory, CULL_BATCH at a time with coalesced
// loads, and each warp runs tile_select's exact test on them in ascending
// chunk order, so every tile gets the same list as from a warp that read
// the boxes from global memory itself.  Three blocks per SM (40 registers).
// Launched behind k_prepass with programmatic serialization: a block traces
// its tiles' rays (frame parameters only) before it waits for the prepass.
constexpr uint32_t CULL_THREADS = 512, CULL_BATCH = 256;
template <bool SINGLE>
__global__ void __launch_bounds__(CULL_THREADS, 3) k_cull(const __grid_constant__ PipeArgs a) {
  __shared__ float s_box[6][CULL_BATCH];
  __shared__ uint16_t s_ci[CULL_BATCH];
  __shared__ uint32_t s_hist[N_COST_BUCKETS];
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  const uint32_t s = blockIdx.x;
  if (threadIdx.x < N_COST_BUCKETS) s_hist[threadIdx.x] = 0u;
  const uint32_t v = SINGLE ? 0u : find_view_super(a, s);
  const vm_frame& f = frame_t<SINGLE>(a, v);
  const ViewDesc vd = view_t<SINGLE>(a, v);
  const uint32_t local_s = s - vd.super_begin, sxv = (vd.tiles_x + 3u) >> 2;
  const uint32_t tx = (local_s % sxv) * 4u + (warp & 3u), ty = (local_s / sxv) * 4u + (warp >> 2);
  const bool has_tile = tx < vd.tiles_x && ty < vd.tiles_y;
  const uint32_t t = vd.tile_begin + ty * vd.tiles_x + tx;
  TilePlanes tp;
  if (has_tile) tp = tile_planes_warp(f, tx * 8u, ty * 8u, lane);
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  asm volatile("griddepcontrol.wait;" ::: "memory");   // the prepass's lists, bounds and zeroed counters
  const F3 cam = ld3(f.cam_pos), fwd = ld3(f.cam_fwd);
  const uint32_t n_vis = min(f.chunk_count, vd.n_chunks);
  const vm_chunk* ch = a.chunks + vd.chunk_off;
  const uint32_t ns = a.super_count[s];
  const bool listed = ns <= a.list_cap;
  const uint16_t* cand = a.super_list + (uint64_t)s * a.list_cap;
  const uint32_t n_test = listed ? ns : n_vis;
  uint16_t* out = a.tile_list + (uint64_t)(has_tile ? t : 0u) * a.list_cap;
  const bool far_reach = has_tile && tp.reach == f.far_;
  uint32_t n = 0;
  for (uint32_t b0 = 0; b0 < n_test; b0 += CULL_BATCH) {
    const uint32_t nb = min(CULL_BATCH, n_test - b0);
    __syncthreads();   // the previous batch is consumed
    for (uint32_t j = threadIdx.x; j < nb; j += CULL_THREADS) {
      const uint32_t ci = listed ? (uint32_t)cand[b0 + j] : b0 + j;
      const float* cp = reinterpret_cast<const float*>(ch + ci);
      s_box[0][j] = __ldg(cp + 0); s_box[1][j] = __ldg(cp + 1); s_box[2][j] = __ldg(cp + 2);
      s_box[3][j] = __ldg(cp + 4); s_box[4][j] = __ldg(cp + 5); s_box[5][j] = __ldg(cp + 6);
      s_ci[j] = (uint16_t)ci;
    }
    __syncthreads();
    if (!has_tile) continue;
    for (uint32_t base = 0; base < nb; base += 32u) {
      const uint32_t j = base + lane;
      uint32_t ci = 0u;
      bool keep = false;
      if (j < nb) {
        ci = s_ci[j];
        const F3 bmin = f3(s_box[0][j], s_box[1][j], s_box[2][j]), bmax = f3(s_box[3][j], s_box[4][j], s_box[5][j]);
        keep = listed ? cull_keep_survivor(f, tp, cam, bmin, bmax, ci, far_reach)
                      : cull_keep_box(f, tp, cam, fwd, bmin, bmax, ci);
      }
      const uint32_t bal = __ballot_sync(FULLMASK, keep);
      if (keep) {
        const uint32_t pos = n + __popc(bal & lanemask_lt());
        if (pos < a.list_cap) out[pos] = (uint16_t)ci;
      }
      n += __popc(bal);
    }
  }
  __syncthreads();
  if (has_tile && lane == 0) {
    a.tile_count[t] = n;
    a.hiz[t] = 0xFFFFFFFFu;   // the primary kernel folds its pixels' minimum in
    const uint32_t c = max(a.item_cost[2u * t], a.item_cost[2u * t + 1u]);
    atomicAdd(&s_hist[cost_bucket(c)], 1u);
  }
  __syncthreads();
  // the block's tiles in the cost histogram: one global atomic per bucket used
  if (threadIdx.x < N_COST_BUCKETS && s_hist[threadIdx.x])
    atomicAdd(&a.work[W_HIST + threadIdx.x], s_hist[threadIdx.x]);
}

// The tiles in decreasing order of the last launch's cost (a counting sort
// over the cost buckets; ties in any order).  Each block ranks its own
// contiguous range of tiles in shared memory and reserves one range per
// bucket with a single global atomic.
constexpr uint32_t ORDER_TILES = 512;    // tiles per block
__global__ void __launch_bounds__(256) k_order(const __grid_constant__ PipeArgs a) {
  __shared__ uint32_t start[N_COST_BUCKETS], count[N_COST_BUCKETS], base[N_COST_BUCKETS];
  const uint32_t t0 = blockIdx.x * ORDER_TILES, t1 = min(t0 + ORDER_TILES, a.total_tiles);
  if (threadIdx.x < N_COST_BUCKETS) count[threadIdx.x] = 0u;
  asm volatile("griddepcontrol.wait;" ::: "memory");   // k_cull's histogram
  if (threadIdx.x == 0) {
    uint32_t s = 0;
    for (uint32_t b = 0; b < N_COST_BUCKETS; ++b) { start[b] = s; s += a.work[W_HIST + b]; }
  }
  __syncthreads();
  uint32_t bk[ORDER_TILES / 256], rank[ORDER_TILES / 256];
#pragma unroll
  for (uint32_t k = 0; k < ORDER_TILES / 256; ++k) {
    const uint32_t t = t0 + k * 256u + threadIdx.x;
    bk[k] = N_COST_BUCKETS;
    if (t < t1) {
      bk[k] = cost_bucket(max(a.item_cost[2u * t], a.item_cost[2u * t + 1u]));
      rank[k] = atomicAdd(&count[bk[k]], 1u);
    }
  }
  __syncthreads();
  if (threadIdx.x < N_COST_BUCKETS)
    base[threadIdx.x] = count[threadIdx.x] ? atomicAdd(&a.work[W_FILL + threadIdx.x], count[threadIdx.x]) : 0u;
  __syncthreads();
#pragma unroll
  for (uint32_t k = 0; k < ORDER_TILES / 256; ++k)
    if (bk[k] < N_COST_BUCKETS) a.tile_order[start[bk[k]] + base[bk[k]] + rank[k]] = t0 + k * 256u + threadIdx.x;
}

// stage: 0 primary, 1 shadow, 2 secondary (a.traffic holds one record per stage)
template <bool COUNT>
__device__ __forceinline__ void flush_traffic(const PipeArgs& a, int stage, const Traffic& tr, uint32_t np,
                                              uint32_t ns, uint32_t nx) {
  if (!COUNT) return;
  unsigned long long v[11] = {tr.chunk, tr.l1, tr.leaf, tr.attr, tr.pal, tr.grid, tr.iters, np, ns, nx, tr.entries};
  unsigned long long* dst = reinterpret_cast<unsigned long long*>(a.traffic + stage);
#pragma unroll
  for (int i = 0; i < 11; ++i) {
    unsigned long long x = v[i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(FULLMASK, x, o);
    if ((threadIdx.x & 31u) == 0 && x) atomicAdd(dst + i, x);
  }
}

// One lane, one pixel, one chunk: march it and fold the key into the pixel's
// best (the engine's atomicMax), keeping the best hit's block id.
template <bool UNDERWATER, bool COUNT, bool TUFTS>
__device__ __forceinline__ void march_entry(const DevWorld& w, const vm_frame& f, const Ray& ray, uint32_t ci,
                                            uint32_t px, uint32_t py, unsigned long long& best, uint32_t& best_id,
                                            Traffic* tr) {
  if (COUNT) tr->entries++;
  const Chunk c = ld_chunk(w, ci);
  if (ray_skips(f, c.fade, px, py)) return;
  // The march may stop at a distance T whose depth key is already below the
  // pixel's best: depth_key falls monotonically with t and the march reports
  // no hit at or beyond its limit, so every hit it skips has a smaller key.
  // T is checked here, not assumed; without a best key the limit is far.
  float t_lim = f.far_;
  const uint32_t bestd = (uint32_t)(best >> 40);
  if (bestd >= 3u) {
    const float t_cut = f.far_ * (1.0f - (float)(bestd - 3u) * (1.0f / 16777215.0f));
    if (t_cut < f.far_ && depth_key(f, t_cut) < bestd) t_lim = t_cut;
  }
  // With the Snell bend a miss of the straight march (over its full length,
  // as the engine marches it) is what lets the bent ray count, so the
  // distance limit is not applied to it.
  const bool bend = UNDERWATER && (w.spec & VM_SPEC_SNELL_BEND) != 0u;
  Hit h = march_chunk<UNDERWATER, false, false, COUNT, true, TUFTS>(w, f, c, ray, bend ? f.far_ : t_lim, tr);
  if (bend && !h.hit) snell_bend<COUNT, true, TUFTS>(w, f, c, ray.d, &h, tr);
  if (h.hit) {
    const unsigned long long k = make_key(f, h, ci);
    if (k > best) { best = k; best_id = h.id; }
  }
}

// The rest of tile_select's scan when a tile's list overflowed its capacity:
// 32 chunks culled per step across the warp, each survivor marched in order.
// Cold code, kept out of the primary loop's instruction stream.
template <bool UNDERWATER, bool COUNT, bool TUFTS>
__device__ __noinline__ void march_overflow(const DevWorld w, const vm_frame& f, const Ray ray, uint32_t start,
                                            uint32_t tx, uint32_t ty, uint32_t px, uint32_t py,
                                            const uint32_t* dk, const uint32_t* suf, bool active,
                                            unsigned long long* best, uint32_t* best_id, Traffic* tr) {
  const uint32_t lane = threadIdx.x & 31u;
  const TilePlanes tp = tile_planes(f, tx * 8u, ty * 8u);
  const F3 fwd = ld3(f.cam_fwd);
  const uint32_t n_vis = min(f.chunk_count, w.n_chunks);
  unsigned long long b = *best;
  uint32_t id = *best_id;
  for (uint32_t base = start; base < n_vis; base += 32u) {
    const uint32_t ci = base + lane;
    uint32_t bal = __ballot_sync(FULLMASK, ci < n_vis && cull_keep(f, tp, ray.o, fwd, w.chunks, ci));
    while (bal) {
      const uint32_t cj = base + (uint32_t)(__ffs(bal) - 1);
      bal &= bal - 1u;
      if (!active) continue;
      const uint32_t bestd = (uint32_t)(b >> 40);
      if (suf[cj] < bestd) { active = false; continue; }
      if (dk[cj] < bestd) continue;
      march_entry<UNDERWATER, COUNT, TUFTS>(w, f, ray, cj, px, py, b, id, tr);
    }
  }
  *best = b;
  *best_id = id;
}

// The reflect leg of a water hit (key: the pixel's key if it hit water, else
// 0) queued for k_secondary_q, and the zero key of the pixels without one.
// The ray direction, hit_t and hit point are recomputed here by the same
// float operations as in k_primary (same values), and the code is out of
// line, so the primary kernel's register allocation stays that of frames
// without reflect legs.  Called by the whole warp.
template <bool TUFTS>
__device__ __noinline__ void enqueue_reflect(const PipeArgs& a, uint32_t v, uint32_t px, uint32_t py, uint64_t pix,
                                             bool valid, unsigned long long key) {
  const vm_frame& f = frame_of(a, v);
  bool want = false;
  SecRay rr;
  if (key != 0ull) {
    const KeyParts k = split_key(key);
    const Chunk c = ld_chunk(world_of(a, view_of(a, v)), k.ci);
    const F3 rd = ray_dir(f, (float)px + 0.5f, (float)py + 0.5f);
    const float th = hit_t(f, c, k.vx, k.vy, k.vz, k.mx, k.my, k.mz, k.nid, rd);
    if (water_reflects(f, th)) {
      rr = reflect_ray<false, TUFTS>(world_of(a, view_of(a, v)), f, ld3(f.cam_pos) + rd * th, rd, k.nid, th, nullptr);
      want = true;
    }
  }
  if (valid && !want) { a.refl_key[pix] = 0ull; a.refl_t[pix] = 0.0f; }
  const uint32_t bal = __ballot_sync(FULLMASK, want);
  if (!bal) return;
  uint32_t b0 = 0;
  if ((threadIdx.x & 31u) == 0) b0 = atomicAdd(&a.work[W_SEC_N], __popc(bal));
  b0 = __shfl_sync(FULLMASK, b0, 0);
  if (want) {
    SecItem& q = a.sec_q[b0 + __popc(bal & lanemask_lt())];
    q.view = v; q.pix = py * f.res[0] + px;
    q.o[0] = rr.o.x; q.o[1] = rr.o.y; q.o[2] = rr.o.z;
    q.d[0] = rr.d.x; q.d[1] = rr.d.y; q.d[2] = rr.d.z;
    q.max_dist = rr.max_dist; q.kind = SEC_REFLECT;
  }
}

// MINB: blocks per SM the register allocation must allow (1: unconstrained),
// the autotuner's occupancy knob.
// REFL: the frame may trace reflect legs (a.do_reflect); without it the
// kernel carries none of that code.  SINGLE: the launch has one view.
// PX: pixels per lane (the packet).  A warp's item is 8 x 4 PX pixels of one
// 8x8 tile: PX = 1 half a tile, PX = 2 the whole tile.  A lane walks its PX
// pixels one after the other and starts its next pixel as soon as one is
// done, so lanes whose rays end early do not idle until the warp's slowest
// ray ends; the pixels' results are then finished together.
// TUFTS: the chunks hold foliage tufts and the context has the atlas: the
// march traces their cross quads (a generic shape, selected per frame).
template <int NW, int MINB, bool UNDERWATER, bool COUNT, bool REFL, bool SINGLE, int PX, bool TUFTS = false>
__global__ void __launch_bounds__(NW * 32, MINB) k_primary(const __grid_constant__ PipeArgs a) {
  static_assert(PX == 1 || PX == 2, "one or two pixels per lane");
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t total = a.total_tiles * (2u / PX);
  // Every lane walks the same tile list: the warp stages the item's first 32
  // entries and their depth bounds in shared memory with one load per lane,
  // so a lane's walk reads them there instead of chaining a list load, a
  // bounds load and only then the chunk record through global memory.
  __shared__ uint32_t s_ci[NW][32], s_dk[NW][32], s_suf[NW][32];
  uint32_t* my_ci = s_ci[threadIdx.x >> 5];
  uint32_t* my_dk = s_dk[threadIdx.x >> 5];
  uint32_t* my_suf = s_suf[threadIdx.x >> 5];
  Traffic tr = {};
  uint32_t np = 0, ns = 0, nx = 0;
  for (;;) {
    uint32_t item = 0;
    if (lane == 0) item = atomicAdd(&a.work[W_PRIMARY], 1u);
    item = __shfl_sync(FULLMASK, item, 0);
    if (item >= total) break;
    const long long clk0 = clock64();
    const uint32_t t = PX == 1 ? a.tile_order[item >> 1] : a.tile_order[item];
    const uint32_t half0 = PX == 1 ? (item & 1u) : 0u;
    const uint32_t v = find_view_t<SINGLE>(a, t);
    const vm_frame& f = frame_t<SINGLE>(a, v);
    const ViewDesc vd = view_t<SINGLE>(a, v);
    const DevWorld w = world_of(a, vd);
    const uint32_t local = t - vd.tile_begin;
    const uint32_t tx = local % vd.tiles_x, ty = local / vd.tiles_x;
    const uint32_t px = tx * 8u + (lane & 7u), py0 = ty * 8u + half0 * 4u + (lane >> 3);
    const uint32_t n = a.tile_count[t];
    const uint32_t m = min(n, a.list_cap);
    const uint16_t* list = a.tile_list + (uint64_t)t * a.list_cap;
    const uint32_t* dk = a.dkmax + vd.chunk_off;
    const uint32_t* suf = a.sufmax + vd.chunk_off;
    __syncwarp();   // the previous item's reads of the staged entries are done
    if (lane < m) {
      const uint32_t c0 = list[lane];
      my_ci[lane] = c0; my_dk[lane] = dk[c0]; my_suf[lane] = suf[c0];
    }
    __syncwarp();
    const F3 cam = ld3(f.cam_pos);
    // the lane's current pixel (slot k of its PX) and its walk
    uint32_t k = 0, py = py0, i = 0;
    bool valid = px < f.res[0] && py < f.res[1];
    F3 rd = ray_dir(f, (float)px + 0.5f, (float)py + 0.5f);
    Ray ray = make_ray(cam, rd);
    unsigned long long best = 0ull;
    uint32_t best_id = 0u;
    bool active = valid;
    // slot 0's result once the lane has moved on to slot 1 (PX == 2)
    unsigned long long best0 = 0ull;
    uint32_t best_id0 = 0u;
    bool active0 = false;
    // Each lane walks its list in order with the same tests as ever; the
    // entries a lane skips (a closer key already found) are passed in an
    // inner loop, so that every round of the warp is one chunk march for
    // each lane that still has one.
    for (;;) {
      uint32_t ci = 0;
      bool go = false;
      for (;;) {
        while (active && i < m) {
          uint32_t sv, dv;
          if (i < 32u) { ci = my_ci[i]; sv = my_suf[i]; dv = my_dk[i]; }
          else { ci = list[i]; sv = suf[ci]; dv = dk[ci]; }
          const uint32_t bestd = (uint32_t)(best >> 40);
          if (sv < bestd) { active = false; break; }
          ++i;
          if (dv < bestd) continue;
          go = true;
          break;
        }
        if (go || PX == 1 || k + 1u >= (uint32_t)PX) break;
        // this pixel's walk is over: keep its result, start the next pixel
        best0 = best; best_id0 = best_id; active0 = active;
        ++k;
        py += 4u;
        valid = px < f.res[0] && py < f.res[1];
        rd = ray_dir(f, (float)px + 0.5f, (float)py + 0.5f);
        ray = make_ray(cam, rd);
        best = 0ull; best_id = 0u; active = valid; i = 0;
      }
      if (!__any_sync(FULLMASK, go)) break;
      if (go) march_entry<UNDERWATER, COUNT, TUFTS>(w, f, ray, ci, px, py, best, best_id, &tr);
    }
#pragma unroll
    for (uint32_t slot = 0; slot < (uint32_t)PX; ++slot) {
    // finish the lane's pixel of this slot (the last one's walk state is live)
    const bool last = slot + 1u == (uint32_t)PX;
    unsigned long long pbest = last ? best : best0;
    uint32_t pbest_id = last ? best_id : best_id0;
    const bool pactive = last ? active : active0;
    const uint32_t ppy = py0 + 4u * slot;
    const bool pvalid = px < f.res[0] && ppy < f.res[1];
    const F3 prd = last ? rd : ray_dir(f, (float)px + 0.5f, (float)ppy + 0.5f);
    if (n > a.list_cap)
      march_overflow<UNDERWATER, COUNT, TUFTS>(w, f, last ? ray : make_ray(cam, prd), (uint32_t)list[a.list_cap - 1] + 1u,
                                        tx, ty, px, ppy, dk, suf, pactive, &pbest, &pbest_id, &tr);
    const uint64_t pix = (uint64_t)ppy * f.res[0] + px;
    if (pvalid) a.vis[vd.pix_off + pix] = pbest;
    if (COUNT && pvalid) ++np;
    {
      // build_hiz (march.wgsl:57-76) on the final visibility: pixels outside
      // the frame count as misses
      const uint32_t d = __reduce_min_sync(FULLMASK, pvalid ? (uint32_t)(pbest >> 40) : 0u);
      if (lane == 0) atomicMin(&a.hiz[vd.tile_begin + local], d);
    }
    // The hit shared by shadow_guide (shadow.wgsl:8-30) and the water / glass
    // legs (resolve.wgsl:1029-1042,1261-1280): hit_t of the key and its point.
    bool want_sh = false, want_sec = false;
    F3 so = {0.0f, 0.0f, 0.0f};
    SecRay sr;

    if (pvalid && pbest != 0ull) {
      const KeyParts k = split_key(pbest);
      const Chunk c = ld_chunk(w, k.ci);
      const float th = hit_t(f, c, k.vx, k.vy, k.vz, k.mx, k.my, k.mz, k.nid, prd);
      const F3 hit = cam + prd * th;
      const bool water = pbest_id == VM_WATER, glass = is_glass_leg(a.spec, pbest_id);
      if (a.do_shadow && shadow_active(f) && !water && !glass) {
        F3 nrm = normal_of(k.nid);
        if (k.nid >= VM_NORMAL_CROSS_A && dot(nrm, prd) > 0.0f) nrm = neg(nrm);
        if (!(dot(nrm, ld3(f.sun_dir)) <= 0.0f) && th >= 0.0f) {
          so = hit + nrm * (0.02f * c.vs);
          want_sh = true;
        }
      }
      if (a.do_secondary && water) {
        const float detail = 1.0f - smoothstep(VM_WATER_REFRACT_NEAR, VM_WATER_REFRACT_FAR, th);
        if ((f.flags & VM_FLAG_WATER_REFRACT) != 0u && detail > 0.0f) {
          const F3 rdir = refract(prd, normal_of(k.nid), 1.0f / VM_WATER_IOR);
          sr.o = hit + rdir * VM_SURFACE_EPS;
          sr.d = rdir;
          sr.max_dist = VM_WATER_REFRACT_DIST;
          sr.water = true;
          want_sec = true;
        }
      } else if (a.do_secondary && glass) {
        sr.o = hit + prd * VM_SURFACE_EPS;
        sr.d = prd;
        sr.max_dist = fmaxf(VM_GLASS_TRANSMIT_DIST, f.far_);
        sr.water = false;
        want_sec = true;
      }
    }
    if (a.do_shadow) {
      if (pvalid && !want_sh) a.shadow[vd.pix_off + pix] = 0.0f;
      const uint32_t bal = __ballot_sync(FULLMASK, want_sh);
      if (bal) {
        uint32_t b0 = 0;
        if (lane == 0) b0 = atomicAdd(&a.work[W_SHADOW_N], __popc(bal));
        b0 = __shfl_sync(FULLMASK, b0, 0);
        if (want_sh) {
          ShadowItem& q = a.shadow_q[b0 + __popc(bal & lanemask_lt())];
          q.view = v; q.pix = (uint32_t)pix; q.o[0] = so.x; q.o[1] = so.y; q.o[2] = so.z;
        }
      }
    }
    if (a.do_secondary) {
      if (pvalid && !want_sec) { a.sec_key[vd.pix_off + pix] = 0ull; a.sec_t[vd.pix_off + pix] = 0.0f; }
      const uint32_t bal = __ballot_sync(FULLMASK, want_sec);
      if (bal) {
        uint32_t b0 = 0;
        if (lane == 0) b0 = atomicAdd(&a.work[W_SEC_N], __popc(bal));
        b0 = __shfl_sync(FULLMASK, b0, 0);
        if (want_sec) {
          SecItem& q = a.sec_q[b0 + __popc(bal & lanemask_lt())];
          q.view = v; q.pix = (uint32_t)pix;
          q.o[0] = sr.o.x; q.o[1] = sr.o.y; q.o[2] = sr.o.z;
          q.d[0] = sr.d.x; q.d[1] = sr.d.y; q.d[2] = sr.d.z;
          q.max_dist = sr.max_dist; q.kind = sr.water ? SEC_REFRACT : SEC_GLASS;
        }
      }
    }
    if (REFL && a.do_reflect)
      enqueue_reflect<TUFTS>(a, v, px, ppy, vd.pix_off + pix, pvalid, pvalid && pbest_id == VM_WATER ? pbest : 0ull);
    }
    if (lane == 0) {
      const uint32_t cost = (uint32_t)min(clock64() - clk0, 0xFFFFFFFFll);
      if (PX == 1) a.item_cost[2u * t + half0] = cost;
      else a.item_cost[2u * t] = a.item_cost[2u * t + 1u] = cost;
    }
  }
  flush_traffic<COUNT>(a, 0, tr, np, ns, nx);
}

// The sun shadow rays (shadow_ray_t, common.wgsl:1156-1195) of the queue.
// Persistent lanes: each holds one ray and steps it one chunk-grid cell at a
// time; a lane whose ray is over takes the next ray of the queue at once
// (warp-aggregated), so a warp never idles behind its longest ray.  With soft
// shadows a queue item is VM_SOFT_SAMPLES jittered rays from the same origin,
// walked one after the other by the lane; the pixel gets the blocked fraction.
template <bool COUNT, bool SINGLE>
__global__ void __launch_bounds__(256, 4) k_shadow(const __grid_constant__ PipeArgs a) {
  const uint32_t n = a.work[W_SHADOW_N];
  const uint32_t lane = threadIdx.x & 31u;
  Traffic tr = {};
  uint32_t ns = 0;
  bool has = false, drained = false;
  uint32_t view = 0u, pix = 0u, sample = 0u, blocked = 0u;
  F3 origin = {0.0f, 0.0f, 0.0f};
  ShadowWalk s;
  for (;;) {
    const uint32_t need = __ballot_sync(FULLMASK, !has);
    if (need && !drained) {
      uint32_t base = 0;
      if (lane == 0) base = atomicAdd(&a.work[W_SHADOW_TAKE], __popc(need));
      base = __shfl_sync(FULLMASK, base, 0);
      drained = base + __popc(need) >= n;
      if (!has) {
        const uint32_t i = base + __popc(need & lanemask_lt());
        if (i < n) {
          const ShadowItem q = a.shadow_q[i];
          view = q.view;
          pix = q.pix;
          origin = f3(q.o[0], q.o[1], q.o[2]);
          sample = 0u;
          blocked = 0u;
          const vm_frame& f = frame_t<SINGLE>(a, view);
          s = shadow_walk_begin(origin, soft_shadows(a.spec) ? soft_sun_dir(f, pix % f.res[0], pix / f.res[0], 0u)
                                                        : ld3(f.sun_dir));
          has = true;
          if (COUNT) ++ns;
        }
      }
    }
    if (__ballot_sync(FULLMASK, has) == 0u) break;
    if (has) {
      const vm_frame& f = frame_t<SINGLE>(a, view);
      const ViewDesc vd = view_t<SINGLE>(a, view);
      const DevWorld w = world_of(a, vd);
      float b;
      if (shadow_walk_step<COUNT>(w, f, s, f.shadow_dist, &b, &tr)) {
        if (!soft_shadows(a.spec)) {
          a.shadow[vd.pix_off + pix] = blocker_distance(b);
          has = false;
        } else {
          blocked += b >= 0.0f ? 1u : 0u;
          if (++sample < VM_SOFT_SAMPLES) {
            s = shadow_walk_begin(origin, soft_sun_dir(f, pix % f.res[0], pix / f.res[0], sample));
            if (COUNT) ++ns;
          } else {
            a.shadow[vd.pix_off + pix] = (float)blocked * (1.0f / (float)VM_SOFT_SAMPLES);
            has = false;
          }
        }
      }
    }
  }
  flush_traffic<COUNT>(a, 1, tr, 0, ns, 0);
  // When launched behind k_secondary_q with programmatic serialization, the
  // kernel ends only once that grid has completed and its writes are
  // visible, so whatever follows in the stream sees both kernels' outputs.
  // That grid waits on nothing and all its blocks were running before this
  // kernel could start; in an ordinary launch this returns at once.
  asm volatile("griddepcontrol.wait;" ::: "memory");
}

// The water / glass rays (trace_world, common.wgsl:1205-1253) of the queue —
// refract and reflect legs of water hits, transmission through glass — on
// persistent lanes like k_shadow: one chunk-grid cell per step, the next ray
// taken as soon as a lane's ray ends.
template <bool COUNT, bool SINGLE, bool TUFTS = false>
__global__ void __launch_bounds__(256, 4) k_secondary_q(const __grid_constant__ PipeArgs a) {
  // a shadow kernel launched after this one with programmatic serialization
  // may take the SMs this kernel's blocks leave (it reads nothing this kernel
  // writes); without one this has no effect
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  const uint32_t n = a.work[W_SEC_N];
  const uint32_t lane = threadIdx.x & 31u;
  Traffic tr = {};
  uint32_t nx = 0;
  bool has = false, drained = false, water = false;
  uint32_t view = 0u, pix = 0u, kind = SEC_GLASS;
  float max_dist = 0.0f;
  WorldWalk s;
  for (;;) {
    const uint32_t need = __ballot_sync(FULLMASK, !has);
    if (need && !drained) {
      uint32_t base = 0;
      if (lane == 0) base = atomicAdd(&a.work[W_SEC_TAKE], __popc(need));
      base = __shfl_sync(FULLMASK, base, 0);
      drained = base + __popc(need) >= n;
      if (!has) {
        const uint32_t i = base + __popc(need & lanemask_lt());
        if (i < n) {
          const SecItem q = a.sec_q[i];
          view = q.view;
          pix = q.pix;
          max_dist = q.max_dist;
          kind = q.kind;
          water = kind != SEC_GLASS;
          s = world_walk_begin(f3(q.o[0], q.o[1], q.o[2]), f3(q.d[0], q.d[1], q.d[2]));
          has = true;
          if (COUNT) ++nx;
        }
      }
    }
    if (__ballot_sync(FULLMASK, has) == 0u) break;
    if (has) {
      const vm_frame& f = frame_t<SINGLE>(a, view);
      const ViewDesc vd = view_t<SINGLE>(a, view);
      const DevWorld w = world_of(a, vd);
      WorldHit h;
      const bool over = water ? world_walk_step<true, COUNT, TUFTS>(w, f, s, max_dist, &h, &tr)
                              : world_walk_step<false, COUNT, TUFTS>(w, f, s, max_dist, &h, &tr);
      if (over) {
        // the key of secondary_trace: traced, glass, hit and the hit's fields
        unsigned long long k = (1ull << 63) | (water ? 0ull : (1ull << 61));
        if (h.hit)
          k |= (1ull << 62) | ((unsigned long long)h.normal << 37) | ((unsigned long long)h.ci << 24) |
               (unsigned long long)((h.vx << 16) | (h.vy << 8) | h.vz);
        if (kind == SEC_REFLECT) {
          a.refl_key[vd.pix_off + pix] = k;
          a.refl_t[vd.pix_off + pix] = h.t;
        } else {
          a.sec_key[vd.pix_off + pix] = k;
          a.sec_t[vd.pix_off + pix] = h.t;
        }
        has = false;
      }
    }
  }
  flush_traffic<COUNT>(a, 2, tr, 0, 0, nx);
}

// ---------------------------------------------------------------------------
// Register levels: the resident warps per SM the allocation must allow.
// 0 unconstrained, 1 24 warps (~80 registers), 2 32 warps (64 registers),
// 3 20 warps (~100 registers), 4 16 warps (128 registers).
template <int NW, int LEVEL>
struct MinBlocks {
  static constexpr int warps = LEVEL == 1 ? 24 : (LEVEL == 2 ? 32 : (LEVEL == 3 ? 20 : 16));
  static constexpr int value = LEVEL == 0 ? 1 : warps / NW;
};

template <int NW, int LEVEL, bool UW, int PX>
static void* primary_fn(bool refl, bool single) {
  constexpr int MB = MinBlocks<NW, LEVEL>::value;
  if (!single) return (void*)k_primary<NW, MB, UW, false, false, false, PX>;   // batches trace no reflect legs
  return refl ? (void*)k_primary<NW, MB, UW, false, true, true, PX> : (void*)k_primary<NW, MB, UW, false, false, true, PX>;
}

template <int NW, int PX>
static void* primary_nw(int level, bool uw, bool refl, bool single) {
  switch (level) {
    case 0: return uw ? primary_fn<NW, 0, true, PX>(refl, single) : primary_fn<NW, 0, false, PX>(refl, single);
    case 1: return uw ? primary_fn<NW, 1, true, PX>(refl, single) : primary_fn<NW, 1, false, PX>(refl, single);
    case 2: return uw ? primary_fn<NW, 2, true, PX>(refl, single) : primary_fn<NW, 2, false, PX>(refl, single);
    case 3: return uw ? primary_fn<NW, 3, true, PX>(refl, single) : primary_fn<NW, 3, false, PX>(refl, single);
    case 4: return uw ? primary_fn<NW, 4, true, PX>(refl, single) : primary_fn<NW, 4, false, PX>(refl, single);
  }
  return nullptr;
}

// the counting run is never timed: 4 warps, unconstrained registers, one
// pixel per lane, the reflect code behind its runtime flag, tufts traced
static void* primary_count(bool uw, bool single) {
  if (single)
    return uw ? (void*)k_primary<4, 1, true, true, true, true, 1, true>
              : (void*)k_primary<4, 1, false, true, true, true, 1, true>;
  return uw ? (void*)k_primary<4, 1, true, true, false, false, 1, true>
            : (void*)k_primary<4, 1, false, true, false, false, 1, true>;
}

// frames with tufts: one generic shape (4 warps, unconstrained registers, one
// pixel per lane), the tuned shapes stay free of the cross-quad code
static void* primary_tufts(bool uw, bool refl, bool single) {
  if (!single)
    return uw ? (void*)k_primary<4, 1, true, false, false, false, 1, true>
              : (void*)k_primary<4, 1, false, false, false, false, 1, true>;
  if (refl)
    return uw ? (void*)k_primary<4, 1, true, false, true, true, 1, true>
              : (void*)k_primary<4, 1, false, false, true, true, 1, true>;
  return uw ? (void*)k_primary<4, 1, true, false, false, true, 1, true>
            : (void*)k_primary<4, 1, false, false, false, true, 1, true>;
}

static void* primary_kernel(const PipeTuning& t, bool uw, bool cnt, bool refl, bool single, bool tufts) {
  if (cnt) return primary_count(uw, single);
  if (tufts) return primary_tufts(uw, refl, single);
  const int px = t.px_per_lane == 2 ? 2 : 1;
  switch (t.primary_warps * 4 + px) {
    case 4 * 4 + 1: return primary_nw<4, 1>(t.reg_level, uw, refl, single);
    case 4 * 4 + 2: return primary_nw<4, 2>(t.reg_level, uw, refl, single);
    case 8 * 4 + 1: return primary_nw<8, 1>(t.reg_level, uw, refl, single);
    case 8 * 4 + 2: return primary_nw<8, 2>(t.reg_level, uw, refl, single);
  }
  return nullptr;
}

// pixels per lane of the primary kernel a launch runs (cnt: the counting or
// the tuft kernel, whose shape is fixed)
static int packet_of(const PipeTuning& t, bool cnt) { return cnt ? 1 : (t.px_per_lane == 2 ? 2 : 1); }

static int block_warps(const PipeTuning& t, bool cnt) { return cnt ? 4 : t.primary_warps; }

int primary_max_ctas_per_sm(const PipeTuning& t, bool underwater, bool count, bool reflect, bool single, bool tufts) {
  void* fn = primary_kernel(t, underwater, count, reflect, single, tufts);
  if (!fn) return 0;
  int n = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, block_warps(t, count || tufts) * 32, 0);
  return n;
}

namespace {

// A launch with programmatic stream serialization: the kernel may start once
// every block of the kernel before it in the stream has started (or run
// griddepcontrol.launch_dependents); it waits for that kernel's results with
// griddepcontrol.wait.
template <typename K>
cudaError_t launch_after(K kernel, uint32_t blocks, uint32_t threads, cudaStream_t s, const PipeArgs& a) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(blocks);
  cfg.blockDim = dim3(threads);
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, a);
}

}  // namespace

cudaError_t launch_pipeline(const PipeArgs& a, const PipeTuning& t, bool underwater, bool count, int sms,
                            cudaStream_t s, const cudaEvent_t* ev) {
  cudaError_t e;
  const auto mark = [&](int i) { return ev ? cudaEventRecord(ev[i], s) : cudaSuccess; };
  if ((e = mark(0)) != cudaSuccess) return e;
  if (a.total_tiles == 0) {
    if ((e = cudaMemsetAsync(a.work, 0, W_WORDS * sizeof(uint32_t), s)) != cudaSuccess) return e;
    for (int i = 1; i < 5; ++i)
      if ((e = mark(i)) != cudaSuccess) return e;
    return cudaSuccess;
  }

  const uint32_t super_blocks = std::min<uint32_t>((a.total_supers + 7) / 8, (uint32_t)sms * 16u);
  // k_cull and k_order with programmatic serialization: each starts once the
  // kernel before it has started all its blocks and waits for its results
  // (griddepcontrol.wait), so the launches' latency and k_cull's ray setup
  // overlap the kernel before
  if (a.frames == nullptr) {
    k_prepass<true><<<a.n_views + super_blocks, BOUNDS_THREADS, 0, s>>>(a);
    e = launch_after(k_cull<true>, a.total_supers, CULL_THREADS, s, a);
  } else {
    k_prepass<false><<<a.n_views + super_blocks, BOUNDS_THREADS, 0, s>>>(a);
    e = launch_after(k_cull<false>, a.total_supers, CULL_THREADS, s, a);
  }
  if (e != cudaSuccess) return e;
  if ((e = launch_after(k_order, (a.total_tiles + ORDER_TILES - 1) / ORDER_TILES, 256u, s, a)) != cudaSuccess)
    return e;
  if ((e = mark(1)) != cudaSuccess) return e;
  const bool refl = a.do_reflect != 0u, single = a.frames == nullptr, tufts = a.tufts != 0u;
  void* fn = primary_kernel(t, underwater, count, refl, single, tufts);
  if (!fn) return cudaErrorInvalidValue;
  const bool fixed = count || tufts;   // a shape the tuning does not choose
  const int nw = block_warps(t, fixed);
  int per = t.ctas_per_sm > 0 && !fixed ? t.ctas_per_sm
                                        : primary_max_ctas_per_sm(t, underwater, count, refl, single, tufts);
  if (per <= 0) per = 1;
  const uint32_t items_blocks = (a.total_tiles * (2u / (uint32_t)packet_of(t, fixed)) + nw - 1) / nw;
  const uint32_t grid = std::min<uint32_t>((uint32_t)sms * (uint32_t)per, items_blocks);
  void* args[] = {(void*)&a};
  if ((e = cudaLaunchKernel(fn, dim3(grid), dim3(nw * 32), args, 0, s)) != cudaSuccess) return e;
  if ((e = mark(2)) != cudaSuccess) return e;
  const uint32_t q_blocks = (uint32_t)sms * 8u;
  if (!count && single && a.do_shadow && a.do_secondary) {
    // The water / glass rays first, on exactly the blocks that fit at once
    // (4 per SM), then the shadow rays with programmatic stream serialization:
    // the shadow kernel needs only the primary kernel's queue, complete
    // before either starts, so its blocks take the SMs the few long water /
    // glass walks leave instead of waiting for the last of them.  Events 3
    // and 4 both follow the two kernels.
    if (tufts) k_secondary_q<false, true, true><<<(uint32_t)sms * 4u, 256, 0, s>>>(a);
    else k_secondary_q<false, true><<<(uint32_t)sms * 4u, 256, 0, s>>>(a);
    if ((e = launch_after(k_shadow<false, true>, q_blocks, 256u, s, a)) != cudaSuccess) return e;
    if ((e = mark(3)) != cudaSuccess) return e;
    if ((e = mark(4)) != cudaSuccess) return e;
    return cudaGetLastError();
  }
  if (a.do_shadow) {
    if (count && single) k_shadow<true, true><<<q_blocks, 256, 0, s>>>(a);
    else if (count) k_shadow<true, false><<<q_blocks, 256, 0, s>>>(a);
    else if (single) k_shadow<false, true><<<q_blocks, 256, 0, s>>>(a);
    else k_shadow<false, false><<<q_blocks, 256, 0, s>>>(a);
  }
  if ((e = mark(3)) != cudaSuccess) return e;
  if (a.do_secondary) {
    if (count && single) k_secondary_q<true, true, true><<<q_blocks, 256, 0, s>>>(a);
    else if (count) k_secondary_q<true, false, true><<<q_blocks, 256, 0, s>>>(a);
    else if (single && tufts) k_secondary_q<false, true, true><<<q_blocks, 256, 0, s>>>(a);
    else if (single) k_secondary_q<false, true><<<q_blocks, 256, 0, s>>>(a);
    else if (tufts) k_secondary_q<false, false, true><<<q_blocks, 256, 0, s>>>(a);
    else k_secondary_q<false, false><<<q_blocks, 256, 0, s>>>(a);
  }
  if ((e = mark(4)) != cudaSuccess) return e;
  return cudaGetLastError();
}

}  // namespace vmk
