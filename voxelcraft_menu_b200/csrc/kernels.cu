// March kernels for sm_100a.
//
// Two ways to produce the same visibility buffer:
//
//  * the engine's own pass sequence (src/render/mod.rs:1738-1794), one kernel
//    per WGSL entry point: tile_select -> finalize -> march (one 64-thread
//    group per (tile, chunk) pair, atomicMax into vis) -> build_hiz ->
//    recover_select -> finalize_recover -> march; then primary_shadow and the
//    water / glass secondary rays.  Same buffers, same counters.
//
//  * a fused, persistent, work-stealing kernel: one CTA per screen tile does
//    the 8x8-tile culling of every chunk into a shared-memory list ordered
//    front to back, marches each pixel through that list with an exact early
//    out (a chunk is skipped once no hit in it can reach the pixel's current
//    key), then traces the pixel's shadow ray and its water / glass ray from
//    compacted queues.  The early out only skips chunks whose best possible
//    key is below the pixel's current key, so the result equals the pair
//    sequence's atomicMax fold bit for bit.
#include "kernels.cuh"
#include <cub/block/block_scan.cuh>
#include <algorithm>

namespace vmk {
using namespace vmd;

#define FULLMASK 0xFFFFFFFFu

__device__ __forceinline__ uint32_t lanemask_lt() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

__device__ __forceinline__ bool shadow_active(const vm_frame& f) {   // shadow.wgsl:31-33
  return (f.flags & VM_FLAG_SHADOWS) != 0u && (f.flags & VM_FLAG_HEATMAP) == 0u && f.daylight > 0.01f;
}

struct KeyParts { uint32_t ci, vx, vy, vz, mx, my, mz, nid; };
__device__ __forceinline__ KeyParts split_key(unsigned long long key) {
  KeyParts k;
  const uint32_t low = (uint32_t)(key & 0xFFFFFFull);
  k.ci = (uint32_t)(key >> 24) & 0x1FFFu;
  k.vx = (low >> 16) & 63u; k.vy = (low >> 8) & 63u; k.vz = low & 63u;
  k.mx = (low >> 22) & 3u; k.my = (low >> 14) & 3u; k.mz = (low >> 6) & 3u;
  k.nid = (uint32_t)(key >> 37) & 7u;
  return k;
}

// shadow_guide (shadow.wgsl:8-30): the sun ray's origin for a visible pixel,
// or false when the pixel casts no shadow ray.
__device__ __forceinline__ bool shadow_setup(const DevWorld& w, const vm_frame& f, unsigned long long key,
                                             uint32_t px, uint32_t py, F3* origin) {
  if (key == 0ull) return false;
  const KeyParts k = split_key(key);
  const Chunk c = ld_chunk(w, k.ci);
  const uint32_t id = block_at(w, c, k.vx, k.vy, k.vz);
  if (id == VM_WATER || id == VM_GLASS) return false;
  const F3 rd = ray_dir(f, (float)px + 0.5f, (float)py + 0.5f);
  F3 n = normal_of(k.nid);
  if (k.nid >= VM_NORMAL_CROSS_A && dot(n, rd) > 0.0f) n = neg(n);
  if (dot(n, ld3(f.sun_dir)) <= 0.0f) return false;
  const float t = hit_t(f, c, k.vx, k.vy, k.vz, k.mx, k.my, k.mz, k.nid, rd);
  if (!(t >= 0.0f)) return false;
  const F3 hit = ld3(f.cam_pos) + rd * t;
  *origin = hit + n * (0.02f * c.vs);
  return true;
}

__device__ __forceinline__ float blocker_distance(float blocker) {   // shadow.wgsl:44
  return blocker >= 0.0f ? fminf(fmaxf(blocker, 0.001f), 65504.0f) : 0.0f;
}

// The one secondary ray of a water or glass hit:
//   water: water_refract_leg (resolve.wgsl:1029-1042), gated by
//          FLAG_WATER_REFRACT and refract_detail > 0 (resolve.wgsl:1098,1524);
//   glass: shade_glass's straight transmission (resolve.wgsl:1276-1280).
struct SecRay { F3 o, d; float max_dist; bool water; };
__device__ __forceinline__ bool secondary_setup(const DevWorld& w, const vm_frame& f, unsigned long long key,
                                                uint32_t px, uint32_t py, SecRay* s) {
  if (key == 0ull) return false;
  const KeyParts k = split_key(key);
  const Chunk c = ld_chunk(w, k.ci);
  const uint32_t id = block_at(w, c, k.vx, k.vy, k.vz);
  const bool water = id == VM_WATER, glass = id == VM_GLASS;
  if (!water && !glass) return false;
  const F3 rd = ray_dir(f, (float)px + 0.5f, (float)py + 0.5f);
  const float t = hit_t(f, c, k.vx, k.vy, k.vz, k.mx, k.my, k.mz, k.nid, rd);
  const F3 hit = ld3(f.cam_pos) + rd * t;
  if (water) {
    const float detail = 1.0f - smoothstep(VM_WATER_REFRACT_NEAR, VM_WATER_REFRACT_FAR, t);
    if (!((f.flags & VM_FLAG_WATER_REFRACT) != 0u && detail > 0.0f)) return false;
    const F3 rdir = refract(rd, normal_of(k.nid), 1.0f / VM_WATER_IOR);
    s->o = hit + rdir * VM_SURFACE_EPS;
    s->d = rdir;
    s->max_dist = VM_WATER_REFRACT_DIST;
    s->water = true;
  } else {
    s->o = hit + rd * VM_SURFACE_EPS;
    s->d = rd;
    s->max_dist = fmaxf(VM_GLASS_TRANSMIT_DIST, f.far_);
    s->water = false;
  }
  return true;
}

template <bool COUNT>
__device__ __forceinline__ void secondary_trace(const DevWorld& w, const vm_frame& f, const SecRay& s,
                                                unsigned long long* out_key, float* out_t, Traffic* tr) {
  const WorldHit h = s.water ? trace_world<true, COUNT>(w, f, s.o, s.d, s.max_dist, tr)
                             : trace_world<false, COUNT>(w, f, s.o, s.d, s.max_dist, tr);
  unsigned long long k = (1ull << 63) | (s.water ? 0ull : (1ull << 61));
  if (h.hit)
    k |= (1ull << 62) | ((unsigned long long)h.normal << 37) | ((unsigned long long)h.ci << 24) |
         (unsigned long long)((h.vx << 16) | (h.vy << 8) | h.vz);
  *out_key = k;
  *out_t = h.t;
}

// ---------------------------------------------------------------------------
// The engine's pass sequence
// ---------------------------------------------------------------------------

// tile_select: tile_select.wgsl:11-92.  One warp per 8x8 tile; lanes test 32
// chunks at a time and append the survivors with one atomic per warp.
__global__ void __launch_bounds__(256) k_tile_select(const vm_frame f, const DevWorld w, const uint32_t* __restrict__ hiz,
                                                     uint32_t* __restrict__ pairs, uint32_t* __restrict__ counters) {
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t tile_id = blockIdx.x * 8u + (threadIdx.x >> 5);
  if (tile_id >= f.tiles[0] * f.tiles[1]) return;
  const uint32_t tx = tile_id % f.tiles[0], ty = tile_id / f.tiles[0];
  const TilePlanes tp = tile_planes(f, tx * 8u, ty * 8u);
  const F3 cam = ld3(f.cam_pos), fwd = ld3(f.cam_fwd);
  const bool use_hiz = (f.flags & VM_FLAG_HIZ) != 0u;
  const uint32_t tile_far = hiz[tile_id];
  const uint32_t mp = f.max_pairs;
  for (uint32_t base = 0; base < f.chunk_count; base += 32u) {
    const uint32_t ci = base + lane;
    bool sel = false, def = false;
    if (ci < f.chunk_count) {
      if (ci == f.camera_chunk) {
        sel = true;
      } else {
        const Chunk c = ld_chunk(w, ci);
        const F3 bmin = ld3(c.aabb_min), bmax = ld3(c.aabb_max);
        const bool out = box_outside(bmin, bmax, fwd, cam) || box_outside(bmin, bmax, tp.n[0], cam) ||
                         box_outside(bmin, bmax, tp.n[1], cam) || box_outside(bmin, bmax, tp.n[2], cam) ||
                         box_outside(bmin, bmax, tp.n[3], cam);
        if (!out) {
          const float dmin = box_distance(cam, bmin, bmax);
          if (dmin < tp.reach) {
            if (use_hiz && depth_key(f, dmin) < tile_far) def = true;
            else sel = true;
          }
        }
      }
    }
    const uint32_t word = (tile_id << 13) | ci;
    const uint32_t bs = __ballot_sync(FULLMASK, sel);
    if (bs) {
      uint32_t b0 = 0;
      if (lane == 0) b0 = atomicAdd(&counters[0], __popc(bs));
      b0 = __shfl_sync(FULLMASK, b0, 0);
      if (sel) { const uint32_t i = b0 + __popc(bs & lanemask_lt()); if (i < mp) pairs[i] = word; }
    }
    const uint32_t bd = __ballot_sync(FULLMASK, def);
    if (bd) {
      uint32_t b0 = 0;
      if (lane == 0) b0 = atomicAdd(&counters[1], __popc(bd));
      b0 = __shfl_sync(FULLMASK, b0, 0);
      if (def) { const uint32_t j = b0 + __popc(bd & lanemask_lt()); if (j < mp) pairs[mp + j] = word; }
    }
  }
}

// finalize / finalize_recover: tile_select.wgsl:112-133 (the indirect
// arguments become the march kernels' grid-stride bound).
__global__ void k_finalize(const uint32_t max_pairs, uint32_t* counters, const uint32_t recover) {
  if (!recover) {
    const uint32_t raw = counters[0];
    counters[4] = raw;
    counters[3] = min(raw, max_pairs);
  } else {
    const uint32_t raw = counters[2];
    counters[5] = raw;
    counters[0] = min(raw, max_pairs);
  }
}

// march: march.wgsl:1-55.  Four 8x8 pixel groups per 256-thread block, grid
// stride over the pair list (the indirect dispatch's role).
template <bool UNDERWATER>
__global__ void __launch_bounds__(256) k_march_pairs(const vm_frame f, const DevWorld w, const uint32_t* __restrict__ pairs,
                                                     const uint32_t* __restrict__ counters, unsigned long long* __restrict__ vis,
                                                     uint32_t* __restrict__ dbg) {
  const uint32_t count = min(counters[0], f.max_pairs);
  const uint32_t group = threadIdx.x >> 6, lid = threadIdx.x & 63u;
  const uint32_t lx = lid & 7u, ly = lid >> 3;
  const bool heat = (f.flags & VM_FLAG_HEATMAP) != 0u && dbg != nullptr;
  const F3 cam = ld3(f.cam_pos);
  for (uint32_t p = blockIdx.x * 4u + group; p < count; p += gridDim.x * 4u) {
    const uint32_t pair = pairs[p];
    const uint32_t tile = pair >> 13, ci = pair & 0x1FFFu;
    const uint32_t px = (tile % f.tiles[0]) * 8u + lx, py = (tile / f.tiles[0]) * 8u + ly;
    if (px >= f.res[0] || py >= f.res[1]) continue;
    const Chunk c = ld_chunk(w, ci);
    if (ray_skips(f, c.fade, px, py)) continue;
    const F3 rd = ray_dir(f, (float)px + 0.5f, (float)py + 0.5f);
    const Hit h = march_chunk<UNDERWATER, false, false, false>(w, f, c, make_ray(cam, rd), f.far_, nullptr);
    const uint64_t pix = (uint64_t)py * f.res[0] + px;
    if (h.hit) atomicMax(&vis[pix], make_key(f, h, ci));
    if (heat) atomicAdd(&dbg[pix], h.iters);
  }
}

// build_hiz: march.wgsl:57-76.  One warp per 8x8 tile.
__global__ void __launch_bounds__(256) k_build_hiz(const vm_frame f, const unsigned long long* __restrict__ vis,
                                                   uint32_t* __restrict__ hiz) {
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t tile = blockIdx.x * 8u + (threadIdx.x >> 5);
  if (tile >= f.tiles[0] * f.tiles[1]) return;
  const uint32_t tx = tile % f.tiles[0], ty = tile / f.tiles[0];
  uint32_t m = 0xFFFFFFFFu;
#pragma unroll
  for (uint32_t k = lane; k < 64u; k += 32u) {
    const uint32_t px = tx * 8u + (k & 7u), py = ty * 8u + (k >> 3);
    uint32_t d = 0u;
    if (px < f.res[0] && py < f.res[1]) d = (uint32_t)(vis[(uint64_t)py * f.res[0] + px] >> 40);
    m = min(m, d);
  }
  m = __reduce_min_sync(FULLMASK, m);
  if (lane == 0) hiz[tile] = m;
}

// recover_select: tile_select.wgsl:94-110
__global__ void __launch_bounds__(256) k_recover(const vm_frame f, const DevWorld w, uint32_t* __restrict__ pairs,
                                                 uint32_t* __restrict__ counters, const uint32_t* __restrict__ hiz) {
  const uint32_t n = min(counters[1], f.max_pairs);
  const F3 cam = ld3(f.cam_pos);
  for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
    const uint32_t pair = pairs[f.max_pairs + j];
    const Chunk c = ld_chunk(w, pair & 0x1FFFu);
    const float dmin = box_distance(cam, ld3(c.aabb_min), ld3(c.aabb_max));
    if (depth_key(f, dmin) >= hiz[pair >> 13]) {
      const uint32_t k = atomicAdd(&counters[2], 1u);
      if (k < f.max_pairs) pairs[k] = pair;
    }
  }
}

// primary_shadow: shadow.wgsl:34-48 (blocker distance per pixel, 0 = lit)
__global__ void __launch_bounds__(128) k_primary_shadow(const vm_frame f, const DevWorld w,
                                                        const unsigned long long* __restrict__ vis, float* __restrict__ out) {
  const uint32_t px = blockIdx.x * 16u + threadIdx.x, py = blockIdx.y * 8u + threadIdx.y;
  if (px >= f.res[0] || py >= f.res[1]) return;
  const uint64_t pix = (uint64_t)py * f.res[0] + px;
  float distance = 0.0f;
  F3 o;
  if (shadow_active(f) && shadow_setup(w, f, vis[pix], px, py, &o))
    distance = blocker_distance(shadow_ray_t<false>(w, f, o, ld3(f.sun_dir), f.shadow_dist, nullptr));
  out[pix] = distance;
}

__global__ void __launch_bounds__(128) k_secondary(const vm_frame f, const DevWorld w, const unsigned long long* __restrict__ vis,
                                                   unsigned long long* __restrict__ sec_key, float* __restrict__ sec_t) {
  const uint32_t px = blockIdx.x * 16u + threadIdx.x, py = blockIdx.y * 8u + threadIdx.y;
  if (px >= f.res[0] || py >= f.res[1]) return;
  const uint64_t pix = (uint64_t)py * f.res[0] + px;
  unsigned long long k = 0ull;
  float t = 0.0f;
  SecRay s;
  if (secondary_setup(w, f, vis[pix], px, py, &s)) secondary_trace<false>(w, f, s, &k, &t, nullptr);
  sec_key[pix] = k;
  sec_t[pix] = t;
}

// Expanded visibility: voxel index over a world box, face id, hit_t.
__global__ void __launch_bounds__(256) k_expand(const vm_frame f, const DevWorld w, const unsigned long long* __restrict__ vis,
                                                int32_t wx, int32_t wy, int32_t wz, uint32_t dx, uint32_t dy, uint32_t dz,
                                                uint32_t* __restrict__ voxel, uint8_t* __restrict__ face, float* __restrict__ tout) {
  const uint64_t npix = (uint64_t)f.res[0] * f.res[1];
  for (uint64_t pix = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; pix < npix; pix += (uint64_t)gridDim.x * blockDim.x) {
    const unsigned long long key = vis[pix];
    if (key == 0ull) { voxel[pix] = 0xFFFFFFFFu; face[pix] = 0xFF; tout[pix] = 0.0f; continue; }
    const KeyParts k = split_key(key);
    const Chunk c = ld_chunk(w, k.ci);
    const int32_t vs = __float2int_rz(c.vs);
    const int32_t gx = __float2int_rz(c.origin[0]) + (int32_t)k.vx * vs - wx;
    const int32_t gy = __float2int_rz(c.origin[1]) + (int32_t)k.vy * vs - wy;
    const int32_t gz = __float2int_rz(c.origin[2]) + (int32_t)k.vz * vs - wz;
    (void)dy;
    voxel[pix] = (uint32_t)gx + dx * ((uint32_t)gz + dz * (uint32_t)gy);
    face[pix] = (uint8_t)k.nid;
    const uint32_t px = (uint32_t)(pix % f.res[0]), py = (uint32_t)(pix / f.res[0]);
    tout[pix] = hit_t(f, c, k.vx, k.vy, k.vz, k.mx, k.my, k.mz, k.nid, ray_dir(f, (float)px + 0.5f, (float)py + 0.5f));
  }
}

// Per view: the largest depth key any hit in chunk ci can produce (from a
// lower bound on its hit distance) and its suffix maximum over the view's
// front-to-back chunk list.  The lower bound allows 1e-5 relative and 0.05
// voxel absolute rounding slack between the box distance and a march's t.
struct MaxOp {
  __device__ __forceinline__ uint32_t operator()(uint32_t a, uint32_t b) const { return a > b ? a : b; }
};

__global__ void __launch_bounds__(1024) k_chunk_bounds(const vm_frame* __restrict__ frames, const ViewDesc* __restrict__ views,
                                                       const vm_frame f0, const ViewDesc v0,
                                                       const vm_chunk* __restrict__ chunks, uint32_t* __restrict__ dkmax,
                                                       uint32_t* __restrict__ sufmax) {
  typedef cub::BlockScan<uint32_t, 1024> Scan;
  __shared__ typename Scan::TempStorage tmp;
  const uint32_t v = blockIdx.x;
  const vm_frame& f = frames ? frames[v] : f0;
  const ViewDesc vd = frames ? views[v] : v0;
  const uint32_t n = min(f.chunk_count, vd.n_chunks);
  const F3 cam = ld3(f.cam_pos);
  const uint32_t per = (n + 1023u) / 1024u;
  // thread t owns [t*per, t*per+per) in reverse order so that a forward
  // inclusive max-scan over threads gives the suffix maximum
  const uint32_t t = 1023u - threadIdx.x;
  uint32_t local = 0u;
  for (uint32_t k = 0; k < per; ++k) {
    const uint32_t ci = t * per + k;
    if (ci < n) {
      const vm_chunk& c = chunks[vd.chunk_off + ci];
      const float dmin = box_distance(cam, ld3(c.aabb_min), ld3(c.aabb_max));
      const float lb = fmaxf(dmin * (1.0f - 1e-5f) - 0.05f * c.voxel_size, 0.0f);
      const uint32_t dk = depth_key(f, lb);
      dkmax[vd.chunk_off + ci] = dk;
      local = max(local, dk);
    }
  }
  uint32_t excl;
  Scan(tmp).ExclusiveScan(local, excl, 0u, MaxOp());
  uint32_t run = excl;   // max over all chunks after this thread's range
  for (int k = (int)per - 1; k >= 0; --k) {
    const uint32_t ci = t * per + (uint32_t)k;
    if (ci < n) {
      run = max(run, dkmax[vd.chunk_off + ci]);
      sufmax[vd.chunk_off + ci] = run;
    }
  }
}

// ---------------------------------------------------------------------------
// Fused persistent kernel
// ---------------------------------------------------------------------------
constexpr uint32_t LIST_CAP = 1024;

template <int TW, int TH, bool UNDERWATER, bool COUNT>
__global__ void __launch_bounds__(TW* TH) k_fused(const FusedArgs a) {
  constexpr uint32_t NT = TW * TH;
  constexpr uint32_t NSUB = NT / 64;
  constexpr uint32_t SUBX = TW / 8;
  constexpr uint32_t NWARP = NT / 32;
  __shared__ __align__(16) vm_frame s_f;
  __shared__ ViewDesc s_v;
  __shared__ uint32_t s_item, s_view, s_subvalid;
  __shared__ float s_pl[NSUB][13];
  __shared__ uint32_t s_ci[LIST_CAP], s_dk[LIST_CAP], s_suf[LIST_CAP];
  __shared__ uint32_t s_wc[NWARP];
  __shared__ uint32_t s_q[NT];
  __shared__ float s_qo[NT][3];
  __shared__ uint32_t s_hz[NWARP];

  const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
  const uint32_t sub = tid >> 6;
  Traffic tr = {0, 0, 0, 0, 0, 0, 0};
  uint32_t n_pri = 0, n_sh = 0, n_sec = 0;
  uint32_t cur_view = 0xFFFFFFFFu;

  for (;;) {
    if (tid == 0) {
      const uint32_t item = atomicAdd(a.work, 1u);
      s_item = item;
      if (item < a.total_tiles && a.frames == nullptr) {
        s_view = 0;
      } else if (item < a.total_tiles) {
        uint32_t lo = 0, hi = a.n_views - 1;
        while (lo < hi) {
          const uint32_t mid = (lo + hi + 1) >> 1;
          if (a.views[mid].tile_begin <= item) lo = mid; else hi = mid - 1;
        }
        s_view = lo;
      }
    }
    __syncthreads();
    const uint32_t item = s_item;
    if (item >= a.total_tiles) break;
    if (s_view != cur_view) {
      cur_view = s_view;
      const uint32_t* src = a.frames ? reinterpret_cast<const uint32_t*>(a.frames + cur_view)
                                     : reinterpret_cast<const uint32_t*>(&a.frame0);
      for (uint32_t i = tid; i < sizeof(vm_frame) / 4; i += NT) reinterpret_cast<uint32_t*>(&s_f)[i] = src[i];
      const uint32_t* vsrc = a.frames ? reinterpret_cast<const uint32_t*>(a.views + cur_view)
                                      : reinterpret_cast<const uint32_t*>(&a.view0);
      if (tid < sizeof(ViewDesc) / 4) reinterpret_cast<uint32_t*>(&s_v)[tid] = vsrc[tid];
      __syncthreads();
    }
    const vm_frame& f = s_f;
    const DevWorld w = {a.chunks + s_v.chunk_off, s_v.n_chunks, a.inners, a.n_inners, a.leaves, a.n_leaves,
                        a.bricks, a.n_bricks, a.grids + s_v.grid_off, s_v.grid_len, a.err};
    const uint32_t local = item - s_v.tile_begin;
    const uint32_t x0 = (local % s_v.tiles_x) * TW, y0 = (local / s_v.tiles_x) * TH;
    const uint32_t px = x0 + (sub % SUBX) * 8u + (tid & 7u), py = y0 + (sub / SUBX) * 8u + ((tid >> 3) & 7u);
    const bool valid = px < f.res[0] && py < f.res[1];

    if (tid < NSUB) {
      const uint32_t sx0 = x0 + (tid % SUBX) * 8u, sy0 = y0 + (tid / SUBX) * 8u;
      const bool sv = sx0 < f.res[0] && sy0 < f.res[1];
      const TilePlanes tp = tile_planes(f, sx0, sy0);
#pragma unroll
      for (int i = 0; i < 4; ++i) { s_pl[tid][3 * i] = tp.n[i].x; s_pl[tid][3 * i + 1] = tp.n[i].y; s_pl[tid][3 * i + 2] = tp.n[i].z; }
      s_pl[tid][12] = tp.reach;
      const uint32_t bits = __ballot_sync(NSUB >= 32 ? FULLMASK : ((1u << NSUB) - 1u), sv);
      if (tid == 0) s_subvalid = bits;
    }
    __syncthreads();

    const F3 cam = ld3(f.cam_pos), fwd = ld3(f.cam_fwd);
    const F3 rd = ray_dir(f, (float)px + 0.5f, (float)py + 0.5f);
    const Ray ray = make_ray(cam, rd);
    const uint32_t n_vis = min(f.chunk_count, s_v.n_chunks);
    const uint32_t my_bit = 1u << sub;
    unsigned long long best = 0ull;
    uint32_t scan = 0;
    for (;;) {
      uint32_t list_n = 0;
      while (scan < n_vis && list_n + NT <= LIST_CAP) {
        const uint32_t ci = scan + tid;
        uint32_t mask = 0u;
        if (ci < n_vis) {
          if (ci == f.camera_chunk) {
            mask = s_subvalid;
          } else {
            const float* cp = reinterpret_cast<const float*>(w.chunks + ci);
            const F3 bmin = {__ldg(cp + 0), __ldg(cp + 1), __ldg(cp + 2)};
            const F3 bmax = {__ldg(cp + 4), __ldg(cp + 5), __ldg(cp + 6)};
            if (!box_outside(bmin, bmax, fwd, cam)) {
              const float dmin = box_distance(cam, bmin, bmax);
#pragma unroll
              for (uint32_t s = 0; s < NSUB; ++s) {
                if (!((s_subvalid >> s) & 1u)) continue;
                const float* pl = s_pl[s];
                const bool out = box_outside(bmin, bmax, f3(pl[0], pl[1], pl[2]), cam) ||
                                 box_outside(bmin, bmax, f3(pl[3], pl[4], pl[5]), cam) ||
                                 box_outside(bmin, bmax, f3(pl[6], pl[7], pl[8]), cam) ||
                                 box_outside(bmin, bmax, f3(pl[9], pl[10], pl[11]), cam);
                if (!out && dmin < pl[12]) mask |= 1u << s;
              }
            }
          }
        }
        const uint32_t bal = __ballot_sync(FULLMASK, mask != 0u);
        if (lane == 0) s_wc[warp] = __popc(bal);
        __syncthreads();
        uint32_t off = list_n, total = 0;
#pragma unroll
        for (uint32_t k = 0; k < NWARP; ++k) {
          const uint32_t c = s_wc[k];
          off += k < warp ? c : 0u;
          total += c;
        }
        if (mask) {
          const uint32_t pos = off + __popc(bal & lanemask_lt());
          s_ci[pos] = ci | (mask << 16);
          s_dk[pos] = a.dkmax[s_v.chunk_off + ci];
          s_suf[pos] = a.sufmax[s_v.chunk_off + ci];
        }
        list_n += total;
        scan += NT;
        __syncthreads();
      }
      if (valid) {
        for (uint32_t i = 0; i < list_n; ++i) {
          const uint32_t e = s_ci[i];
          if (!((e >> 16) & my_bit)) continue;
          const uint32_t bestd = (uint32_t)(best >> 40);
          if (s_suf[i] < bestd) break;
          if (s_dk[i] < bestd) continue;
          const uint32_t ci = e & 0xFFFFu;
          const Chunk c = ld_chunk(w, ci);
          if (ray_skips(f, c.fade, px, py)) continue;
          const Hit h = march_chunk<UNDERWATER, false, false, COUNT>(w, f, c, ray, f.far_, &tr);
          if (h.hit) {
            const unsigned long long k = make_key(f, h, ci);
            best = k > best ? k : best;
          }
        }
      }
      if (scan >= n_vis) break;
      const uint32_t rem = a.sufmax[s_v.chunk_off + scan];
      if (__syncthreads_and(!valid || rem < (uint32_t)(best >> 40))) break;
    }
    if (COUNT && valid) ++n_pri;
    const uint64_t pix = s_v.pix_off + (uint64_t)py * f.res[0] + px;
    if (valid) a.vis[pix] = best;

    // Hi-Z of the final visibility per 8x8 tile (build_hiz's reduction)
    {
      uint32_t d = valid ? (uint32_t)(best >> 40) : 0u;
      d = __reduce_min_sync(FULLMASK, d);
      if (lane == 0) s_hz[warp] = d;
    }

    // shadow rays from a compacted queue
    F3 so = {0.0f, 0.0f, 0.0f};
    const bool want_sh = a.do_shadow && valid && shadow_active(f) && shadow_setup(w, f, best, px, py, &so);
    {
      const uint32_t bal = __ballot_sync(FULLMASK, want_sh);
      if (lane == 0) s_wc[warp] = __popc(bal);
      __syncthreads();
      if (tid < NSUB && ((s_subvalid >> tid) & 1u)) {
        const uint32_t sx0 = x0 + (tid % SUBX) * 8u, sy0 = y0 + (tid / SUBX) * 8u;
        a.hiz[s_v.hiz_off + (sy0 / 8u) * f.tiles[0] + sx0 / 8u] = min(s_hz[2 * tid], s_hz[2 * tid + 1]);
      }
      uint32_t off = 0, total = 0;
#pragma unroll
      for (uint32_t k = 0; k < NWARP; ++k) { const uint32_t c = s_wc[k]; off += k < warp ? c : 0u; total += c; }
      if (want_sh) {
        const uint32_t pos = off + __popc(bal & lanemask_lt());
        s_q[pos] = tid;
        s_qo[pos][0] = so.x; s_qo[pos][1] = so.y; s_qo[pos][2] = so.z;
      }
      if (a.do_shadow && valid && !want_sh) a.shadow[pix] = 0.0f;
      __syncthreads();
      for (uint32_t k = tid; k < total; k += NT) {
        const uint32_t lt = s_q[k];
        const uint32_t qsub = lt >> 6;
        const uint32_t qx = x0 + (qsub % SUBX) * 8u + (lt & 7u), qy = y0 + (qsub / SUBX) * 8u + ((lt >> 3) & 7u);
        const float b = shadow_ray_t<COUNT>(w, f, f3(s_qo[k][0], s_qo[k][1], s_qo[k][2]), ld3(f.sun_dir), f.shadow_dist, &tr);
        a.shadow[s_v.pix_off + (uint64_t)qy * f.res[0] + qx] = blocker_distance(b);
        if (COUNT) ++n_sh;
      }
      __syncthreads();
    }

    // water / glass secondary rays from a compacted queue
    if (a.do_secondary) {
      SecRay sr;
      const bool want = valid && secondary_setup(w, f, best, px, py, &sr);
      const uint32_t bal = __ballot_sync(FULLMASK, want);
      if (lane == 0) s_wc[warp] = __popc(bal);
      __syncthreads();
      uint32_t off = 0, total = 0;
#pragma unroll
      for (uint32_t k = 0; k < NWARP; ++k) { const uint32_t c = s_wc[k]; off += k < warp ? c : 0u; total += c; }
      if (want) s_q[off + __popc(bal & lanemask_lt())] = tid;
      if (valid && !want) { a.sec_key[pix] = 0ull; a.sec_t[pix] = 0.0f; }
      __syncthreads();
      for (uint32_t k = tid; k < total; k += NT) {
        const uint32_t lt = s_q[k];
        const uint32_t qsub = lt >> 6;
        const uint32_t qx = x0 + (qsub % SUBX) * 8u + (lt & 7u), qy = y0 + (qsub / SUBX) * 8u + ((lt >> 3) & 7u);
        const uint64_t qpix = s_v.pix_off + (uint64_t)qy * f.res[0] + qx;
        SecRay q;
        secondary_setup(w, f, a.vis[qpix], qx, qy, &q);
        unsigned long long sk; float st;
        secondary_trace<COUNT>(w, f, q, &sk, &st, &tr);
        a.sec_key[qpix] = sk;
        a.sec_t[qpix] = st;
        if (COUNT) ++n_sec;
      }
      __syncthreads();
    }
  }
  if (COUNT) {
    atomicAdd(&a.traffic->chunk, (unsigned long long)tr.chunk);
    atomicAdd(&a.traffic->l1, (unsigned long long)tr.l1);
    atomicAdd(&a.traffic->leaf, (unsigned long long)tr.leaf);
    atomicAdd(&a.traffic->attr, (unsigned long long)tr.attr);
    atomicAdd(&a.traffic->pal, (unsigned long long)tr.pal);
    atomicAdd(&a.traffic->grid, (unsigned long long)tr.grid);
    atomicAdd(&a.traffic->iters, (unsigned long long)tr.iters);
    atomicAdd(&a.traffic->rays_primary, (unsigned long long)n_pri);
    atomicAdd(&a.traffic->rays_shadow, (unsigned long long)n_sh);
    atomicAdd(&a.traffic->rays_secondary, (unsigned long long)n_sec);
  }
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
cudaError_t launch_tile_select(const vm_frame& f, const DevWorld& w, const uint32_t* hiz, uint32_t* pairs,
                               uint32_t* counters, cudaStream_t s) {
  const uint32_t n = f.tiles[0] * f.tiles[1];
  if (n == 0) return cudaSuccess;
  k_tile_select<<<(n + 7) / 8, 256, 0, s>>>(f, w, hiz, pairs, counters);
  return cudaGetLastError();
}

cudaError_t launch_finalize(const vm_frame& f, uint32_t* counters, bool recover, cudaStream_t s) {
  k_finalize<<<1, 1, 0, s>>>(f.max_pairs, counters, recover ? 1u : 0u);
  return cudaGetLastError();
}

cudaError_t launch_march_pairs(const vm_frame& f, const DevWorld& w, const uint32_t* pairs, const uint32_t* counters,
                               unsigned long long* vis, uint32_t* dbg, int sms, cudaStream_t s) {
  const uint32_t grid = (uint32_t)sms * 8u;
  if (f.flags & VM_FLAG_UNDERWATER) k_march_pairs<true><<<grid, 256, 0, s>>>(f, w, pairs, counters, vis, dbg);
  else k_march_pairs<false><<<grid, 256, 0, s>>>(f, w, pairs, counters, vis, dbg);
  return cudaGetLastError();
}

cudaError_t launch_build_hiz(const vm_frame& f, const unsigned long long* vis, uint32_t* hiz, cudaStream_t s) {
  const uint32_t n = f.tiles[0] * f.tiles[1];
  if (n == 0) return cudaSuccess;
  k_build_hiz<<<(n + 7) / 8, 256, 0, s>>>(f, vis, hiz);
  return cudaGetLastError();
}

cudaError_t launch_recover(const vm_frame& f, const DevWorld& w, uint32_t* pairs, uint32_t* counters,
                           const uint32_t* hiz, int sms, cudaStream_t s) {
  k_recover<<<(uint32_t)sms * 4u, 256, 0, s>>>(f, w, pairs, counters, hiz);
  return cudaGetLastError();
}

cudaError_t launch_primary_shadow(const vm_frame& f, const DevWorld& w, const unsigned long long* vis, float* out,
                                  cudaStream_t s) {
  if (f.res[0] == 0 || f.res[1] == 0) return cudaSuccess;
  dim3 g((f.res[0] + 15) / 16, (f.res[1] + 7) / 8);
  k_primary_shadow<<<g, dim3(16, 8), 0, s>>>(f, w, vis, out);
  return cudaGetLastError();
}

cudaError_t launch_secondary(const vm_frame& f, const DevWorld& w, const unsigned long long* vis,
                             unsigned long long* sec_key, float* sec_t, cudaStream_t s) {
  if (f.res[0] == 0 || f.res[1] == 0) return cudaSuccess;
  dim3 g((f.res[0] + 15) / 16, (f.res[1] + 7) / 8);
  k_secondary<<<g, dim3(16, 8), 0, s>>>(f, w, vis, sec_key, sec_t);
  return cudaGetLastError();
}

cudaError_t launch_expand(const vm_frame& f, const DevWorld& w, const unsigned long long* vis, int32_t wx, int32_t wy,
                          int32_t wz, uint32_t dx, uint32_t dy, uint32_t dz, uint32_t* voxel, uint8_t* face, float* t,
                          cudaStream_t s) {
  const uint64_t npix = (uint64_t)f.res[0] * f.res[1];
  if (npix == 0) return cudaSuccess;
  const uint32_t grid = (uint32_t)std::min<uint64_t>((npix + 255) / 256, 148ull * 16);
  k_expand<<<grid, 256, 0, s>>>(f, w, vis, wx, wy, wz, dx, dy, dz, voxel, face, t);
  return cudaGetLastError();
}

cudaError_t launch_chunk_bounds(const vm_frame* frames, const ViewDesc* views, uint32_t n_views, const vm_frame& f0,
                                const ViewDesc& v0, const vm_chunk* chunks, uint32_t* dkmax, uint32_t* sufmax,
                                cudaStream_t s) {
  if (n_views == 0) return cudaSuccess;
  k_chunk_bounds<<<n_views, 1024, 0, s>>>(frames, views, f0, v0, chunks, dkmax, sufmax);
  return cudaGetLastError();
}

template <int TW, int TH>
static cudaError_t launch_fused_t(const FusedArgs& a, bool underwater, bool count, uint32_t grid, cudaStream_t s) {
  if (underwater) {
    if (count) k_fused<TW, TH, true, true><<<grid, TW * TH, 0, s>>>(a);
    else k_fused<TW, TH, true, false><<<grid, TW * TH, 0, s>>>(a);
  } else {
    if (count) k_fused<TW, TH, false, true><<<grid, TW * TH, 0, s>>>(a);
    else k_fused<TW, TH, false, false><<<grid, TW * TH, 0, s>>>(a);
  }
  return cudaGetLastError();
}

cudaError_t launch_fused(const FusedArgs& a, int variant, bool underwater, bool count, uint32_t grid, cudaStream_t s) {
  if (a.total_tiles == 0 || grid == 0) return cudaSuccess;
  switch (variant) {
    case FUSED_8x8: return launch_fused_t<8, 8>(a, underwater, count, grid, s);
    case FUSED_16x8: return launch_fused_t<16, 8>(a, underwater, count, grid, s);
    case FUSED_16x16: return launch_fused_t<16, 16>(a, underwater, count, grid, s);
    case FUSED_32x16: return launch_fused_t<32, 16>(a, underwater, count, grid, s);
  }
  return cudaErrorInvalidValue;
}

template <int TW, int TH>
static int occ_t(bool underwater, bool count) {
  int n = 0;
  if (underwater) {
    if (count) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_fused<TW, TH, true, true>, TW * TH, 0);
    else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_fused<TW, TH, true, false>, TW * TH, 0);
  } else {
    if (count) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_fused<TW, TH, false, true>, TW * TH, 0);
    else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_fused<TW, TH, false, false>, TW * TH, 0);
  }
  return n;
}

int fused_max_ctas_per_sm(int variant, bool underwater, bool count) {
  switch (variant) {
    case FUSED_8x8: return occ_t<8, 8>(underwater, count);
    case FUSED_16x8: return occ_t<16, 8>(underwater, count);
    case FUSED_16x16: return occ_t<16, 16>(underwater, count);
    case FUSED_32x16: return occ_t<32, 16>(underwater, count);
  }
  return 0;
}

}  // namespace vmk
