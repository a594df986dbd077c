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
#include "ray_stages.cuh"
#include <algorithm>
#include <cuda_fp16.h>

namespace vmk {
using namespace vmd;

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
    Hit h = march_chunk<UNDERWATER, false, false, false, false, true>(w, f, c, make_ray(cam, rd), f.far_, nullptr);
    if (UNDERWATER && (w.spec & VM_SPEC_SNELL_BEND) != 0u && !h.hit) snell_bend<false, false, true>(w, f, c, rd, &h, nullptr);
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
  if (shadow_active(f) && shadow_setup(w, f, vis[pix], px, py, &o)) {
    if (soft_shadows(w.spec)) {
      // the blocked fraction of the jittered rays
      uint32_t blocked = 0;
      for (uint32_t s = 0; s < VM_SOFT_SAMPLES; ++s)
        blocked += shadow_ray_t<false>(w, f, o, soft_sun_dir(f, px, py, s), f.shadow_dist, nullptr) >= 0.0f ? 1u : 0u;
      distance = (float)blocked * (1.0f / (float)VM_SOFT_SAMPLES);
    } else {
      distance = blocker_distance(shadow_ray_t<false>(w, f, o, ld3(f.sun_dir), f.shadow_dist, nullptr));
    }
  }
  out[pix] = distance;
}

__global__ void __launch_bounds__(128) k_secondary(const vm_frame f, const DevWorld w, const unsigned long long* __restrict__ vis,
                                                   unsigned long long* __restrict__ sec_key, float* __restrict__ sec_t,
                                                   unsigned long long* __restrict__ refl_key,
                                                   float* __restrict__ refl_t) {
  const uint32_t px = blockIdx.x * 16u + threadIdx.x, py = blockIdx.y * 8u + threadIdx.y;
  if (px >= f.res[0] || py >= f.res[1]) return;
  const uint64_t pix = (uint64_t)py * f.res[0] + px;
  unsigned long long k = 0ull;
  float t = 0.0f;
  SecRay s;
  if (secondary_setup(w, f, vis[pix], px, py, &s)) secondary_trace<false, true>(w, f, s, &k, &t, nullptr);
  sec_key[pix] = k;
  sec_t[pix] = t;
  if (refl_key) {
    k = 0ull;
    t = 0.0f;
    if (reflect_setup<true>(w, f, vis[pix], px, py, &s)) secondary_trace<false, true>(w, f, s, &k, &t, nullptr);
    refl_key[pix] = k;
    refl_t[pix] = t;
  }
}

// water_sec (resolve.wgsl:1468-1535): the engine's schedule of the water
// legs, one per (1 << shift)^2 pixel block (WATER_SEC_SHIFT = 1: 2x2).  The
// block's water pixel nearest the camera (smallest hit_t, the first in x-major
// order on a tie) traces the refract leg (water_refract_leg, along the face
// normal) and the reflect leg (water_reflect_leg, along water_ctx's
// mirror_t); blocks without water, or legs their detail gate turns off, get
// key 0.  Keys as the secondary keys (bit 61 clear: water), t the leg's hit
// distance.
__global__ void __launch_bounds__(128) k_water_sec(const vm_frame f, const DevWorld w,
                                                   const unsigned long long* __restrict__ vis, uint32_t shift,
                                                   unsigned long long* __restrict__ refr_key, float* __restrict__ refr_t,
                                                   unsigned long long* __restrict__ refl_key,
                                                   float* __restrict__ refl_t) {
  const uint32_t span = 1u << shift;
  const uint32_t hw = (f.res[0] + span - 1u) >> shift, hh = (f.res[1] + span - 1u) >> shift;
  const uint32_t hx = blockIdx.x * 16u + threadIdx.x, hy = blockIdx.y * 8u + threadIdx.y;
  if (hx >= hw || hy >= hh) return;
  float best_t = 3.4e38f;
  bool has = false;
  KeyParts best = {};
  uint32_t bpx = 0, bpy = 0;
  for (uint32_t i = 0; i < span; ++i)
    for (uint32_t j = 0; j < span; ++j) {
      const uint32_t pxs = span * hx + i, pys = span * hy + j;
      if (pxs >= f.res[0] || pys >= f.res[1]) continue;
      const unsigned long long key = vis[(uint64_t)pys * f.res[0] + pxs];
      if (key == 0ull) continue;
      const KeyParts k = split_key(key);
      const Chunk c = ld_chunk(w, k.ci);
      if (block_at(w, c, k.vx, k.vy, k.vz) != VM_WATER) continue;
      const F3 rd0 = ray_dir(f, (float)pxs + 0.5f, (float)pys + 0.5f);
      const float ts = hit_t(f, c, k.vx, k.vy, k.vz, k.mx, k.my, k.mz, k.nid, rd0);
      if (ts < best_t) { best_t = ts; best = k; bpx = pxs; bpy = pys; has = true; }
    }
  unsigned long long kr = 0ull, km = 0ull;
  float tr_ = 0.0f, tm = 0.0f;
  if (has) {
    const F3 rd = ray_dir(f, (float)bpx + 0.5f, (float)bpy + 0.5f);
    const F3 hit = ld3(f.cam_pos) + rd * best_t;
    SecRay s;
    if ((f.flags & VM_FLAG_WATER_REFRACT) != 0u &&
        1.0f - smoothstep(VM_WATER_REFRACT_NEAR, VM_WATER_REFRACT_FAR, best_t) > 0.0f) {
      s.d = refract(rd, normal_of(best.nid), 1.0f / VM_WATER_IOR);
      s.o = hit + s.d * VM_SURFACE_EPS;
      s.max_dist = VM_WATER_REFRACT_DIST;
      s.water = true;
      secondary_trace<false, true>(w, f, s, &kr, &tr_, nullptr);
    }
    if (water_reflects(f, best_t)) {
      s = reflect_ray<false, true>(w, f, hit, rd, best.nid, best_t, nullptr);
      secondary_trace<false, true>(w, f, s, &km, &tm, nullptr);
    }
  }
  const uint64_t h = (uint64_t)hy * hw + hx;
  refr_key[h] = kr; refr_t[h] = tr_;
  refl_key[h] = km; refl_t[h] = tm;
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
                             unsigned long long* sec_key, float* sec_t, unsigned long long* refl_key, float* refl_t,
                             cudaStream_t s) {
  if (f.res[0] == 0 || f.res[1] == 0) return cudaSuccess;
  dim3 g((f.res[0] + 15) / 16, (f.res[1] + 7) / 8);
  k_secondary<<<g, dim3(16, 8), 0, s>>>(f, w, vis, sec_key, sec_t, refl_key, refl_t);
  return cudaGetLastError();
}

cudaError_t launch_water_sec(const vm_frame& f, const DevWorld& w, const unsigned long long* vis, uint32_t shift,
                             unsigned long long* refr_key, float* refr_t, unsigned long long* refl_key,
                             float* refl_t, cudaStream_t s) {
  const uint32_t span = 1u << shift;
  const uint32_t hw = (f.res[0] + span - 1u) >> shift, hh = (f.res[1] + span - 1u) >> shift;
  if (hw == 0 || hh == 0) return cudaSuccess;
  k_water_sec<<<dim3((hw + 15) / 16, (hh + 7) / 8), dim3(16, 8), 0, s>>>(f, w, vis, shift, refr_key, refr_t, refl_key,
                                                                           refl_t);
  return cudaGetLastError();
}

// The blocker distances in the engine's shadow target format
// (shadow_dist_tex, texture_storage_2d<r16float>, shadow.wgsl:1): binary16,
// rounded to nearest even.  Four pixels per thread (16 B in, 8 B out).
__global__ void __launch_bounds__(256) k_to_r16f(const float* __restrict__ in, uint16_t* __restrict__ out,
                                                 uint64_t n) {
  const uint64_t n4 = n / 4u, stride = (uint64_t)gridDim.x * blockDim.x;
  const uint64_t i0 = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  for (uint64_t i = i0; i < n4; i += stride) {
    const float4 v = reinterpret_cast<const float4*>(in)[i];
    ushort4 h;
    h.x = __half_as_ushort(__float2half_rn(v.x));
    h.y = __half_as_ushort(__float2half_rn(v.y));
    h.z = __half_as_ushort(__float2half_rn(v.z));
    h.w = __half_as_ushort(__float2half_rn(v.w));
    reinterpret_cast<ushort4*>(out)[i] = h;
  }
  for (uint64_t i = 4u * n4 + i0; i < n; i += stride) out[i] = __half_as_ushort(__float2half_rn(in[i]));
}

cudaError_t launch_to_r16f(const float* in, uint16_t* out, uint64_t n, int sms, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  const uint64_t want = (n / 4u + 255u) / 256u;
  const uint32_t blocks = (uint32_t)std::max<uint64_t>(1u, std::min<uint64_t>(want, (uint64_t)sms * 8u));
  k_to_r16f<<<blocks, 256, 0, s>>>(in, out, n);
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

}  // namespace vmk
