// Bilateral reconstruction of the sun shadow: shadow_horizontal and
// shadow_vertical (shadow.wgsl:62-116) with SPEC_SOFT_SHADOWS on, fused into
// one kernel.
//
// The engine runs two full-screen passes through two textures and evaluates
// shadow_guide (a key decode, a tree lookup of the block id, ray_dir and
// hit_t) for every tap: 2 * (2L + 1) times per pixel.  Here one CTA owns a
// 32x32 pixel tile: it evaluates the guide and loads the blocker distance once
// for every pixel of the tile and its L-pixel halo into shared memory, runs
// the horizontal pass for the tile's columns over all halo rows, and the
// vertical pass for the tile, writing only the mask (work that cannot change
// a result is skipped, see k_soften).  The horizontal result
// is rounded to binary16 between the passes and the blocker distance on load,
// as the engine's rg16float / r16float targets store them, so both passes see
// the values the engine's would.  Everything but expf is exact (this unit is
// compiled with --fmad=false, IEEE division), so the mask differs from the
// CPU restatement only through expf's last bits.
#include <cuda_fp16.h>
#include <atomic>
#include "kernels.cuh"
#include "ray_stages.cuh"

namespace vmk {

constexpr int SOFT_TILE = 32;                 // output tile edge
constexpr uint32_t SOFT_THREADS = 512;
constexpr int SOFT_WARPS = SOFT_THREADS / 32;

__device__ __forceinline__ float f16_store(float x) { return __half2float(__float2half_rn(x)); }

// shadow_radius: shadow.wgsl:49-54 (SUN_ANGLE = 0.0093, common.wgsl:1535)
__device__ __forceinline__ float soft_radius(float proj, float distance, float depth, float penumbra, float limit) {
  const float r = distance * 0.0093f * penumbra * proj / fmaxf(depth, 0.01f);
  return r >= 0.5f ? fminf(r, limit) : 0.0f;
}

// Shared memory of one CTA: per pixel of the (32 + 2L)^2 region the guide
// (hit point and t, normal as id + flip bit, voxel size, valid), the stored
// distance, its shadow_radius and the visibility key; the horizontal pass for
// the tile's 32 columns; per region row 64-bit masks of the columns with
// distance > 0, of those within L of one (row window) and of those whose
// (2L+1)^2 square holds one.
enum : uint8_t { G_FLIP = 8u, G_VALID = 128u };
struct SoftSmem {
  float4* hit_t;
  unsigned long long* key;
  float2* h;
  float* dist;
  float* rad;
  float* scale;
  uint8_t* code;
  unsigned long long *row, *near, *need;
};

__device__ __forceinline__ SoftSmem soft_smem(void* base, int rw) {
  const int region = rw * rw;
  SoftSmem s;
  char* p = reinterpret_cast<char*>(base);
  s.hit_t = reinterpret_cast<float4*>(p); p += (size_t)region * sizeof(float4);
  s.key = reinterpret_cast<unsigned long long*>(p); p += (size_t)region * 8;
  s.row = reinterpret_cast<unsigned long long*>(p); p += (size_t)rw * 8;
  s.near = reinterpret_cast<unsigned long long*>(p); p += (size_t)rw * 8;
  s.need = reinterpret_cast<unsigned long long*>(p); p += (size_t)rw * 8;
  s.h = reinterpret_cast<float2*>(p); p += (size_t)SOFT_TILE * rw * sizeof(float2);
  s.dist = reinterpret_cast<float*>(p); p += (size_t)region * 4;
  s.rad = reinterpret_cast<float*>(p); p += (size_t)region * 4;
  s.scale = reinterpret_cast<float*>(p); p += (size_t)region * 4;
  s.code = reinterpret_cast<uint8_t*>(p);
  return s;
}

size_t soften_smem_bytes(uint32_t limit) {
  const size_t rw = SOFT_TILE + 2 * limit, region = rw * rw;
  return region * (16 + 8 + 4 + 4 + 4 + 1) + rw * 3 * 8 + (size_t)SOFT_TILE * rw * 8;
}

__device__ __forceinline__ F3 guide_normal(uint8_t code) {
  const F3 n = normal_of(code & 7u);
  return (code & G_FLIP) ? neg(n) : n;
}

// The centre guide of a tap loop, read once
struct Centre { F3 n, hit; float scale; };
__device__ __forceinline__ Centre centre_of(const SoftSmem& s, int a) {
  const float4 h = s.hit_t[a];
  return {guide_normal(s.code[a]), f3(h.x, h.y, h.z), s.scale[a]};
}

// shadow_compatible: shadow.wgsl:55-60, centre a against the guide of pixel b
__device__ __forceinline__ bool soft_compatible(const SoftSmem& s, const Centre& a, int b) {
  const uint8_t cb = s.code[b];
  if (!(cb & G_VALID)) return false;
  const F3 nb = guide_normal(cb);
  if (dot(a.n, nb) < 0.95f) return false;
  const float tolerance = fmaxf(0.01f, 0.01f * fminf(a.scale, s.scale[b]));
  const float4 bh = s.hit_t[b];
  const F3 d = f3(bh.x, bh.y, bh.z) - a.hit;
  return fabsf(dot(d, a.n)) <= tolerance && fabsf(dot(d, nb)) <= tolerance;
}

__device__ __forceinline__ unsigned long long shifted(unsigned long long m, int j) {
  return j >= 0 ? (m << j) : (m >> -j);
}

// Work skipped without changing a result:
//  * a tap is skipped when its radius is below |k| or its guides are not
//    compatible; the radius test comes first, so the compatibility test and
//    expf run only for taps that can contribute;
//  * shadow_radius is 0 at distance 0, so a horizontal result is
//    (occlusion, 0) unless a pixel of its row window has distance > 0, and a
//    vertical result is its horizontal occlusion unless a row window of its
//    column window holds one; those passes are skipped where the masks say
//    so, and a guide, which only they read, is evaluated only in the
//    (2L+1)^2 square around a pixel with distance > 0 (elsewhere: invalid,
//    which gives the same results).  All those windows lie inside the
//    CTA's region.
__global__ void __launch_bounds__(SOFT_THREADS) k_soften(const __grid_constant__ vm_frame f,
                                                         const __grid_constant__ DevWorld w,
                                                         const unsigned long long* __restrict__ vis,
                                                         const float* __restrict__ dist, float* __restrict__ mask,
                                                         uint32_t limit, float penumbra) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int L = (int)limit, RW = SOFT_TILE + 2 * L, region = RW * RW;
  const SoftSmem s = soft_smem(smem_raw, RW);
  const int W = (int)f.res[0], H = (int)f.res[1];
  const int x0 = (int)blockIdx.x * SOFT_TILE - L, y0 = (int)blockIdx.y * SOFT_TILE - L;   // region origin
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  const bool active = shadow_active(f);

  // 1. stored distance and key of every region pixel (0 outside the frame),
  //    PER independent loads in flight per thread
  constexpr int PER = 4;
  for (int i0 = threadIdx.x; i0 < region; i0 += SOFT_THREADS * PER) {
    float dd[PER];
    unsigned long long kk[PER];
#pragma unroll
    for (int j = 0; j < PER; ++j) {
      const int i = i0 + j * (int)SOFT_THREADS;
      const int px = x0 + i % RW, py = y0 + i / RW;
      dd[j] = 0.0f;
      kk[j] = 0ull;
      if (i < region && px >= 0 && py >= 0 && px < W && py < H) {
        const uint64_t pix = (uint64_t)py * (uint64_t)W + (uint64_t)px;
        dd[j] = __ldg(dist + pix);
        kk[j] = __ldg(vis + pix);
      }
    }
#pragma unroll
    for (int j = 0; j < PER; ++j) {
      const int i = i0 + j * (int)SOFT_THREADS;
      if (i < region) { s.dist[i] = f16_store(dd[j]); s.key[i] = kk[j]; }
    }
  }
  __syncthreads();

  // 2. per row: columns with distance > 0 (two ballots of 32 columns)
  int any_row = 0;
  for (int r = (int)warp; r < RW; r += SOFT_WARPS) {
    const int c0 = (int)lane, c1 = (int)lane + 32;
    const unsigned lo = __ballot_sync(FULLMASK, s.dist[r * RW + c0] > 0.0f);
    const unsigned hi = __ballot_sync(FULLMASK, c1 < RW && s.dist[r * RW + c1] > 0.0f);
    const unsigned long long m = ((unsigned long long)hi << 32) | lo;
    if (lane == 0) s.row[r] = m;
    any_row |= m != 0ull ? 1 : 0;
  }
  const bool any = __syncthreads_or(any_row) && active;

  if (any) {
    // 3. row windows, then square windows, as column masks
    const unsigned long long cols = RW >= 64 ? ~0ull : ((1ull << RW) - 1ull);
    if ((int)threadIdx.x < RW) {
      const unsigned long long m = s.row[threadIdx.x];
      unsigned long long nr = 0ull;
      for (int j = -L; j <= L; ++j) nr |= shifted(m, j);
      s.near[threadIdx.x] = nr & cols;
    }
    __syncthreads();
    if ((int)threadIdx.x < RW) {
      const int r = (int)threadIdx.x;
      unsigned long long nd = 0ull;
      for (int j = max(r - L, 0); j <= min(r + L, RW - 1); ++j) nd |= s.near[j];
      s.need[r] = nd;
    }
    __syncthreads();

    // 4. shadow_guide (shadow.wgsl:8-30) where a square window needs it
    const F3 sun = ld3(f.sun_dir), cam = ld3(f.cam_pos);
    const float proj = (float)f.res[1] / (2.0f * fmaxf(f.tan_half_fov, 0.001f));
    const float flimit = (float)limit;
    for (int i = threadIdx.x; i < region; i += SOFT_THREADS) {
      const int c = i % RW, r = i / RW;
      uint8_t code = 0;
      float rad = 0.0f;
      const unsigned long long key = s.key[i];
      if (((s.need[r] >> c) & 1ull) && key != 0ull) {
        const int px = x0 + c, py = y0 + r;
        const KeyParts k = split_key(key);
        const Chunk ch = ld_chunk(w, k.ci);
        const uint32_t id = block_at(w, ch, k.vx, k.vy, k.vz);
        if (id != VM_WATER && !is_glass_leg(w.spec, id)) {
          const F3 rd = ray_dir(f, (float)px + 0.5f, (float)py + 0.5f);
          F3 n = normal_of(k.nid);
          bool flip = false;
          if (k.nid >= VM_NORMAL_CROSS_A && dot(n, rd) > 0.0f) { n = neg(n); flip = true; }
          if (!(dot(n, sun) <= 0.0f)) {
            const float t = hit_t(f, ch, k.vx, k.vy, k.vz, k.mx, k.my, k.mz, k.nid, rd);
            const F3 hit = cam + rd * t;
            s.hit_t[i] = make_float4(hit.x, hit.y, hit.z, t);
            s.scale[i] = ch.vs;
            if (t >= 0.0f) {
              code = (uint8_t)(k.nid | (flip ? G_FLIP : 0u) | G_VALID);
              rad = soft_radius(proj, s.dist[i], t, penumbra, flimit);
            }
          }
        }
      }
      s.code[i] = code;
      s.rad[i] = rad;
    }
    __syncthreads();

    // 5. shadow_horizontal for the tile's columns, every region row
    for (int i = threadIdx.x; i < SOFT_TILE * RW; i += SOFT_THREADS) {
      const int tc = i % SOFT_TILE, r = i / SOFT_TILE, c = L + tc, p = r * RW + c;
      float hx = s.dist[p] > 0.0f ? 1.0f : 0.0f, hy = 0.0f;
      if (((s.near[r] >> c) & 1ull) && (s.code[p] & G_VALID)) {
        const float rc = s.rad[p];
        const Centre cp = centre_of(s, p);
        float sum = hx, weight = 1.0f, support = rc;
        for (int k = -L; k <= L; ++k) {
          if (k == 0) continue;
          const int q = p + k;
          const float rr = fmaxf(rc, s.rad[q]);
          if (rr < fabsf((float)k)) continue;
          if (!soft_compatible(s, cp, q)) continue;
          const float wk = expf(-2.0f * (float)(k * k) / fmaxf(rr * rr, 0.25f));
          sum += (s.dist[q] > 0.0f ? 1.0f : 0.0f) * wk;
          weight += wk;
          support = fmaxf(support, rr);
        }
        hx = sum / weight;
        hy = support;
      }
      s.h[r * SOFT_TILE + tc] = make_float2(f16_store(hx), f16_store(hy));
    }
    __syncthreads();
  }

  // 6. shadow_vertical for the tile; the mask before r8unorm quantisation
  for (int i = threadIdx.x; i < SOFT_TILE * SOFT_TILE; i += SOFT_THREADS) {
    const int tc = i % SOFT_TILE, tr = i / SOFT_TILE;
    const int px = (int)blockIdx.x * SOFT_TILE + tc, py = (int)blockIdx.y * SOFT_TILE + tr;
    if (px >= W || py >= H) continue;
    const int r = tr + L, c = tc + L, p = r * RW + c;
    float occ;
    if (!any) {
      occ = s.dist[p] > 0.0f ? 1.0f : 0.0f;   // f16_store of 0 or 1 is itself
    } else {
      const float2 hp = s.h[r * SOFT_TILE + tc];
      occ = hp.x;
      if (((s.need[r] >> c) & 1ull) && (s.code[p] & G_VALID)) {
        const Centre cp = centre_of(s, p);
        float sum = hp.x, weight = 1.0f;
        for (int k = -L; k <= L; ++k) {
          if (k == 0) continue;
          const int q = p + k * RW;
          const float2 hq = s.h[(r + k) * SOFT_TILE + tc];
          const float rr = fmaxf(hp.y, hq.y);
          if (rr < fabsf((float)k)) continue;
          if (!soft_compatible(s, cp, q)) continue;
          const float wk = expf(-2.0f * (float)(k * k) / fmaxf(rr * rr, 0.25f));
          sum += hq.x * wk;
          weight += wk;
        }
        occ = sum / weight;
      }
    }
    mask[(uint64_t)py * (uint64_t)W + (uint64_t)px] = fminf(fmaxf(1.0f - occ, 0.0f), 1.0f);
  }
}

cudaError_t launch_soften(const vm_frame& f, const DevWorld& w, const unsigned long long* vis, const float* dist,
                          float* mask, uint32_t limit, float penumbra, cudaStream_t s) {
  if (limit < 1u || limit > SOFTEN_MAX_LIMIT) return cudaErrorInvalidValue;
  const size_t smem = soften_smem_bytes(limit);
  // the kernel's dynamic shared memory limit, raised once per device
  static std::atomic<uint64_t> attr_set{0};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const uint64_t bit = 1ull << (dev & 63);
  if ((attr_set.load() & bit) == 0) {
    e = cudaFuncSetAttribute(k_soften, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)soften_smem_bytes(SOFTEN_MAX_LIMIT));
    if (e != cudaSuccess) return e;
    attr_set.fetch_or(bit);
  }
  const dim3 grid((f.res[0] + SOFT_TILE - 1) / SOFT_TILE, (f.res[1] + SOFT_TILE - 1) / SOFT_TILE);
  k_soften<<<grid, SOFT_THREADS, smem, s>>>(f, w, vis, dist, mask, limit, penumbra);
  return cudaGetLastError();
}

}  // namespace vmk
