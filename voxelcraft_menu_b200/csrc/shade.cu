// Differentiable shading over a fixed visibility buffer, sm_100a.
//
// The traversal stays discrete and exact: a G-buffer pass (gbuffer.cu)
// decodes, once, what the march produced for every pixel (block id and face
// of the primary hit, the sun shadow's verdict, the water refraction leg's
// hit and length, the fog's optical length) into 16 bytes.  The shading
// model is then a smooth function of the parameters only, restating the
// reference's terms:
//   sun:      A[id] * SUN_RGB * lit * max(n.s, 0)       (resolve.wgsl:746-756,787)
//   sky:      A[id] * K * 0.5                           (resolve.wgsl:786)
//   water:    under * tr + body * (1 - tr), tr = exp(-alpha * d),
//             body = A[WATER] * K                       (common.wgsl:1262-1265,
//                                                        resolve.wgsl:1163-1170)
//   fog:      c * T + K * (1 - T), T = exp(-clamp(rho * L, 0, 60)) with
//             L = e * path of transmittance_from        (common.wgsl:1332-1341,
//                                                        resolve.wgsl:1453-1458)
// with parameters A (256 x 3 albedo), s (sun direction, normalised inside),
// K (sky ambient RGB), rho (fog density) and alpha (water absorption RGB).
// The adjoint recomputes the forward per pixel (fused with the L2 loss when
// given the target) and accumulates parameter gradients per block in FP32
// (a few hundred terms per lane), then into FP64 globals.  Unlike the march,
// this file is compiled with floating-point contraction: the model is held to
// tolerances against FP64, not to bit equality.
#include <cuda_runtime.h>
#include <atomic>
#include <cstdint>

#include "shade.cuh"

namespace vmk {

// the hit's normal; cross-quad normals face the ray (shadow.wgsl:23), which
// the G-buffer records as G_FLIP
__device__ __forceinline__ F3 nrm_of(uint32_t code) {
  const F3 n = normal_of((code >> 8) & 7u);
  return (code & G_FLIP) ? neg(n) : n;
}

// Gradient accumulators of one lane.  Albedo rows below COL_ROWS (every
// block the world generator places; the engine has VM_BLOCK_COUNT = 26) go to
// the warp's column table in shared memory, one column per lane, so the adds
// need neither atomics nor a bank conflict; the water row stays in registers
// and any other row goes to the block's table with shared atomics.
constexpr uint32_t COL_ROWS = 16;
constexpr uint32_t COL_FLOATS = COL_ROWS * 3 * 32;   // per warp

struct GradAcc {
  float gs[3] = {0, 0, 0};        // d/d(normalised sun)
  float gK[3] = {0, 0, 0};
  float grho = 0.0f;
  float galpha[3] = {0, 0, 0};
  float gW[3] = {0, 0, 0};        // water albedo row
  float loss = 0.0f;
  float* col = nullptr;           // this lane's column: col[(row * 3 + ch) * 32]
  float* sA = nullptr;            // the block's table for rows >= COL_ROWS
};

__device__ __forceinline__ void row_add(GradAcc* acc, uint32_t row, const float* v) {
  if (row < COL_ROWS) {
    float* c = acc->col + row * 96u;
    c[0] += v[0]; c[32] += v[1]; c[64] += v[2];
  } else {
    atomicAdd(&acc->sA[3 * row], v[0]); atomicAdd(&acc->sA[3 * row + 1], v[1]); atomicAdd(&acc->sA[3 * row + 2], v[2]);
  }
}

// One pixel: colour c_out and, with BWD, the adjoint of colour -> parameters
// for dL/dcolour = io, or (tgt) the L2 loss against the target io.
// P is the parameter vector staged in shared memory.
template <bool BWD>
__device__ __forceinline__ void shade_px(const GBuf& g, const float* __restrict__ P, const ShadeK& k, F3 sn,
                                         float c_out[3], const float* io, bool tgt, GradAcc* acc) {
  const float K[3] = {P[P_SKY], P[P_SKY + 1], P[P_SKY + 2]};
  const bool hit = (g.code & G_HIT) != 0u;
  if (!hit) {
    for (int ch = 0; ch < 3; ++ch) c_out[ch] = K[ch];
    if (BWD) {
      for (int ch = 0; ch < 3; ++ch) {
        const float dc = tgt ? 2.0f * (K[ch] - io[ch]) : io[ch];
        if (tgt) acc->loss += 0.25f * dc * dc;
        acc->gK[ch] += dc;
      }
    }
    return;
  }
  const uint32_t id = g.code & 0xFFu;
  const bool water = id == VM_WATER;
  float c[3];
  float ndl = 0.0f, lit = 0.0f, ndl2 = 0.0f, tr[3] = {0, 0, 0}, under[3] = {0, 0, 0};
  bool traced = false, hit2 = false;
  uint32_t id2 = 0u;
  F3 n = {0, 0, 0}, n2 = {0, 0, 0};
  const float* Aw = P + 3 * VM_WATER;
  if (!water) {
    n = nrm_of(g.code);
    lit = (g.code & G_SOFT) ? 1.0f - (float)((g.code >> G_SOFT_SHIFT) & 7u) * (1.0f / (float)VM_SOFT_SAMPLES)
                            : ((g.code & G_LIT) ? 1.0f : 0.0f);
    ndl = fmaxf(dot(n, sn), 0.0f);
    const float* A = P + 3 * id;
    for (int ch = 0; ch < 3; ++ch) c[ch] = A[ch] * (k.sun_rgb[ch] * lit * ndl + K[ch] * 0.5f);
  } else {
    traced = (g.code & G_TRACED) != 0u;
    for (int ch = 0; ch < 3; ++ch) c[ch] = Aw[ch] * K[ch];
    if (traced) {
      hit2 = (g.code & G_HIT2) != 0u;
      if (hit2) {
        id2 = (g.code >> 16) & 0xFFu;
        n2 = normal_of((g.code >> 24) & 7u);
        ndl2 = fmaxf(dot(n2, sn), 0.0f);
        const float* A2 = P + 3 * id2;
        for (int ch = 0; ch < 3; ++ch) under[ch] = A2[ch] * (k.sun_rgb[ch] * ndl2 + K[ch] * 0.5f);
      }
      const float d = fmaxf(g.d, 0.0f);
      for (int ch = 0; ch < 3; ++ch) {
        tr[ch] = expf(-P[P_ABS + ch] * d);
        c[ch] = under[ch] * tr[ch] + c[ch] * (1.0f - tr[ch]);
      }
    }
  }
  const float tau = P[P_FOG] * g.fog;
  const float T = expf(-fminf(fmaxf(tau, 0.0f), 60.0f));
  for (int ch = 0; ch < 3; ++ch) c_out[ch] = c[ch] * T + K[ch] * (1.0f - T);
  if (!BWD) return;

  // ---- adjoint ----
  float dc[3], dTsum = 0.0f;
  for (int ch = 0; ch < 3; ++ch) {
    float x = io[ch];
    if (tgt) {
      x = 2.0f * (c_out[ch] - io[ch]);
      acc->loss += 0.25f * x * x;
    }
    dTsum += x * (c[ch] - K[ch]);
    acc->gK[ch] += x * (1.0f - T);
    dc[ch] = x * T;
  }
  if (tau > 0.0f && tau < 60.0f) acc->grho += dTsum * (-T * g.fog);
  if (!water) {
    const float* A = P + 3 * id;
    float dndl = 0.0f, gA[3];
    for (int ch = 0; ch < 3; ++ch) {
      gA[ch] = dc[ch] * (k.sun_rgb[ch] * lit * ndl + K[ch] * 0.5f);
      acc->gK[ch] += dc[ch] * A[ch] * 0.5f;
      dndl += dc[ch] * A[ch] * k.sun_rgb[ch] * lit;
    }
    row_add(acc, id, gA);
    if (ndl > 0.0f) { acc->gs[0] += dndl * n.x; acc->gs[1] += dndl * n.y; acc->gs[2] += dndl * n.z; }
    return;
  }
  if (!traced) {
    for (int ch = 0; ch < 3; ++ch) { acc->gW[ch] += dc[ch] * K[ch]; acc->gK[ch] += dc[ch] * Aw[ch]; }
    return;
  }
  const float* A2 = P + 3 * id2;
  const float d = fmaxf(g.d, 0.0f);
  float dndl2 = 0.0f, gA2[3];
  for (int ch = 0; ch < 3; ++ch) {
    const float body = Aw[ch] * K[ch];
    const float dunder = dc[ch] * tr[ch];
    const float dbody = dc[ch] * (1.0f - tr[ch]);
    acc->galpha[ch] += dc[ch] * (under[ch] - body) * tr[ch] * (-d);
    acc->gW[ch] += dbody * K[ch];
    acc->gK[ch] += dbody * Aw[ch];
    gA2[ch] = dunder * (k.sun_rgb[ch] * ndl2 + K[ch] * 0.5f);
    if (hit2) {
      acc->gK[ch] += dunder * A2[ch] * 0.5f;
      dndl2 += dunder * A2[ch] * k.sun_rgb[ch];
    }
  }
  if (hit2) {
    row_add(acc, id2, gA2);
    if (ndl2 > 0.0f) { acc->gs[0] += dndl2 * n2.x; acc->gs[1] += dndl2 * n2.y; acc->gs[2] += dndl2 * n2.z; }
  }
}

__device__ __forceinline__ void stage_params(float* sP, const float* __restrict__ P) {
  for (int i = threadIdx.x; i < NP; i += blockDim.x) sP[i] = P[i];
}

__device__ __forceinline__ F3 sun_unit(const float* P, float* inv_len) {
  const F3 s = {P[P_SUN], P[P_SUN + 1], P[P_SUN + 2]};
  const float l = sqrtf(dot(s, s));
  *inv_len = 1.0f / l;
  return {s.x / l, s.y / l, s.z / l};
}

// FPF pixels per thread and step, their G-buffer loads issued together
constexpr uint32_t FPF = 4;
__global__ void __launch_bounds__(256) k_shade_fwd(const GBuf* __restrict__ gb, uint64_t n, const float* __restrict__ P,
                                                   ShadeK k, float* __restrict__ color, const float* __restrict__ target,
                                                   double* __restrict__ loss) {
  __shared__ float sP[NP];
  __shared__ double sLoss[8];
  stage_params(sP, P);
  __syncthreads();
  float inv_len;
  const F3 sn = sun_unit(sP, &inv_len);
  float acc = 0.0f;           // a few dozen terms per thread; the block sum is FP64
  const uint64_t step = (uint64_t)gridDim.x * blockDim.x * FPF;
  for (uint64_t i0 = (uint64_t)blockIdx.x * blockDim.x * FPF + threadIdx.x; i0 < n; i0 += step) {
    GBuf gv[FPF];
#pragma unroll
    for (uint32_t u = 0; u < FPF; ++u) {
      const uint64_t i = i0 + (uint64_t)u * blockDim.x;
      if (i < n) gv[u] = gb[i];
    }
#pragma unroll
    for (uint32_t u = 0; u < FPF; ++u) {
      const uint64_t i = i0 + (uint64_t)u * blockDim.x;
      if (i >= n) break;
      float c[3];
      shade_px<false>(gv[u], sP, k, sn, c, nullptr, false, nullptr);
      if (color) { color[3 * i] = c[0]; color[3 * i + 1] = c[1]; color[3 * i + 2] = c[2]; }
      if (target) {
        for (int ch = 0; ch < 3; ++ch) { const float e = c[ch] - target[3 * i + ch]; acc += e * e; }
      }
    }
  }
  if (loss) {
    double a = acc;
    for (int o = 16; o > 0; o >>= 1) a += __shfl_down_sync(0xFFFFFFFFu, a, o);
    if ((threadIdx.x & 31u) == 0) sLoss[threadIdx.x >> 5] = a;
    __syncthreads();
    if (threadIdx.x == 0) {
      double s = 0.0;
      for (uint32_t wv = 0; wv < (blockDim.x >> 5); ++wv) s += sLoss[wv];
      atomicAdd(loss, s);
    }
  }
}

// dL/dparams.  dcolor: dL/dcolour per pixel, or nullptr to use the L2 loss
// against target (dL/dc = 2 (c - target)), whose value then goes to loss.
// A warp walks runs of 32 x SEG consecutive pixels; the loads of PF pixels
// are issued together, then the pixels shaded.
constexpr uint32_t SEG = 8;
constexpr uint32_t PF = 4;
constexpr uint32_t BWD_WARPS = 8;
constexpr size_t BWD_SMEM = (size_t)BWD_WARPS * COL_FLOATS * sizeof(float);   // column tables (dynamic)
__global__ void __launch_bounds__(BWD_WARPS * 32, 3) k_shade_bwd(const GBuf* __restrict__ gb, uint64_t n,
                                                                 const float* __restrict__ P, ShadeK k,
                                                                 const float* __restrict__ dcolor,
                                                                 const float* __restrict__ target,
                                                                 double* __restrict__ grad, double* __restrict__ loss) {
  constexpr int NS = 14;                   // sun 3, sky 3, fog 1, absorb 3, water albedo 3, loss
  extern __shared__ float sCol[];          // [warp][row * 3 + ch][lane]
  __shared__ float sA[768];
  __shared__ float sP[NP];
  __shared__ float sScal[BWD_WARPS][NS];
  __shared__ float sRows[BWD_WARPS][COL_ROWS * 3];
  __shared__ uint32_t sNext;
  for (int i = threadIdx.x; i < 768; i += blockDim.x) sA[i] = 0.0f;
  for (uint32_t i = threadIdx.x; i < BWD_WARPS * COL_FLOATS; i += blockDim.x) sCol[i] = 0.0f;
  stage_params(sP, P);
  if (threadIdx.x == 0) sNext = 0u;
  __syncthreads();
  float inv_len;
  const F3 sn = sun_unit(sP, &inv_len);
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  GradAcc acc;
  acc.col = sCol + warp * COL_FLOATS + lane;
  acc.sA = sA;
  const bool tgt = dcolor == nullptr;
  const float* __restrict__ src = tgt ? target : dcolor;
  const uint64_t runs = (n + 32 * SEG - 1) / (32 * SEG);
  // The block owns runs blockIdx.x + q * gridDim.x (spread over the image, so
  // every block sees the same mix of sky and geometry); its warps take them
  // in turn from a shared counter, so none idles while another has work.
  for (;;) {
    uint32_t q = 0u;
    if (lane == 0) q = atomicAdd(&sNext, 1u);
    q = __shfl_sync(0xFFFFFFFFu, q, 0);
    const uint64_t run = (uint64_t)blockIdx.x + (uint64_t)q * gridDim.x;
    if (run >= runs) break;
    const uint64_t base = run * (32 * SEG) + lane;
#pragma unroll 1
    for (uint32_t j0 = 0; j0 < SEG; j0 += PF) {
      GBuf gv[PF];
      float iov[PF][3];
#pragma unroll
      for (uint32_t u = 0; u < PF; ++u) {
        const uint64_t i = base + (uint64_t)(j0 + u) * 32;
        if (i < n) {
          gv[u] = gb[i];
          iov[u][0] = src[3 * i]; iov[u][1] = src[3 * i + 1]; iov[u][2] = src[3 * i + 2];
        }
      }
#pragma unroll
      for (uint32_t u = 0; u < PF; ++u) {
        if (base + (uint64_t)(j0 + u) * 32 < n) {
          float c[3];
          shade_px<true>(gv[u], sP, k, sn, c, iov[u], tgt, &acc);
        }
      }
    }
  }
  // the warp's columns: lane l sums entries l and l + 32 over the 32 lanes,
  // reading lane (l + j) mod 32 at step j so that no two lanes share a bank
  __syncwarp();
  const float* wcol = sCol + warp * COL_FLOATS;
  for (uint32_t e = lane; e < COL_ROWS * 3; e += 32) {
    float x = 0.0f;
    for (uint32_t j = 0; j < 32; ++j) x += wcol[e * 32 + ((lane + j) & 31u)];
    sRows[warp][e] = x;
  }
  // scalar parameters, the water row and the loss: warp sums, then block sums
  const float v[NS] = {acc.gs[0], acc.gs[1], acc.gs[2], acc.gK[0], acc.gK[1], acc.gK[2], acc.grho,
                       acc.galpha[0], acc.galpha[1], acc.galpha[2], acc.gW[0], acc.gW[1], acc.gW[2], acc.loss};
#pragma unroll
  for (int j = 0; j < NS; ++j) {
    float x = v[j];
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xFFFFFFFFu, x, o);
    if (lane == 0) sScal[warp][j] = x;
  }
  __syncthreads();
  if (threadIdx.x < COL_ROWS * 3) {
    float x = 0.0f;
    for (uint32_t wv = 0; wv < BWD_WARPS; ++wv) x += sRows[wv][threadIdx.x];
    sA[threadIdx.x] += x;     // rows below COL_ROWS never reach sA through atomics
  }
  if (threadIdx.x >= 64 && threadIdx.x < 64 + NS) {
    const uint32_t q = threadIdx.x - 64;
    double x = 0.0;
    for (uint32_t wv = 0; wv < BWD_WARPS; ++wv) x += sScal[wv][q];
    if (q < 3) {
      // through s / |s|: ds = (I - sn sn^T) dsn / |s|
      double d0 = 0.0, d1 = 0.0, d2 = 0.0;
      for (uint32_t wv = 0; wv < BWD_WARPS; ++wv) { d0 += sScal[wv][0]; d1 += sScal[wv][1]; d2 += sScal[wv][2]; }
      const double proj = d0 * sn.x + d1 * sn.y + d2 * sn.z;
      const double snq = q == 0 ? sn.x : (q == 1 ? sn.y : sn.z);
      atomicAdd(grad + P_SUN + q, (x - proj * snq) * (double)inv_len);
    } else if (q < 6) {
      atomicAdd(grad + P_SKY + (q - 3), x);
    } else if (q == 6) {
      atomicAdd(grad + P_FOG, x);
    } else if (q < 10) {
      atomicAdd(grad + P_ABS + (q - 7), x);
    } else if (q < 13) {
      atomicAdd(grad + 3 * VM_WATER + (q - 10), x);
    } else if (loss && tgt) {
      atomicAdd(loss, x);
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < 768; i += blockDim.x)
    if (sA[i] != 0.0f) atomicAdd(grad + i, (double)sA[i]);
}

}  // namespace vmk

// ===========================================================================
// C ABI
// ===========================================================================
using vmk::GBuf;

extern "C" int vm_shade_forward(const void* d_gbuf, uint64_t n_pixels, const float* d_params,
                                const vm_shade_consts* consts, float* d_color, const float* d_target, double* d_loss,
                                void* stream) {
  if (!d_gbuf || !d_params || (!d_color && !d_loss) || (d_loss && !d_target)) return VM_E_INVALID;
  if (n_pixels == 0) return VM_OK;
  const uint32_t grid = vmk::resident_grid(vmk::k_shade_fwd, (n_pixels + 256 * vmk::FPF - 1) / (256 * vmk::FPF));
  vmk::k_shade_fwd<<<grid, 256, 0, (cudaStream_t)stream>>>((const GBuf*)d_gbuf, n_pixels, d_params,
                                                            vmk::shade_consts(consts), d_color, d_target, d_loss);
  return cudaGetLastError() == cudaSuccess ? VM_OK : VM_E_CUDA;
}

extern "C" int vm_shade_backward(const void* d_gbuf, uint64_t n_pixels, const float* d_params,
                                 const vm_shade_consts* consts, const float* d_grad_color, const float* d_target,
                                 double* d_grad_params, double* d_loss, void* stream) {
  if (!d_gbuf || !d_params || !d_grad_params || (!d_grad_color && !d_target)) return VM_E_INVALID;
  if (n_pixels == 0) return VM_OK;
  // the kernel's dynamic shared memory limit, raised once per device
  static std::atomic<uint64_t> attr_set{0};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return VM_E_CUDA;
  const uint64_t bit = 1ull << (dev & 63);
  if ((attr_set.load() & bit) == 0) {
    if (cudaFuncSetAttribute(vmk::k_shade_bwd, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)vmk::BWD_SMEM) !=
        cudaSuccess)
      return VM_E_CUDA;
    attr_set.fetch_or(bit);
  }
  // BWD_WARPS warps per block, each walking runs of 32 x SEG pixels
  const uint32_t grid = vmk::resident_grid(vmk::k_shade_bwd, (n_pixels + 256 * vmk::SEG - 1) / (256 * vmk::SEG),
                                           vmk::BWD_SMEM);
  vmk::k_shade_bwd<<<grid, vmk::BWD_WARPS * 32, vmk::BWD_SMEM, (cudaStream_t)stream>>>(
      (const GBuf*)d_gbuf, n_pixels, d_params, vmk::shade_consts(consts), d_grad_color, d_target, d_grad_params,
      d_loss);
  return cudaGetLastError() == cudaSuccess ? VM_OK : VM_E_CUDA;
}
