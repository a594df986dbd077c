// The G-buffer of the differentiable shading stage and the constants of its
// model, shared by the G-buffer pass (gbuffer.cu, compiled with the march's
// exact float contract) and the forward / adjoint kernels (shade.cu).
#pragma once
#include <cstdint>

#include "../../include/voxmarch.h"
#include "kernels.cuh"
#include "march_device.cuh"

namespace vmk {
using namespace vmd;

constexpr int NP = VM_SHADE_NPARAMS;   // 256*3 albedo + sun 3 + sky 3 + fog 1 + absorb 3
constexpr int P_SUN = 768, P_SKY = 771, P_FOG = 774, P_ABS = 775;
constexpr uint32_t G_HIT = 1u << 11, G_LIT = 1u << 12, G_TRACED = 1u << 13, G_HIT2 = 1u << 14, G_FLIP = 1u << 15;
// soft shadows: G_SOFT set and the number of blocked jittered rays in bits 27-29
constexpr uint32_t G_SOFT = 1u << 30, G_SOFT_SHIFT = 27;

struct __align__(16) GBuf {   // vm_shade_gbuf: one 128-bit load per pixel
  uint32_t code;
  float t, d, fog;
};
static_assert(sizeof(GBuf) == VM_SHADE_GBUF_BYTES, "GBuf is vm_shade_gbuf");
static_assert(sizeof(GBuf) == sizeof(vm_shade_gbuf), "GBuf is vm_shade_gbuf");

struct ShadeK {            // constants of the model
  float sun_rgb[3];
  float fog_falloff, fog_height;
};

inline ShadeK shade_consts(const vm_shade_consts* c) {
  ShadeK k;
  const float sun[3] = {1.0f, 0.8469f, 0.5647f};   // resolve.wgsl:787, times the 0.78 gain
  for (int i = 0; i < 3; ++i) k.sun_rgb[i] = c ? c->sun_rgb[i] : sun[i] * 0.78f;
  k.fog_falloff = c ? c->fog_falloff : 0.0f;
  k.fog_height = c ? c->fog_height : 0.0f;
  return k;
}

// One wave: the SM count times the blocks of 256 threads an SM holds, or
// fewer when the work needs fewer.
template <class K>
inline uint32_t resident_grid(K kernel, uint64_t blocks_needed, size_t dyn_smem = 0) {
  int dev = 0, sms = 148, per_sm = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, 256, dyn_smem);
  const uint64_t cap = (uint64_t)sms * (uint64_t)(per_sm > 0 ? per_sm : 1);
  return (uint32_t)(blocks_needed < 1 ? 1 : (blocks_needed < cap ? blocks_needed : cap));
}

}  // namespace vmk
