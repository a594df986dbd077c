// G-buffer of the differentiable shading stage, sm_100a.
//
// Decodes, once per batch, what the march produced for every pixel into the
// 16-byte vm_shade_gbuf: block id and face of the primary hit, the sun
// shadow's verdict, the water refraction leg's hit and length, the hit
// distance and the fog's optical length per unit density.  The hit distance
// and the ray direction follow the march's exact float contract (this file
// is compiled with --fmad=false like the march), so t matches the oracle bit
// for bit.
#include <cuda_runtime.h>

#include "ray_stages.cuh"
#include "shade.cuh"

namespace vmk {

// e * path of transmittance_from (common.wgsl:1332-1341): the fog's optical
// length per unit density along the primary ray, from the camera height y0,
// the hit distance s and the ray's y direction.
__device__ __forceinline__ float fog_length(float y0, float s, float rdy, const ShadeK& k) {
  const float lambda = k.fog_falloff;
  const float x = fminf(fmaxf(lambda * s * rdy, -60.0f), 60.0f);
  float path = s;
  if (fabsf(x) > 1e-4f) path = s * (1.0f - expf(-x)) / x;
  return expf(-fminf(fmaxf(lambda * (y0 - k.fog_height), -60.0f), 60.0f)) * path;
}

__global__ void __launch_bounds__(256) k_gbuffer(const __grid_constant__ PipeArgs a, ShadeK sk,
                                                 GBuf* __restrict__ out, uint64_t total_px) {
  for (uint64_t gp = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; gp < total_px;
       gp += (uint64_t)gridDim.x * blockDim.x) {
    // view of this pixel: the last view whose pixel offset is <= gp
    uint32_t lo = 0, hi = a.n_views - 1;
    while (lo < hi) {
      const uint32_t mid = (lo + hi + 1) >> 1;
      if (a.views[mid].pix_off <= gp) lo = mid; else hi = mid - 1;
    }
    const vm_frame& f = a.frames[lo];
    const ViewDesc vd = a.views[lo];
    const DevWorld w = {a.chunks + vd.chunk_off, vd.n_chunks, a.inners, a.n_inners, a.leaves, a.n_leaves,
                        a.bricks, a.n_bricks, a.grids + vd.grid_off, vd.grid_len, a.err, a.spec, a.atlas_alpha,
                        a.atlas_layers, {a.tuft_layer[0], a.tuft_layer[1], a.tuft_layer[2]}};
    const uint64_t pix = gp - vd.pix_off;
    GBuf g;
    g.code = 0u; g.t = 0.0f; g.d = 0.0f; g.fog = 0.0f;
    const unsigned long long key = a.vis[gp];
    if (key != 0ull) {
      const uint32_t px = (uint32_t)(pix % f.res[0]), py = (uint32_t)(pix / f.res[0]);
      const F3 rd = ray_dir(f, (float)px + 0.5f, (float)py + 0.5f);
      const KeyParts k = split_key(key);
      const Chunk c = ld_chunk(w, k.ci);
      const uint32_t id = block_at(w, c, k.vx, k.vy, k.vz);
      g.t = hit_t(f, c, k.vx, k.vy, k.vz, k.mx, k.my, k.mz, k.nid, rd);
      g.fog = fog_length(f.cam_pos[1], g.t, rd.y, sk);
      const float sh = a.shadow[gp];
      g.code = (id & 0xFFu) | (k.nid << 8) | G_HIT | (sh == 0.0f ? G_LIT : 0u);
      if ((a.spec & VM_SPEC_SOFT_RAYS) != 0u)   // the blocked fraction of VM_SOFT_SAMPLES rays
        g.code |= G_SOFT | ((uint32_t)(sh * (float)VM_SOFT_SAMPLES + 0.5f) << G_SOFT_SHIFT);
      // cross-quad normals face the ray (shadow.wgsl:23)
      if (k.nid >= VM_NORMAL_CROSS_A && dot(normal_of(k.nid), rd) > 0.0f) g.code |= G_FLIP;
      const unsigned long long s2 = a.sec_key[gp];
      if (id == VM_WATER && (s2 >> 63)) {
        g.code |= G_TRACED;
        g.d = a.sec_t[gp];
        if ((s2 >> 62) & 1ull) {
          const KeyParts k2 = split_key(s2);
          const Chunk c2 = ld_chunk(w, k2.ci);
          const uint32_t id2 = block_at(w, c2, k2.vx, k2.vy, k2.vz);
          g.code |= G_HIT2 | ((id2 & 0xFFu) << 16) | ((k2.nid & 7u) << 24);
        }
      }
    }
    out[gp] = g;
  }
}

}  // namespace vmk

// defined in capi.cu: the batch's pipeline arguments
int vm_internal_batch_args(vm_ctx* ctx, vmk::PipeArgs* out, uint64_t* pixels, void** stream);

extern "C" int vm_shade_gbuffer(vm_ctx* ctx, const vm_shade_consts* consts, void* d_gbuf) {
  if (!ctx || !d_gbuf) return VM_E_INVALID;
  vmk::PipeArgs a;
  uint64_t px = 0;
  void* stream = nullptr;
  int rc = vm_internal_batch_args(ctx, &a, &px, &stream);
  if (rc) return rc;
  if (px == 0) return VM_OK;
  const uint32_t grid = vmk::resident_grid(vmk::k_gbuffer, (px + 255) / 256);
  vmk::k_gbuffer<<<grid, 256, 0, (cudaStream_t)stream>>>(a, vmk::shade_consts(consts), (vmk::GBuf*)d_gbuf, px);
  return cudaGetLastError() == cudaSuccess ? VM_OK : VM_E_CUDA;
}
