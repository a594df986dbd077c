// k_resolve: the colour of every sky and opaque-surface pixel of a rendered
// frame (lane 0 of the engine's resolve pass, resolve.wgsl:1378-1466), from
// the frame's visibility keys and sun visibility.  One thread per pixel, a
// warp per 32 pixels of a row: the key loads and colour stores coalesce, the
// material lookups (chunk records, light bricks, tree nodes, atlas, probe
// field, shaft envelope) are L2-resident gathers.  Bound: instruction issue
// (transcendentals, the 9-sample light gather, the noise octaves).
#include "resolve.cuh"
#include "kernels.cuh"

namespace vmd {

__device__ __noinline__ F3 shade_surface(const DevWorld& w, const vm_frame& f, const Look& L, uint32_t ci, uint32_t vx, uint32_t vy,
                            uint32_t vz, uint32_t id, uint32_t nid, F3 hit, F3 rd, float dist, float lit_in) {
  const Chunk c = ld_chunk(w, ci);
  const float vs = c.vs;
  const bool foliage = nid >= VM_NORMAL_CROSS_A;
  F3 n = normal_of(nid);
  if (foliage && dot(n, rd) > 0.0f) n = neg(n);
  const F3 sun = ld3(f.sun_dir);
  F3 spec_pre = {0.0f, 0.0f, 0.0f};
  if ((L.spec_hi & HI_SKY_SPECULAR) != 0u)
    spec_pre = sky_base(f, L, reflect(rd, n), 1.0f) * schlick_ground(clampf(dot(n, neg(rd)), 0.0f, 1.0f));
  const uint32_t axis = nid >> 1u;
  const F3 box_min = ld3(c.origin) + f3((float)vx, (float)vy, (float)vz) * vs;
  const F3 lq = (hit - box_min) / vs;
  const F3 local = {clampf(lq.x, 0.0f, 1.0f), clampf(lq.y, 0.0f, 1.0f), clampf(lq.z, 0.0f, 1.0f)};
  const uint32_t fi = id * 8u + nid;
  const uint32_t face_word = fi < L.n_faces ? __ldg(L.faces + fi) : 0u;
  const uint32_t layer = face_word & 0xFFFFu;
  float u, v;
  face_uv(nid, local, &u, &v);
  if ((f.flags & VM_FLAG_TEX_VARIATION) != 0u) permute_uv(&u, &v, face_word >> 16u, perm_key(box_min, nid));
  float fa, fb;
  int32_t ta[3] = {0, 0, 0}, tb[3] = {0, 0, 0};
  if (axis == 0u) { fa = local.y; fb = local.z; ta[1] = 1; tb[2] = 1; }
  else if (axis == 1u) { fa = local.x; fb = local.z; ta[0] = 1; tb[2] = 1; }
  else { fa = local.x; fb = local.y; ta[0] = 1; tb[1] = 1; }
  const float grazing = fmaxf(fabsf(dot(n, rd)), 0.25f);
  const float footprint = fmaxf(dist, 1e-3f) * 2.0f * f.tan_half_fov / (float)f.res[1] * 16.0f / vs / grazing;
  const float lod = clampf(log2f(fmaxf(footprint, 1e-4f)) + f.mip_bias, 0.0f, 3.0f);
  const float4 texel = atlas_sample(L, u, v, layer, lod);
  F3 albedo = {texel.x, texel.y, texel.z};
  const float tint_mask = foliage ? 1.0f : texel.w;
  if ((f.flags & VM_FLAG_TINT) != 0u && tint_mask > 0.0f) {
    const float k = tint_mask * f.tint_strength;
    albedo = albedo * mix3(f3(1.0f, 1.0f, 1.0f), biome_tint(f, L, hit.x, hit.z), k);
  }
  if ((L.spec_hi & HI_SHORE_WET) != 0u && id == VM_SAND) {
    const float wet = 1.0f - smoothstep(f.sea_level, f.sea_level + 1.5f, hit.y);
    albedo = albedo * mixf(1.0f, 0.62f, wet);
  }
  if ((L.spec_hi & HI_FOLIAGE_RICH) != 0u && (foliage || ((id == VM_GRASS || id == VM_MEADOW) && nid == VM_NORMAL_PY))) {
    const float hr = hash_alpha(box_min);
    const float hv = hash_alpha(box_min + f3(17.31f, 7.77f, 3.03f));
    F3 rich = {1.0f, 1.0f, 1.0f};
    if (hr < 0.16f) rich = f3(1.30f, 1.10f, 0.55f);
    else if (hr > 0.97f) rich = f3(1.35f, 0.72f, 0.95f);
    albedo = albedo * rich * mixf(0.88f, 1.10f, hv);
  }
  if ((L.spec_hi & HI_CANOPY_RELIEF) != 0u && is_cutout_id(id)) {
    const float clump = cloud_noise(box_min.x * 0.21f + box_min.y * 0.313f, box_min.z * 0.21f + box_min.y * 0.173f);
    const float relief = mixf(0.72f, 1.34f, clump * clump);
    const float micro = mixf(0.92f, 1.08f, hash_alpha(box_min));
    const float toward_sun = clampf(dot(n, sun) * 0.5f + 0.5f, 0.0f, 1.0f);
    albedo = albedo * relief * micro * mixf(0.84f, 1.0f, toward_sun);
  }
  const F3 sky_tint = surface_sky_fill(f, L, n);
  const bool light_rgb = (f.flags & VM_FLAG_LIGHT_RGB) != 0u;
  const bool gather = (w.spec & VM_SPEC_EMITTER_GATHER) != 0u;
  float ao = 1.0f, sky_sm = 0.0f;
  F3 amb = {0.0f, 0.0f, 0.0f};
  const int32_t nx = (int32_t)n.x, ny = (int32_t)n.y, nz = (int32_t)n.z;   // axis normals only (foliage below)
  if (foliage) {
    const uint32_t packed = light_at(w, c, (int32_t)vx, (int32_t)vy, (int32_t)vz);
    const float sk = light_curve(light_sky(packed)) * f.daylight;
    sky_sm = sk;
    if (light_rgb) {
      amb = block_ambient(light_curve3(light_block_rgb(packed)), sk, sky_tint);
    } else {
      const float bk = light_curve(light_block_level(packed));
      amb = mix3(sky_tint, block_tint(), bk / fmaxf(sk + bk, 1e-4f)) * fmaxf(sk, bk);
    }
  } else {
    const F3 air_c = box_min + f3(0.5f * vs, 0.5f * vs, 0.5f * vs) + n * vs;
    const F3 step_a = f3((float)ta[0], (float)ta[1], (float)ta[2]) * vs;
    const F3 step_b = f3((float)tb[0], (float)tb[1], (float)tb[2]) * vs;
    const int32_t ax = (int32_t)vx + nx, ay = (int32_t)vy + ny, az = (int32_t)vz + nz;
    const int32_t sx = ta[0] + tb[0], sy = ta[1] + tb[1], sz = ta[2] + tb[2];
    const bool local_only = ax - sx >= 0 && ay - sy >= 0 && az - sz >= 0 && ax + sx <= 63 && ay + sy <= 63 &&
                            az + sz <= 63;
    uint2 nb[9];
    if (local_only) {
      gather_face(w, c, ax, ay, az, ta[0], ta[1], ta[2], tb[0], tb[1], tb[2], nb);
    } else {
#pragma unroll 1
      for (int i = 0; i < 9; ++i)
        nb[i] = world_sample(w, f, air_c + step_a * ((float)(i % 3) - 1.0f) + step_b * ((float)(i / 3) - 1.0f));
    }
    float sky_n[9], blk_n[9], open_n[9];
    uint32_t any_blk = 0u;
#pragma unroll
    for (int i = 0; i < 9; ++i) {
      sky_n[i] = light_curve(light_sky(nb[i].x)) * f.daylight;
      if (light_rgb) {
        if (gather) any_blk |= nb[i].x & 0xFFFu;
        blk_n[i] = 0.0f;
      } else {
        blk_n[i] = light_curve(light_block_level(nb[i].x));
      }
      open_n[i] = 1.0f - (float)nb[i].y;
    }
    F3 blk4 = {0.0f, 0.0f, 0.0f};
    if (gather && light_rgb && any_blk != 0u) blk4 = light_curve3(light_block_rgb(nb[4].x));
    const bool ao_on = (f.flags & VM_FLAG_AO) != 0u;
    F3 amb_c[4];
    float sky_c[4], ao_c[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int ia = 4 + ((k & 1) * 2 - 1);
      const int ib = 4 + ((k >> 1) * 2 - 1) * 3;
      const int ic = ia + ib - 4;
      const float inv = 1.0f / (1.0f + open_n[ia] + open_n[ib] + open_n[ic]);
      const float sk = (sky_n[4] + sky_n[ia] * open_n[ia] + sky_n[ib] * open_n[ib] + sky_n[ic] * open_n[ic]) * inv;
      sky_c[k] = sk;
      if (light_rgb) {
        if (gather && any_blk != 0u) {
          const F3 ba = light_curve3(light_block_rgb(nb[ia].x));
          const F3 bb = light_curve3(light_block_rgb(nb[ib].x));
          const F3 bc = light_curve3(light_block_rgb(nb[ic].x));
          const F3 bkv = (blk4 + ba * open_n[ia] + bb * open_n[ib] + bc * open_n[ic]) * inv;
          amb_c[k] = block_ambient(bkv, sk, sky_tint);
        } else {
          amb_c[k] = sky_tint * sk;
        }
      } else {
        const float bk = (blk_n[4] + blk_n[ia] * open_n[ia] + blk_n[ib] * open_n[ib] + blk_n[ic] * open_n[ic]) * inv;
        amb_c[k] = mix3(sky_tint, block_tint(), bk / fmaxf(sk + bk, 1e-4f)) * fmaxf(sk, bk);
      }
      const float s1 = 1.0f - open_n[ia];
      const float s2 = 1.0f - open_n[ib];
      const float occ = (s1 > 0.5f && s2 > 0.5f) ? 3.0f : s1 + s2 + 1.0f - open_n[ic];
      ao_c[k] = ao_on ? 1.0f - occ * 0.25f : 1.0f;
    }
    ao = mixf(mixf(ao_c[0], ao_c[1], fa), mixf(ao_c[2], ao_c[3], fa), fb);
    sky_sm = mixf(mixf(sky_c[0], sky_c[1], fa), mixf(sky_c[2], sky_c[3], fa), fb);
    amb = mix3(mix3(amb_c[0], amb_c[1], fa), mix3(amb_c[2], amb_c[3], fa), fb);
  }
  float direct = 0.0f;
  const float ndl = dot(n, sun);
  if (ndl > 0.0f && f.daylight > 0.01f) {
    float lit = 1.0f;
    if ((f.flags & VM_FLAG_SHADOWS) != 0u) {
      lit = lit_in;
      if ((f.flags & VM_FLAG_DISTANT_SHADOWS) != 0u && lit > 0.0f)
        lit = lit * terrain_shade(f, L, hit + sun * f.shadow_dist);
    }
    if (lit > 0.0f) {
      const float cloud_fp = fmaxf(dist, 1e-3f) * 2.0f * f.tan_half_fov / (float)f.res[1] * exp2f(f.mip_bias);
      lit = lit * cloud_shade(f, hit, cloud_fp);
    }
    direct = lit * ndl * sky_sm;
    if ((L.spec_hi & HI_CAUSTICS) != 0u) {
      const float cdepth = f.sea_level - hit.y;
      if (cdepth > 0.0f && cdepth < 8.0f && direct > 0.0f) {
        const float k = cdepth / fmaxf(sun.y, 1e-3f);
        const float spx = hit.x - sun.x * k, spz = hit.z - sun.z * k;
        const float a = f.wave_amp, l0 = f.wave_scale, ph = f.time * f.wave_speed * WAVE_TAU;
        const F3 g0 = wave_octave(spx, spz, 0.913089f, 0.407760f, l0, a * 0.42f, ph, 0.35f, 0.0f, 0.0f, 0.0f, false);
        const F3 g1 = wave_octave(spx, spz, -0.388685f, 0.921371f, l0 / 2.17f, a * 0.27f, ph * 1.4731f, 0.35f, 0.0f,
                                  0.0f, 0.0f, false);
        const float r0 = g0.x * g0.x + g0.y * g0.y;
        const float r1 = g1.x * g1.x + g1.y * g1.y;
        const float sheets = r0 * r1 * 4000.0f;
        direct = direct * (1.0f + sheets * expf(-cdepth * 0.30f));
      }
    }
  }
  const bool probe_cube = (f.flags & VM_FLAG_PROBE_CUBE) != 0u, probe_bounce = (f.flags & VM_FLAG_PROBE_BOUNCE) != 0u;
  float4 probe = make_float4(1.0f, 1.0f, 1.0f, 1.0f);
  if (probe_cube || probe_bounce) probe = probe_field(L, hit + n * 2.0f, nid);
  const bool repair = lighting_repair(L);
  float shade = repair ? 1.0f : face_shade(nid);
  if (probe_cube) shade = shade * probe.w;
  const F3 ambient_rgb = amb * 0.50f;
  const F3 sun_rgb = f3(1.0000f, 0.8469f, 0.5647f) * (direct * (repair ? 0.78f : 0.52f));
  F3 floor_rgb = f3(0.85f, 0.90f, 1.00f) * f.ambient;
  const F3 probe_rgb = {probe.x, probe.y, probe.z};
  if (probe_bounce) floor_rgb = floor_rgb * probe_rgb;
  if ((f.flags & VM_FLAG_PROBE_SUN) != 0u) {
    const float gain = (f.flags & VM_FLAG_PROBE_SUN_HIGH) != 0u ? 0.25f : 0.10f;
    floor_rgb = floor_rgb + f3(0.85f, 0.90f, 1.00f) * probe_rgb * (gain * sky_sm);
  }
  const F3 spec_rgb = spec_pre * (sky_sm * 0.5f);
  // surface_light / surface_radiance: resolve.wgsl:7-17
  const F3 light = repair ? ambient_rgb * ao * shade + sun_rgb + floor_rgb
                          : ((ambient_rgb + sun_rgb) * ao + floor_rgb) * shade;
  if (repair && id == VM_GLOWSTONE) return albedo * (f3(1.0f, 0.7111f, 0.3024f) * 1.5f + light * 0.15f);
  return albedo * light + spec_rgb;
}

}  // namespace vmd

namespace vmk {
using namespace vmd;

// The sun visibility the resolve reads (primary_sun, the shadow pass's r8unorm
// mask): the soft-shadow mask when one was made, else 1 - blocked from the
// blocker distance; stored through the r8unorm target's rounding.
__device__ __forceinline__ float sun_visibility(const float* mask, const float* dist, bool soft, uint64_t pix) {
  const float m = mask != nullptr ? mask[pix] : (soft ? 1.0f - dist[pix] : (dist[pix] > 0.0f ? 0.0f : 1.0f));
  return floorf(clampf(m, 0.0f, 1.0f) * 255.0f + 0.5f) / 255.0f;
}

// SKY: the pass over the sky pixels (sky_color with clouds and the sun
// shafts), else the pass over the opaque surfaces.  Two launches over the
// frame instead of one with both paths: each kernel's code is half the size
// (the single kernel stalled on instruction fetch) and a warp runs one path.
template <bool SKY>
__global__ void __launch_bounds__(128, 8) k_resolve(const __grid_constant__ vm_frame f, const __grid_constant__ DevWorld w,
                                                    const __grid_constant__ Look L,
                                                    const unsigned long long* __restrict__ vis,
                                                    const float* __restrict__ mask, const float* __restrict__ dist,
                                                    bool soft, float4* __restrict__ out) {
  const uint32_t px = blockIdx.x * 32u + threadIdx.x, py = blockIdx.y * 4u + threadIdx.y;
  if (px >= f.res[0] || py >= f.res[1]) return;
  const uint64_t pix = (uint64_t)py * f.res[0] + px;
  const unsigned long long key = vis[pix];
  if ((key == 0ull) != SKY) return;
  const F3 cam = ld3(f.cam_pos);
  const F3 rd = ray_dir(f, (float)px + 0.5f, (float)py + 0.5f);
  F3 color;
  if (SKY) {
    const float shaft = sun_shaft(f, L, cam, rd, f.far_, 1.0f, px, py);
    color = sky_color(f, L, cam, rd, 0.0f, shaft);
  } else {
    const uint32_t nid = (uint32_t)(key >> 37) & 7u;
    const uint32_t ci = (uint32_t)(key >> 24) & 0x1FFFu;
    const uint32_t low = (uint32_t)(key & 0xFFFFFFull);
    const uint32_t vx = (low >> 16) & 63u, vy = (low >> 8) & 63u, vz = low & 63u;
    const uint32_t mx = (low >> 22) & 3u, my = (low >> 14) & 3u, mz = (low >> 6) & 3u;
    const Chunk c = ld_chunk(w, ci);
    const float t = hit_t(f, c, vx, vy, vz, mx, my, mz, nid, rd);
    const F3 hit = cam + rd * t;
    const uint32_t id = block_at(w, c, vx, vy, vz);
    if (id == VM_WATER || ((w.spec & VM_SPEC_GLASS) != 0u && id == VM_GLASS)) {
      out[pix] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);   // the water and glass lanes' pixels
      return;
    }
    color = shade_surface(w, f, L, ci, vx, vy, vz, id, nid, hit, rd, t, sun_visibility(mask, dist, soft, pix));
    const float alpha = 1.0f - transmittance_from(f, cam.y, t, rd);
    const float shaft = sun_shaft(f, L, cam, rd, t, alpha, px, py);
    color = mix3(color, sky_base(f, L, rd, shaft), alpha);
  }
  out[pix] = make_float4(color.x, color.y, color.z, 1.0f);
}

cudaError_t launch_resolve(const vm_frame& f, const DevWorld& w, const Look& L, const unsigned long long* vis,
                           const float* mask, const float* dist, bool soft_rays, float4* out, cudaStream_t s) {
  const dim3 block(32, 4), grid((f.res[0] + 31u) / 32u, (f.res[1] + 3u) / 4u);
  k_resolve<false><<<grid, block, 0, s>>>(f, w, L, vis, mask, dist, soft_rays, out);
  k_resolve<true><<<grid, block, 0, s>>>(f, w, L, vis, mask, dist, soft_rays, out);
  return cudaGetLastError();
}

}  // namespace vmk
