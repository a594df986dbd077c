// k_resolve: the colour of every sky and opaque-surface pixel of a rendered
// frame (lane 0 of the engine's resolve pass, resolve.wgsl:1378-1466), from
// the frame's visibility keys and sun visibility.  One thread per pixel, a
// warp per 32 pixels of a row: the key loads and colour stores coalesce, the
// material lookups (chunk records, light bricks, tree nodes, atlas, probe
// field, shaft envelope) are L2-resident gathers.  Bound: instruction issue
// (transcendentals, the 9-sample light gather, the noise octaves).
#include "resolve.cuh"
#include "kernels.cuh"
#include "ray_stages.cuh"

namespace vmd {

// The light terms of a surface hit (resolve.wgsl:617-747 of shade_hit), from
// the light word of a foliage voxel, the one voxel in front of the face (flat
// secondaries) or the 3x3 gather with AO (smooth light).
static __device__ __noinline__ LightTerms surface_light_terms(const DevWorld& w, const vm_frame& f, const Look& L,
                                                              uint32_t ci, uint32_t vx, uint32_t vy, uint32_t vz,
                                                              uint32_t nid, F3 n, F3 hit, bool smooth) {
  const Chunk c = ld_chunk(w, ci);
  const float vs = c.vs;
  const bool foliage = nid >= VM_NORMAL_CROSS_A;
  const uint32_t axis = nid >> 1u;
  const F3 box_min = ld3(c.origin) + f3((float)vx, (float)vy, (float)vz) * vs;
  const F3 lq = (hit - box_min) / vs;
  const F3 local = {clampf(lq.x, 0.0f, 1.0f), clampf(lq.y, 0.0f, 1.0f), clampf(lq.z, 0.0f, 1.0f)};
  float fa, fb;
  int32_t ta[3] = {0, 0, 0}, tb[3] = {0, 0, 0};
  if (axis == 0u) { fa = local.y; fb = local.z; ta[1] = 1; tb[2] = 1; }
  else if (axis == 1u) { fa = local.x; fb = local.z; ta[0] = 1; tb[2] = 1; }
  else { fa = local.x; fb = local.y; ta[0] = 1; tb[1] = 1; }
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
      amb = mix3(sky_tint, block_tint(), wdiv(bk, fmaxf(sk + bk, 1e-4f))) * fmaxf(sk, bk);
    }
  } else if (!smooth) {
    // one light sample: the voxel in front of the face, in this chunk or
    // through the grid
    const int32_t ax = (int32_t)vx + nx, ay = (int32_t)vy + ny, az = (int32_t)vz + nz;
    uint32_t packed1;
    if (ax >= 0 && ay >= 0 && az >= 0 && ax <= 63 && ay <= 63 && az <= 63)
      packed1 = light_at(w, c, ax, ay, az);
    else
      packed1 = world_sample(w, f, box_min + f3(0.5f * vs, 0.5f * vs, 0.5f * vs) + n * vs).x;
    const float sk1 = light_curve(light_sky(packed1)) * f.daylight;
    sky_sm = sk1;
    if (light_rgb) {
      amb = block_ambient(light_curve3(light_block_rgb(packed1)), sk1, sky_tint);
    } else {
      const float bk1 = light_curve(light_block_level(packed1));
      amb = mix3(sky_tint, block_tint(), wdiv(bk1, fmaxf(sk1 + bk1, 1e-4f))) * fmaxf(sk1, bk1);
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
      const float inv = wdiv(1.0f, 1.0f + open_n[ia] + open_n[ib] + open_n[ic]);
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
        amb_c[k] = mix3(sky_tint, block_tint(), wdiv(bk, fmaxf(sk + bk, 1e-4f))) * fmaxf(sk, bk);
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
  return {amb, sky_sm, ao};
}

template <bool EXTRA>
__device__ __noinline__ F3 shade_surface(const DevWorld& w, const vm_frame& f, const Look& L, uint32_t ci, uint32_t vx,
                                         uint32_t vy, uint32_t vz, uint32_t id, uint32_t nid, F3 hit, F3 rd, float dist,
                                         float shadow_dist, bool smooth, bool do_spec, float lit_in,
                                         const LightTerms* pre) {
  const Chunk c = ld_chunk(w, ci);
  const float vs = c.vs;
  const bool foliage = nid >= VM_NORMAL_CROSS_A;
  F3 n = normal_of(nid);
  if (foliage && dot(n, rd) > 0.0f) n = neg(n);
  const F3 sun = ld3(f.sun_dir);
  F3 spec_pre = {0.0f, 0.0f, 0.0f};
  if ((L.spec_hi & HI_SKY_SPECULAR) != 0u && do_spec)
    spec_pre = sky_base(f, L, reflect(rd, n), 1.0f) * schlick_ground(clampf(dot(n, neg(rd)), 0.0f, 1.0f));
  const F3 box_min = ld3(c.origin) + f3((float)vx, (float)vy, (float)vz) * vs;
  const F3 lq = (hit - box_min) / vs;
  const F3 local = {clampf(lq.x, 0.0f, 1.0f), clampf(lq.y, 0.0f, 1.0f), clampf(lq.z, 0.0f, 1.0f)};
  const uint32_t fi = id * 8u + nid;
  const uint32_t face_word = fi < L.n_faces ? __ldg(L.faces + fi) : 0u;
  const uint32_t layer = face_word & 0xFFFFu;
  float u, v;
  face_uv(nid, local, &u, &v);
  if ((f.flags & VM_FLAG_TEX_VARIATION) != 0u) permute_uv(&u, &v, face_word >> 16u, perm_key(box_min, nid));
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
    const float wet = 1.0f - wsmooth(f.sea_level, f.sea_level + 1.5f, hit.y);
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
  LightTerms lt;
  if (pre != nullptr) lt = *pre;
  else lt = surface_light_terms(w, f, L, ci, vx, vy, vz, nid, n, hit, smooth);
  F3 amb = lt.amb;
  const float sky_sm = lt.sky_sm, ao = lt.ao;
  // SPEC_PROBE_AMBIENT / SPEC_PROBE_TAP (resolve.wgsl:500-505): the ambient
  // from the probe tap alone (the light words' ambient unused), or scaled by it
  const bool probe_ambient = EXTRA && (f.flags & VM_FLAG_PROBE_AMBIENT) != 0u;
  if (probe_ambient) amb = probe_tap(L, hit);
  else if (EXTRA && (f.flags & VM_FLAG_PROBE_TAP) != 0u) amb = amb * probe_tap(L, hit);
  float direct = 0.0f, visibility = 1.0f;
  const float ndl = dot(n, sun);
  if (ndl > 0.0f && f.daylight > 0.01f) {
    float lit = 1.0f;
    if ((f.flags & VM_FLAG_SHADOWS) != 0u) {
      lit = lit_in >= 0.0f ? lit_in : (shadow_ray_hit(w, f, hit + n * (0.02f * vs), sun, shadow_dist) ? 0.0f : 1.0f);
      if ((f.flags & VM_FLAG_DISTANT_SHADOWS) != 0u && lit > 0.0f)
        lit = lit * terrain_shade(f, L, hit + sun * shadow_dist);
    }
    if (lit > 0.0f) {
      const float cloud_fp = fmaxf(dist, 1e-3f) * 2.0f * f.tan_half_fov / (float)f.res[1] * exp2f(f.mip_bias);
      lit = lit * cloud_shade(f, hit, cloud_fp);
    }
    visibility = lit;
    direct = lit * ndl * sky_sm;
    if ((L.spec_hi & HI_CAUSTICS) != 0u) {
      const float cdepth = f.sea_level - hit.y;
      if (cdepth > 0.0f && cdepth < 8.0f && direct > 0.0f) {
        const float k = wdiv(cdepth, fmaxf(sun.y, 1e-3f));
        const float spx = hit.x - sun.x * k, spz = hit.z - sun.z * k;
        const float a = f.wave_amp, l0 = f.wave_scale, ph = f.time * f.wave_speed * WAVE_TAU;
        const F3 g0 = wave_octave(spx, spz, 0.913089f, 0.407760f, l0, a * 0.42f, ph, 0.35f, 0.0f, 0.0f, 0.0f, false);
        const F3 g1 = wave_octave(spx, spz, -0.388685f, 0.921371f, l0 / 2.17f, a * 0.27f, ph * 1.4731f, 0.35f, 0.0f,
                                  0.0f, 0.0f, false);
        const float r0 = g0.x * g0.x + g0.y * g0.y;
        const float r1 = g1.x * g1.x + g1.y * g1.y;
        const float sheets = r0 * r1 * 4000.0f;
        direct = direct * (1.0f + sheets * wexp(-cdepth * 0.30f));
      }
    }
  }
  const bool probe_cube = (f.flags & VM_FLAG_PROBE_CUBE) != 0u, probe_bounce = (f.flags & VM_FLAG_PROBE_BOUNCE) != 0u;
  float4 probe = make_float4(1.0f, 1.0f, 1.0f, 1.0f);
  if (!probe_ambient && (probe_cube || probe_bounce)) probe = probe_field(L, hit + n * 2.0f, nid);
  const bool repair = lighting_repair(L);
  float shade = 1.0f;
  if (!probe_ambient) {
    shade = repair ? 1.0f : face_shade(nid);
    if (probe_cube) shade = shade * probe.w;
  }
  const F3 ambient_rgb = amb * 0.50f;
  const F3 sun_rgb = f3(1.0000f, 0.8469f, 0.5647f) * (direct * (repair ? 0.78f : 0.52f));
  F3 floor_rgb = {0.0f, 0.0f, 0.0f};
  if (!probe_ambient) {
    floor_rgb = f3(0.85f, 0.90f, 1.00f) * f.ambient;
    const F3 probe_rgb = {probe.x, probe.y, probe.z};
    if (probe_bounce) floor_rgb = floor_rgb * probe_rgb;
    if ((f.flags & VM_FLAG_PROBE_SUN) != 0u) {
      const float gain = (f.flags & VM_FLAG_PROBE_SUN_HIGH) != 0u ? 0.25f : 0.10f;
      floor_rgb = floor_rgb + f3(0.85f, 0.90f, 1.00f) * probe_rgb * (gain * sky_sm);
    }
  }
  // SURFACE_DEBUG 1-4 (resolve.wgsl:579-582): normal, sun visibility, sun, ambient
  if (EXTRA) {
    const uint32_t debug_view = surface_debug(L);
    if (debug_view == 1u) return add_s(n * 0.5f, 0.5f);
    if (debug_view == 2u) return f3(visibility, visibility, visibility);
    if (debug_view == 3u) return sun_rgb;
    if (debug_view == 4u) return ambient_rgb * ao + floor_rgb;
  }
  const F3 spec_rgb = spec_pre * (sky_sm * 0.5f);
  // surface_light / surface_radiance: resolve.wgsl:7-17
  const F3 light = repair ? ambient_rgb * ao * shade + sun_rgb + floor_rgb
                          : ((ambient_rgb + sun_rgb) * ao + floor_rgb) * shade;
  if (repair && id == VM_GLOWSTONE) return albedo * (f3(1.0f, 0.7111f, 0.3024f) * 1.5f + light * 0.15f);
  return albedo * light + spec_rgb;
}


// ---------------------------------------------------------------------------
// the water and glass lanes: resolve.wgsl:896-1320

constexpr uint32_t HI_SHORE_FOAM = 16u, HI_WATER_SEC = 32u, HI_GLASS_REFLECT = 128u, HI_WATER_LOOK = 4096u;
constexpr float WATER_LOOK_RIPPLE_AMP = 0.16f;

// look_ripple: resolve.wgsl:995-1008, the water look's two short ripples
// (gradient), phase-warped under SPEC_WATER_REPAIR
static __device__ __noinline__ float2 look_ripple(const DevWorld& w, float px, float pz, float time, float w1,
                                                  float w2) {
  const float d1x = 0.86f, d1z = 0.51f, d2x = -0.42f, d2z = 0.91f;
  const float k1 = (float)(6.2832 / 1.15), k2 = (float)(6.2832 / 0.62);   // abstract-float constants, folded first
  float ph_x = 0.0f, ph_z = 0.0f;
  if ((w.spec & VM_SPEC_WATER_REPAIR) != 0u) {
    ph_x = sinf(px * 0.071f + pz * 0.113f) * 2.0f;
    ph_z = sinf(px * -0.097f + pz * 0.053f + 1.9f) * 2.0f;
  }
  const float a1 = cosf((px * d1x + pz * d1z) * k1 + time * 1.7f + ph_x) * w1;
  const float a2 = cosf((px * d2x + pz * d2z) * k2 - time * 2.3f + ph_z) * w2;
  return make_float2(d1x * a1 + d2x * a2, d1z * a1 + d2z * a2);
}
constexpr float WATER_SHADOW_DIST = 16.0f;    // SPEC_WATER_SHADOW_DIST
constexpr float GLASS_SHADOW_DIST = 48.0f;

__device__ __forceinline__ bool secondary_smooth(const vm_frame& f) { return (f.flags & VM_FLAG_FLAT_SECONDARY) == 0u; }

__device__ __forceinline__ float medium_light(const vm_frame& f, uint32_t packed) {
  const float sky_l = light_curve(light_sky(packed)) * f.daylight;
  const float blk_l = light_curve(light_block_level(packed));
  return fmaxf(sky_l, blk_l) * 0.50f + f.ambient;
}

// water_medium: common.wgsl:1262-1265 (WATER_EXT per channel)
__device__ __forceinline__ F3 water_medium(const vm_frame& f, F3 c, float d, F3 body) {
  const float dd = fmaxf(d, 0.0f);
  const F3 tr = {wexp(-0.280f * f.water_absorb * dd), wexp(-0.055f * f.water_absorb * dd),
                 wexp(-0.020f * f.water_absorb * dd)};
  return c * tr + body * f3(1.0f - tr.x, 1.0f - tr.y, 1.0f - tr.z);
}
__device__ __forceinline__ float schlick_f0(float f0, float cos_i) {   // schlick / schlick_glass
  const float m = clampf(1.0f - cos_i, 0.0f, 1.0f);
  const float m2 = m * m;
  return f0 + (1.0f - f0) * m2 * m2 * m;
}

struct WaterCtx {
  F3 body; float ml;
  F3 n, nw, nt;
  float gloss; bool waved;
  float refract_detail, reflect_detail;
  F3 mirror, mirror_t, hit, rd;
  float t, roughness;
};

// water_ctx: resolve.wgsl:1078-1166 (SPEC_WATER_LOOK off)
static __device__ __noinline__ WaterCtx water_ctx(const DevWorld& w, const vm_frame& f, const Look& L, uint32_t ci,
                                                  uint32_t vx, uint32_t vy, uint32_t vz, uint32_t nid, F3 hit, F3 rd,
                                                  float t) {
  WaterCtx x;
  const Chunk c = ld_chunk(w, ci);
  const float vs = c.vs;
  const F3 n = normal_of(nid);
  const F3 box_min = ld3(c.origin) + f3((float)vx, (float)vy, (float)vz) * vs;
  const F3 lq = (hit - box_min) / vs;
  const F3 local = {clampf(lq.x, 0.0f, 1.0f), clampf(lq.y, 0.0f, 1.0f), clampf(lq.z, 0.0f, 1.0f)};
  const float footprint = fmaxf(t, 1e-3f) * 2.0f * f.tan_half_fov / (float)f.res[1] * 16.0f / vs;
  const float lod = clampf(log2f(fmaxf(footprint, 1e-4f)) + f.mip_bias, 0.0f, 3.0f);
  const uint32_t fi = VM_WATER * 8u + nid;
  const uint32_t layer = (fi < L.n_faces ? __ldg(L.faces + fi) : 0u) & 0xFFFFu;
  float u, v;
  face_uv(nid, local, &u, &v);
  float4 tint = atlas_sample(L, u, v, layer, lod);
  if ((w.spec & VM_SPEC_WATER_REPAIR) != 0u) tint = atlas_sample(L, 0.5f, 0.5f, layer, 3.0f);
  x.ml = medium_light(f, light_at(w, c, (int32_t)vx, (int32_t)vy, (int32_t)vz));
  x.body = f3(tint.x, tint.y, tint.z) * x.ml;
  x.refract_detail = 1.0f - smoothstep(VM_WATER_REFRACT_NEAR, VM_WATER_REFRACT_FAR, t);
  x.reflect_detail = 1.0f - smoothstep(VM_WATER_REFLECT_NEAR, VM_WATER_REFLECT_FAR, t);
  const float px_world = fmaxf(t, 1e-3f) * 2.0f * f.tan_half_fov / (float)f.res[1];
  F3 nw = n, nt = n;
  float gloss = 1.0f, unresolved = 0.0f;
  const bool waved = (f.flags & VM_FLAG_WAVES) != 0u && nid == VM_NORMAL_PY;
  if (waved) {
    float kk = 0.0f, vhx = 0.0f, vhz = 0.0f;
    const bool aniso = (f.flags & VM_FLAG_WAVE_ANISO) != 0u;
    if (aniso) {
      const float k = 1.0f / fmaxf(fabsf(rd.y), WAVE_GRAZE_MIN);
      kk = k * k - 1.0f;
      const float r = 1.0f / sqrtf(fmaxf(rd.x * rd.x + rd.z * rd.z, 1e-12f));
      vhx = rd.x * r; vhz = rd.z * r;
    }
    float shoal = 1.0f;
    if ((f.flags & VM_FLAG_WAVE_SHOAL) != 0u) {
      const F3 dro = {floorf(hit.x) + 0.5f, hit.y - VM_SURFACE_EPS, floorf(hit.z) + 0.5f};
      const WorldHit dh = trace_world<true, false, true>(w, f, dro, f3(0.001f, -0.999999f, 0.001f), SHOAL_DEPTH,
                                                          nullptr);
      shoal = smoothstep(0.0f, SHOAL_DEPTH, dh.hit ? dh.t : SHOAL_DEPTH);
    }
    const F3 wf = wave_field(f, hit.x, hit.z, px_world, vhx, vhz, kk, aniso, shoal);
    unresolved = fmaxf(wf.z, 0.0f);
    nw = unit(f3(-wf.x, 1.0f, -wf.y));
    const float gl = sqrtf(wf.x * wf.x + wf.y * wf.y);
    const float lim = fminf(1.0f, f.wave_reflect_slope / fmaxf(gl, 1e-6f));
    nt = unit(f3(-(wf.x * lim), 1.0f, -(wf.y * lim)));
    gloss = wdiv(1.0f, 1.0f + 0.5f * 320.0f * wf.z);
  }
  if ((L.spec_hi & HI_WATER_LOOK) != 0u && nid == VM_NORMAL_PY) {
    // SPEC_WATER_LOOK (resolve.wgsl:1138-1153): sub-pixel ripples on the
    // mirror normal, their unresolved part added to the optical roughness
    const float pix = px_world / fmaxf(fabsf(rd.y), WAVE_GRAZE_MIN);
    const float range_gate = (1.0f - smoothstep(48.0f, 96.0f, t)) * smoothstep(0.08f, 0.20f, fabsf(rd.y));
    const float fade_115 = range_gate * smoothstep(2.0f, 4.0f, 1.15f / fmaxf(pix, 1e-4f));
    const float fade_62 = range_gate * smoothstep(2.0f, 4.0f, 0.62f / fmaxf(pix, 1e-4f));
    unresolved += WATER_LOOK_RIPPLE_AMP * WATER_LOOK_RIPPLE_AMP * 0.5f *
                  (0.36f * (1.0f - fade_115 * fade_115) + 0.16f * (1.0f - fade_62 * fade_62));
    const float2 rp = look_ripple(w, hit.x, hit.z, f.time * f.wave_speed, 0.60f * fade_115, 0.40f * fade_62);
    nw = unit(nw + f3(rp.x, 0.0f, rp.y) * WATER_LOOK_RIPPLE_AMP);
  }
  const float rough = clampf(1.0f - wexp(-8.0f * unresolved), 0.0f, 1.0f);
  nw = unit(nw * (1.0f - rough) + n * rough);
  nt = unit(nt * (1.0f - rough) + n * rough);
  x.n = n; x.nw = nw; x.nt = nt; x.gloss = gloss; x.waved = waved;
  x.mirror = reflect(rd, nw);
  F3 mt = reflect(rd, nt);
  if (waved) mt = unit(f3(mt.x, fmaxf(mt.y, 0.0f), mt.z));
  x.mirror_t = mt;
  x.hit = hit; x.rd = rd; x.t = t; x.roughness = rough;
  return x;
}

// the colour of a leg's hit (shade_hit with a traced sun test)
static __device__ __noinline__ F3 shade_leg(const DevWorld& w, const vm_frame& f, const Look& L, const WorldHit& h,
                                            F3 p, F3 d, float dist, float shadow_dist) {
  const Chunk c = ld_chunk(w, h.ci);
  const uint32_t id = block_at(w, c, h.vx, h.vy, h.vz);
  return shade_surface<true>(w, f, L, h.ci, h.vx, h.vy, h.vz, id, h.normal, p, d, dist, shadow_dist, secondary_smooth(f),
                       false, -1.0f, nullptr);
}

// water_refract_leg / water_reflect_leg: resolve.wgsl:1029-1058, as
// (rgb, depth) and (rgb, 1 when hit)
static __device__ __noinline__ float4 water_refract_leg(const DevWorld& w, const vm_frame& f, const Look& L, F3 hit,
                                                        F3 n, F3 rd, float t) {
  const F3 rdir = refract(rd, n, 1.0f / VM_WATER_IOR);
  const F3 ro2 = hit + rdir * VM_SURFACE_EPS;
  const WorldHit h2 = trace_world<true, false, true>(w, f, ro2, rdir, VM_WATER_REFRACT_DIST, nullptr);
  F3 under = {0.0f, 0.0f, 0.0f};
  float depth = VM_WATER_REFRACT_DIST;
  if (h2.hit) {
    under = shade_leg(w, f, L, h2, ro2 + rdir * h2.t, rdir, t + h2.t, WATER_SHADOW_DIST);
    depth = h2.t;
  }
  return make_float4(under.x, under.y, under.z, depth);
}
static __device__ __noinline__ float4 water_reflect_leg(const DevWorld& w, const vm_frame& f, const Look& L, F3 hit,
                                                        F3 n, F3 mirror_t, float t) {
  const F3 ro3 = hit + n * VM_SURFACE_EPS;
  const WorldHit h3 = trace_world<true, false, true>(w, f, ro3, mirror_t, VM_WATER_REFLECT_DIST, nullptr);
  if (!h3.hit) return make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  F3 lit = shade_leg(w, f, L, h3, ro3 + mirror_t * h3.t, mirror_t, t + h3.t, f.shadow_dist);
  lit = mix3(lit, sky_base(f, L, mirror_t, 1.0f), 1.0f - transmittance_from(f, hit.y, h3.t, mirror_t));
  return make_float4(lit.x, lit.y, lit.z, 1.0f);
}

// ---------------------------------------------------------------------------
// the underwater resolve: resolve.wgsl:1321-1376,1449-1464

constexpr uint32_t FLAG_SNELL = 8388608u;   // the engine's FLAG_SNELL frame flag

// water_path: common.wgsl:1293-1298, the part of a camera ray under the sea
__device__ __forceinline__ float water_path(const vm_frame& f, float t, F3 rd) {
  if (rd.y <= 0.0f) return t;
  return clampf((f.sea_level - f.cam_pos[1]) / rd.y, 0.0f, t);
}
// underwater_body: resolve.wgsl:1321-1323 (WATER_BODY, resolve.wgsl:894)
static __device__ __noinline__ F3 underwater_body(const DevWorld& w, const vm_frame& f) {
  return f3(0.0100f, 0.0947f, 0.1474f) * medium_light(f, world_sample(w, f, ld3(f.cam_pos)).x);
}
// surface_from_below: resolve.wgsl:1325-1376, the sea surface seen from
// below (SNELL_MIN_DEPTH 3, WATER_DARK_DEPTH 15, SNELL_DIM_MAX 0.9:
// common.wgsl:167-171)
static __device__ __noinline__ F3 surface_from_below(const DevWorld& w, const vm_frame& f, F3 above, F3 rd,
                                                     float dist) {
  if ((f.flags & FLAG_SNELL) == 0u) return above;
  const float depth = f.sea_level - f.cam_pos[1];
  const float s = smoothstep(3.0f, 15.0f, depth);
  if (s <= 0.0f) return above;
  if (rd.y <= 0.0f) return above;
  const float t_surf = (f.sea_level - f.cam_pos[1]) / rd.y;
  if (t_surf >= dist || t_surf <= 0.0f) return above;
  const F3 surf = ld3(f.cam_pos) + rd * t_surf;
  const float mirror_detail = 1.0f - smoothstep(VM_WATER_REFRACT_NEAR, VM_WATER_REFRACT_FAR, t_surf);
  F3 nup = {0.0f, 1.0f, 0.0f};
  if ((f.flags & VM_FLAG_WAVES) != 0u && mirror_detail > 0.0f) {
    const float px_world = fmaxf(t_surf, 1e-3f) * 2.0f * f.tan_half_fov / (float)f.res[1];
    float kk = 0.0f, vhx = 0.0f, vhz = 0.0f;
    const bool aniso = (f.flags & VM_FLAG_WAVE_ANISO) != 0u;
    if (aniso) {
      const float k = 1.0f / fmaxf(fabsf(rd.y), WAVE_GRAZE_MIN);
      kk = k * k - 1.0f;
      const float r = 1.0f / sqrtf(fmaxf(rd.x * rd.x + rd.z * rd.z, 1e-12f));
      vhx = rd.x * r; vhz = rd.z * r;
    }
    const F3 wf = wave_field(f, surf.x, surf.z, px_world, vhx, vhz, kk, aniso, 1.0f);
    nup = unit(f3(-wf.x, 1.0f, -wf.y));   // wave_normal
  }
  const float cos_i = clampf(dot(rd, nup), 1e-3f, 1.0f);
  const float sin2_t = VM_WATER_IOR * VM_WATER_IOR * (1.0f - cos_i * cos_i);
  float fr = 1.0f;
  if (sin2_t < 1.0f) fr = schlick_f0(0.02f, sqrtf(1.0f - sin2_t));
  const F3 below = underwater_body(w, f);
  const F3 transmitted = mix3(above, underwater_body(w, f), s * 0.9f);
  return mix3(transmitted, below, fr * s);
}
// the camera-ray tail of an underwater frame (resolve.wgsl:1460-1464)
__device__ __forceinline__ F3 underwater_tail(const DevWorld& w, const vm_frame& f, F3 color, F3 rd, float dist) {
  color = surface_from_below(w, f, color, rd, dist);
  return water_medium(f, color, water_path(f, dist, rd), underwater_body(w, f));
}

// foam_hash / foam_mottle: resolve.wgsl:1011-1027
__device__ __forceinline__ float foam_hash(float ix, float iy) {
  const int32_t qx = __float2int_rz(ix), qy = __float2int_rz(iy);
  return (float)((hash_u32((uint32_t)qx * 374761393u + (uint32_t)qy * 668265263u) >> 8u) & 0xFFFFFFu) / 16777216.0f;
}
static __device__ __noinline__ float foam_mottle(float x, float z, float time) {
  const float k = (float)(1.0 / 0.7);     // the WGSL constant 1.0 / 0.7, folded before the f32 conversion
  const float px = x * k, pz = z * k;
  const float ix = floorf(px), iz = floorf(pz);
  const float wx = px - ix, wz = pz - iz;
  const float ux = wx * wx * (3.0f - 2.0f * wx), uz = wz * wz * (3.0f - 2.0f * wz);
  const float m0 = mixf(foam_hash(ix, iz), foam_hash(ix + 1.0f, iz), ux);
  const float m1 = mixf(foam_hash(ix, iz + 1.0f), foam_hash(ix + 1.0f, iz + 1.0f), ux);
  const float m = mixf(m0, m1, uz);
  const float ph = time * 0.55f * 4.0f + foam_hash(ix * 2.23f, iz * 2.71f) * 6.28318f;
  return m * (0.5f + 0.5f * sinf(ph));
}

// water_compose: resolve.wgsl:1169-1207 (SPEC_WATER_LOOK off)
static __device__ __noinline__ F3 water_compose(const vm_frame& f, const Look& L, const WaterCtx& x, float4 leg_r,
                                                float4 leg_m) {
  F3 refr = x.body;
  float column_depth = VM_WATER_REFRACT_DIST;
  if ((f.flags & VM_FLAG_WATER_REFRACT) != 0u && x.refract_detail > 0.0f) {
    refr = mix3(refr, water_medium(f, f3(leg_r.x, leg_r.y, leg_r.z), leg_r.w, x.body), x.refract_detail);
    column_depth = leg_r.w;
  }
  if ((L.spec_hi & HI_WATER_LOOK) != 0u && x.refract_detail > 0.0f) {
    // SPEC_WATER_LOOK (resolve.wgsl:1178-1183): murk with depth, a shallow tint
    const float depth_f = clampf(wdiv(column_depth, 7.0f), 0.0f, 1.0f);
    refr = refr * mix3(f3(1.0f, 1.0f, 1.0f), f3(0.82f, 0.90f, 0.70f), depth_f);
    const float shall = 1.0f - wsmooth(0.0f, 2.0f, column_depth);
    refr = mix3(refr, f3(0.55f, 0.74f, 0.68f) * x.ml, shall * 0.45f * x.refract_detail);
  }
  if ((L.spec_hi & HI_SHORE_FOAM) != 0u && x.refract_detail > 0.0f && column_depth < 2.5f) {
    const float shall = 1.0f - wsmooth(0.0f, 2.5f, column_depth);
    const float m = foam_mottle(x.hit.x, x.hit.z, f.time * f.wave_speed);
    const float foam = shall * wsmooth(0.45f, 0.75f, m) * x.refract_detail;
    refr = mix3(refr, f3(0.92f, 0.97f, 1.0f) * x.ml, clampf(foam, 0.0f, 1.0f) * 0.85f);
  }
  const F3 sun = ld3(f.sun_dir);
  F3 refl = sky_color(f, L, x.hit, x.mirror, x.t, 1.0f) +
            f3(1.0000f, 0.8469f, 0.5647f) *
                (wpow(fmaxf(dot(x.mirror, sun), 0.0f), 320.0f * x.gloss) * 2.5f * x.gloss * f.daylight);
  if ((f.flags & VM_FLAG_WATER_REFLECT) != 0u && x.reflect_detail > 0.0f && leg_m.w > 0.0f)
    refl = mix3(refl, f3(leg_m.x, leg_m.y, leg_m.z), x.reflect_detail);
  // SURFACE_DEBUG 5-7 (resolve.wgsl:1200-1202): water normal, reflected, refracted
  const uint32_t debug_view = surface_debug(L);
  if (debug_view == 5u) return add_s(x.n * 0.5f, 0.5f);
  if (debug_view == 6u) return refl;
  if (debug_view == 7u) return refr;
  refl = mix3(refl, sky_base(f, L, x.n, 1.0f), x.roughness * 0.65f);
  return mix3(refr, refl, schlick_f0(0.02f, fmaxf(-dot(x.rd, x.nw), 1e-3f)));
}

// shade_water: resolve.wgsl:1209-1221
static __device__ __noinline__ F3 shade_water(const DevWorld& w, const vm_frame& f, const Look& L, uint32_t ci,
                                              uint32_t vx, uint32_t vy, uint32_t vz, uint32_t nid, F3 hit, F3 rd,
                                              float t) {
  const WaterCtx x = water_ctx(w, f, L, ci, vx, vy, vz, nid, hit, rd, t);
  float4 leg_r = make_float4(0.0f, 0.0f, 0.0f, VM_WATER_REFRACT_DIST);
  if ((f.flags & VM_FLAG_WATER_REFRACT) != 0u && x.refract_detail > 0.0f)
    leg_r = water_refract_leg(w, f, L, hit, x.n, rd, t);
  float4 leg_m = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  if ((f.flags & VM_FLAG_WATER_REFLECT) != 0u && x.reflect_detail > 0.0f)
    leg_m = water_reflect_leg(w, f, L, hit, x.n, x.mirror_t, t);
  return water_compose(f, L, x, leg_r, leg_m);
}

// shade_glass: resolve.wgsl:1261-1319
static __device__ __noinline__ F3 shade_glass(const DevWorld& w, const vm_frame& f, const Look& L, uint32_t ci,
                                              uint32_t vx, uint32_t vy, uint32_t vz, uint32_t nid, F3 hit, F3 rd,
                                              float t) {
  const Chunk c = ld_chunk(w, ci);
  const float vs = c.vs;
  F3 n = normal_of(nid);
  if (dot(n, rd) > 0.0f) n = neg(n);
  const F3 box_min = ld3(c.origin) + f3((float)vx, (float)vy, (float)vz) * vs;
  const F3 lq = (hit - box_min) / vs;
  const F3 local = {clampf(lq.x, 0.0f, 1.0f), clampf(lq.y, 0.0f, 1.0f), clampf(lq.z, 0.0f, 1.0f)};
  const float footprint = fmaxf(t, 1e-3f) * 2.0f * f.tan_half_fov / (float)f.res[1] * 16.0f / vs;
  const float lod = clampf(log2f(fmaxf(footprint, 1e-4f)) + f.mip_bias, 0.0f, 3.0f);
  const uint32_t fi = VM_GLASS * 8u + nid;
  const uint32_t layer = (fi < L.n_faces ? __ldg(L.faces + fi) : 0u) & 0xFFFFu;
  float u, v;
  face_uv(nid, local, &u, &v);
  const float4 tx = atlas_sample(L, u, v, layer, lod);
  const F3 tint = {tx.x, tx.y, tx.z};
  const F3 ro2 = hit + rd * VM_SURFACE_EPS;
  const float reach = fmaxf(VM_GLASS_TRANSMIT_DIST, f.far_);
  const WorldHit h2 = trace_world<false, false, true>(w, f, ro2, rd, reach, nullptr);
  F3 through = sky_color(f, L, ro2, rd, t, 1.0f);
  if (h2.hit) {
    const F3 p2 = ro2 + rd * h2.t;
    const Chunk c2 = ld_chunk(w, h2.ci);
    if (block_at(w, c2, h2.vx, h2.vy, h2.vz) == VM_WATER)
      through = shade_water(w, f, L, h2.ci, h2.vx, h2.vy, h2.vz, h2.normal, p2, rd, t + h2.t);
    else
      through = shade_leg(w, f, L, h2, p2, rd, t + h2.t, GLASS_SHADOW_DIST);
    through = mix3(through, sky_base(f, L, rd, 1.0f), 1.0f - transmittance_from(f, hit.y, h2.t, rd));
  }
  const F3 mirror = reflect(rd, n);
  F3 refl = sky_color(f, L, hit, mirror, t, 1.0f);
  if ((L.spec_hi & HI_GLASS_REFLECT) != 0u) {
    const F3 origin = hit + n * VM_SURFACE_EPS;
    const WorldHit r = trace_world<false, false, true>(w, f, origin, mirror, reach, nullptr);
    if (r.hit) {
      const F3 point = origin + mirror * r.t;
      const Chunk c3 = ld_chunk(w, r.ci);
      if (block_at(w, c3, r.vx, r.vy, r.vz) == VM_WATER)
        refl = shade_water(w, f, L, r.ci, r.vx, r.vy, r.vz, r.normal, point, mirror, t + r.t);
      else
        refl = shade_leg(w, f, L, r, point, mirror, t + r.t, GLASS_SHADOW_DIST);
      refl = mix3(refl, sky_base(f, L, mirror, 1.0f), 1.0f - transmittance_from(f, hit.y, r.t, mirror));
    }
  }
  return mix3(through * tint, refl, schlick_f0(0.0426f, fmaxf(-dot(rd, n), 1e-3f)));
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

// The engine's rgba16float water_sec targets: binary16, round to nearest even.
__device__ __forceinline__ ushort4 to_half4(float4 v) {
  return make_ushort4(__half_as_ushort(__float2half_rn(v.x)), __half_as_ushort(__float2half_rn(v.y)),
                      __half_as_ushort(__float2half_rn(v.z)), __half_as_ushort(__float2half_rn(v.w)));
}
__device__ __forceinline__ float4 from_half4(ushort4 h) {
  return make_float4(__half2float(__ushort_as_half(h.x)), __half2float(__ushort_as_half(h.y)),
                     __half2float(__ushort_as_half(h.z)), __half2float(__ushort_as_half(h.w)));
}

// the resolve's lanes, as k_resolve's PART
constexpr uint8_t LANE_OPAQUE = 0, LANE_SKY = 1, LANE_WATER = 2, LANE_GLASS = 3, LANE_WATER_OWN = 4;

// The colour pass of water_sec (resolve.wgsl:1468-1535): per (2^shift)^2
// block the water pixel of least hit distance (first in x-major order on
// ties), its water_ctx and both legs shaded, stored as the engine's
// rgba16float targets (refract: colour and depth; reflect: colour, 1 if hit).
__global__ void __launch_bounds__(128) k_water_legs(const __grid_constant__ vm_frame f, const __grid_constant__ DevWorld w,
                                                    const __grid_constant__ Look L,
                                                    const unsigned long long* __restrict__ vis,
                                                    const uint8_t* __restrict__ lane, uint32_t shift,
                                                    ushort4* __restrict__ refr, ushort4* __restrict__ refl) {
  const uint32_t span = 1u << shift;
  const uint32_t hw = (f.res[0] + span - 1u) >> shift, hh = (f.res[1] + span - 1u) >> shift;
  const uint32_t hx = blockIdx.x * 16u + threadIdx.x, hy = blockIdx.y * 8u + threadIdx.y;
  if (hx >= hw || hy >= hh) return;
  float4 leg_r = make_float4(0.0f, 0.0f, 0.0f, VM_WATER_REFRACT_DIST), leg_m = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  float best_t = 3.4e38f;
  bool has = false;
  KeyParts best = {};
  uint32_t bpx = 0, bpy = 0;
  for (uint32_t i = 0; i < span; ++i)
    for (uint32_t j = 0; j < span; ++j) {
      const uint32_t pxs = span * hx + i, pys = span * hy + j;
      if (pxs >= f.res[0] || pys >= f.res[1]) continue;
      const uint64_t pix = (uint64_t)pys * f.res[0] + pxs;
      if (lane[pix] != LANE_WATER && lane[pix] != LANE_WATER_OWN) continue;
      const KeyParts k = split_key(vis[pix]);
      const Chunk c = ld_chunk(w, k.ci);
      const F3 rd0 = ray_dir(f, (float)pxs + 0.5f, (float)pys + 0.5f);
      const float ts = hit_t(f, c, k.vx, k.vy, k.vz, k.mx, k.my, k.mz, k.nid, rd0);
      if (ts < best_t) { best_t = ts; best = k; bpx = pxs; bpy = pys; has = true; }
    }
  if (has) {
    const F3 rd = ray_dir(f, (float)bpx + 0.5f, (float)bpy + 0.5f);
    const F3 hit = ld3(f.cam_pos) + rd * best_t;
    const WaterCtx x = water_ctx(w, f, L, best.ci, best.vx, best.vy, best.vz, best.nid, hit, rd, best_t);
    if ((f.flags & VM_FLAG_WATER_REFRACT) != 0u && x.refract_detail > 0.0f)
      leg_r = water_refract_leg(w, f, L, hit, x.n, rd, best_t);
    if ((f.flags & VM_FLAG_WATER_REFLECT) != 0u && x.reflect_detail > 0.0f)
      leg_m = water_reflect_leg(w, f, L, hit, x.n, x.mirror_t, best_t);
  }
  const uint64_t h = (uint64_t)hy * hw + hx;
  refr[h] = to_half4(leg_r);
  refl[h] = to_half4(leg_m);
}

// water_share_safe: resolve.wgsl:1223-1245: the block's pixels all hit flat
// water on the same +Y plane, close in distance
__device__ __noinline__ bool water_share_safe(const vm_frame& f, const DevWorld& w, const unsigned long long* vis,
                                              uint32_t shift, uint32_t px, uint32_t py, uint32_t nid, F3 hit, float t) {
  if (nid != VM_NORMAL_PY) return false;
  const uint32_t span = 1u << shift;
  const uint32_t bx = (px >> shift) * span, by = (py >> shift) * span;
  for (uint32_t y = 0; y < span; ++y)
    for (uint32_t x = 0; x < span; ++x) {
      const uint32_t qx = bx + x, qy = by + y;
      if (qx >= f.res[0] || qy >= f.res[1]) continue;
      const unsigned long long key = vis[(uint64_t)qy * f.res[0] + qx];
      if (key == 0ull) return false;
      const KeyParts k = split_key(key);
      if (k.nid != nid) return false;
      const Chunk c = ld_chunk(w, k.ci);
      if (block_at(w, c, k.vx, k.vy, k.vz) != VM_WATER) return false;
      const F3 rd = ray_dir(f, (float)qx + 0.5f, (float)qy + 0.5f);
      const float td = hit_t(f, c, k.vx, k.vy, k.vz, k.mx, k.my, k.mz, k.nid, rd);
      const F3 hd = ld3(f.cam_pos) + rd * td;
      if (fabsf(hd.y - hit.y) > 0.01f || fabsf(td - t) > fmaxf(0.1f, fminf(1.0f, t * 0.02f))) return false;
    }
  return true;
}

// the water_sec targets; decided: k_resolve_lanes sent the pixels of unsafe
// blocks to LANE_WATER_OWN, so every LANE_WATER pixel composes its block's legs
struct WaterSec { const ushort4* refr; const ushort4* refl; uint32_t shift, hw; bool decided; };

// A warp's pixels of one kind appended to a compact list (one atomic per
// warp; the lanes of a 32-wide row stay together in the list).
__device__ __forceinline__ void append_pixel(bool mine, uint32_t* list, uint32_t* count, uint32_t pix) {
  const uint32_t bal = __ballot_sync(FULLMASK, mine);
  if (bal == 0u) return;
  uint32_t base = 0u;
  if ((threadIdx.x & 31u) == 0u) base = atomicAdd(count, (uint32_t)__popc(bal));
  base = __shfl_sync(FULLMASK, base, 0);
  if (mine) list[base + (uint32_t)__popc(bal & lanemask_lt())] = pix;
}

// The lane of every pixel: the engine's resolve picks a pixel's shading by
// its hit's block (resolve.wgsl:1378-1466).  Decided once per pixel, a byte
// each, so that every lane's kernel passes over the other lanes' pixels with
// one byte load instead of a chunk record load and a tree walk.  With the
// half-resolution legs under SPEC_WATER_REPAIR (DECIDE), water_share_safe
// (resolve.wgsl:1223-1245) is decided here as well: a 32x4 tile holds whole
// 2x2 blocks, so each thread decodes its own pixel (hit distance, hit
// height, normal, water or not) into shared memory and the test reads its
// block there; water pixels of unsafe blocks take LANE_WATER_OWN.  The glass
// pixels and those, few and clustered, each tracing long legs, also go to
// compact lists, so that their kernels run full warps over them instead of
// the frame's grid with a few live lanes per warp.
template <bool DECIDE>
__global__ void __launch_bounds__(128) k_resolve_lanes(const __grid_constant__ vm_frame f,
                                                       const __grid_constant__ DevWorld w,
                                                       const unsigned long long* __restrict__ vis,
                                                       uint8_t* __restrict__ lane, uint32_t* __restrict__ glass_list,
                                                       uint32_t* __restrict__ own_list, uint32_t* __restrict__ counts) {
  __shared__ float s_hy[4][32], s_t[4][32];
  __shared__ uint8_t s_code[4][32];   // bit 0 in the frame, 1 a key, 2 water, bits 3-5 the normal
  const uint32_t tx = threadIdx.x, ty = threadIdx.y;
  const uint32_t px = blockIdx.x * 32u + tx, py = blockIdx.y * 4u + ty;
  const bool inside = px < f.res[0] && py < f.res[1];
  const uint32_t pix = inside ? py * f.res[0] + px : 0u;
  uint32_t ln = LANE_SKY, code = 0u, nid = 0u;
  float hy = 0.0f, t = 0.0f;
  if (inside) {
    code = 1u;
    const unsigned long long key = vis[pix];
    if (key != 0ull) {
      const KeyParts k = split_key(key);
      const Chunk c = ld_chunk(w, k.ci);
      const uint32_t id = block_at(w, c, k.vx, k.vy, k.vz);
      ln = id == VM_WATER ? LANE_WATER : ((w.spec & VM_SPEC_GLASS) != 0u && id == VM_GLASS ? LANE_GLASS : LANE_OPAQUE);
      code |= 2u;
      if (DECIDE && ln == LANE_WATER) {
        const F3 rd = ray_dir(f, (float)px + 0.5f, (float)py + 0.5f);
        t = hit_t(f, c, k.vx, k.vy, k.vz, k.mx, k.my, k.mz, k.nid, rd);
        hy = (ld3(f.cam_pos) + rd * t).y;
        nid = k.nid;
        code |= 4u | (nid << 3);
      }
    }
  }
  if (DECIDE) {
    s_hy[ty][tx] = hy;
    s_t[ty][tx] = t;
    s_code[ty][tx] = (uint8_t)code;
    __syncthreads();
    if (ln == LANE_WATER) {
      bool safe = nid == VM_NORMAL_PY;
      const uint32_t bx = tx & ~1u, by = ty & ~1u;
      for (uint32_t y = 0; y < 2u && safe; ++y)
        for (uint32_t x = 0; x < 2u && safe; ++x) {
          const uint32_t q = s_code[by + y][bx + x];
          if ((q & 1u) == 0u) continue;
          if ((q & 2u) == 0u || ((q >> 3) & 7u) != nid || (q & 4u) == 0u) { safe = false; break; }
          if (fabsf(s_hy[by + y][bx + x] - hy) > 0.01f ||
              fabsf(s_t[by + y][bx + x] - t) > fmaxf(0.1f, fminf(1.0f, t * 0.02f)))
            safe = false;
        }
      if (!safe) ln = LANE_WATER_OWN;
    }
  }
  append_pixel(ln == LANE_GLASS, glass_list, counts, pix);
  append_pixel(ln == LANE_WATER_OWN, own_list, counts + 1, pix);
  if (inside) lane[pix] = (uint8_t)ln;
}

// The pixels of a compact list: glass (WHICH 0, shade_glass,
// resolve.wgsl:1261-1319) or water with its own legs (WHICH 1, shade_water),
// before the fog blend; a thread per pixel over a grid of resident blocks.
template <int WHICH>
__global__ void __launch_bounds__(128, 8) k_resolve_list(const __grid_constant__ vm_frame f,
                                                         const __grid_constant__ DevWorld w,
                                                         const __grid_constant__ Look L,
                                                         const unsigned long long* __restrict__ vis,
                                                         const uint32_t* __restrict__ list,
                                                         const uint32_t* __restrict__ count,
                                                         float4* __restrict__ out) {
  const uint32_t n = *count;
  const F3 cam = ld3(f.cam_pos);
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t pix = list[i];
    const uint32_t px = pix % f.res[0], py = pix / f.res[0];
    const KeyParts k = split_key(vis[pix]);
    const F3 rd = ray_dir(f, (float)px + 0.5f, (float)py + 0.5f);
    const Chunk c = ld_chunk(w, k.ci);
    const float t = hit_t(f, c, k.vx, k.vy, k.vz, k.mx, k.my, k.mz, k.nid, rd);
    const F3 hit = cam + rd * t;
    const F3 color = WHICH == 0 ? shade_glass(w, f, L, k.ci, k.vx, k.vy, k.vz, k.nid, hit, rd, t)
                                : shade_water(w, f, L, k.ci, k.vx, k.vy, k.vz, k.nid, hit, rd, t);
    out[pix] = make_float4(color.x, color.y, color.z, 1.0f);   // the fog blend follows (k_resolve_blend)
  }
}

// The light terms of every opaque-surface pixel, ahead of k_resolve<0>: the
// 3x3 light and AO gather (tree walks, light bricks, the neighbour chunks)
// in a kernel of its own, so that the shading kernel's code stays small.
// Writes (amb, sky_sm) into the pixel's colour, which k_resolve<0> reads and
// overwrites, and the AO into light_ao.
__global__ void __launch_bounds__(128, 12) k_resolve_light(const __grid_constant__ vm_frame f,
                                                          const __grid_constant__ DevWorld w,
                                                          const __grid_constant__ Look L,
                                                          const unsigned long long* __restrict__ vis,
                                                          const uint8_t* __restrict__ lane,
                                                          float4* __restrict__ out, float* __restrict__ light_ao) {
  const uint32_t px = blockIdx.x * 32u + threadIdx.x, py = blockIdx.y * 4u + threadIdx.y;
  if (px >= f.res[0] || py >= f.res[1]) return;
  const uint64_t pix = (uint64_t)py * f.res[0] + px;
  if (lane[pix] != LANE_OPAQUE) return;
  const unsigned long long key = vis[pix];
  const uint32_t nid = (uint32_t)(key >> 37) & 7u;
  const uint32_t ci = (uint32_t)(key >> 24) & 0x1FFFu;
  const uint32_t low = (uint32_t)(key & 0xFFFFFFull);
  const uint32_t vx = (low >> 16) & 63u, vy = (low >> 8) & 63u, vz = low & 63u;
  const uint32_t mx = (low >> 22) & 3u, my = (low >> 14) & 3u, mz = (low >> 6) & 3u;
  const Chunk c = ld_chunk(w, ci);
  const F3 rd = ray_dir(f, (float)px + 0.5f, (float)py + 0.5f);
  const float t = hit_t(f, c, vx, vy, vz, mx, my, mz, nid, rd);
  const F3 hit = ld3(f.cam_pos) + rd * t;
  F3 n = normal_of(nid);
  if (nid >= VM_NORMAL_CROSS_A && dot(n, rd) > 0.0f) n = neg(n);
  const LightTerms lt = surface_light_terms(w, f, L, ci, vx, vy, vz, nid, n, hit, true);
  out[pix] = make_float4(lt.amb.x, lt.amb.y, lt.amb.z, lt.sky_sm);
  light_ao[pix] = lt.ao;
}

// PART 0: the opaque surfaces, 1: the sky, 2: water (the glass pixels and the
// water pixels with their own legs run from compact lists, k_resolve_list).
// A launch per lane over the frame instead of one kernel with every path:
// each kernel carries a part of the code (one kernel stalled on instruction
// fetch) and its warps run one path.
// 12 blocks of 4 warps per SM (40 registers, a few bytes spilled): more
// warps hide the L2 gathers of the issue-bound lanes (8 blocks: 2% slower).
// EXTRA: the frame is underwater, uses the probe-tap / probe-ambient variants
// or a surface debug view (their code is compiled out of the other launches).
template <int PART, bool EXTRA>
__global__ void __launch_bounds__(128, 12) k_resolve(const __grid_constant__ vm_frame f, const __grid_constant__ DevWorld w,
                                                    const __grid_constant__ Look L,
                                                    const unsigned long long* __restrict__ vis,
                                                    const float* __restrict__ mask, const float* __restrict__ dist,
                                                    const uint8_t* __restrict__ lane, bool soft, WaterSec ws,
                                                    const float* __restrict__ light_ao, float4* __restrict__ out) {
  const uint32_t px = blockIdx.x * 32u + threadIdx.x, py = blockIdx.y * 4u + threadIdx.y;
  if (px >= f.res[0] || py >= f.res[1]) return;
  const uint64_t pix = (uint64_t)py * f.res[0] + px;
  if (lane[pix] != (uint8_t)PART) return;
  const unsigned long long key = vis[pix];
  const F3 cam = ld3(f.cam_pos);
  const F3 rd = ray_dir(f, (float)px + 0.5f, (float)py + 0.5f);
  F3 color;
  const bool underwater = EXTRA && (f.flags & VM_FLAG_UNDERWATER) != 0u;
  if (PART == 1) {
    const float shaft = underwater ? 1.0f : sun_shaft(f, L, cam, rd, f.far_, 1.0f, px, py);
    color = sky_color(f, L, cam, rd, 0.0f, shaft);
    if (underwater && surface_debug(L) == 0u) color = underwater_tail(w, f, color, rd, f.far_);
  } else {
    const uint32_t nid = (uint32_t)(key >> 37) & 7u;
    const uint32_t ci = (uint32_t)(key >> 24) & 0x1FFFu;
    const uint32_t low = (uint32_t)(key & 0xFFFFFFull);
    const uint32_t vx = (low >> 16) & 63u, vy = (low >> 8) & 63u, vz = low & 63u;
    const uint32_t mx = (low >> 22) & 3u, my = (low >> 14) & 3u, mz = (low >> 6) & 3u;
    const Chunk c = ld_chunk(w, ci);
    const float t = hit_t(f, c, vx, vy, vz, mx, my, mz, nid, rd);
    const F3 hit = cam + rd * t;
    if (PART == 0) {
      const uint32_t id = block_at(w, c, vx, vy, vz);
      LightTerms lt;
      if (light_ao != nullptr) {
        const float4 a = out[pix];
        lt = {f3(a.x, a.y, a.z), a.w, light_ao[pix]};
      }
      color = shade_surface<EXTRA>(w, f, L, ci, vx, vy, vz, id, nid, hit, rd, t, f.shadow_dist, true, true,
                            sun_visibility(mask, dist, soft, pix), light_ao != nullptr ? &lt : nullptr);
    } else if (PART == 2) {
      if (ws.refr != nullptr && (ws.decided || (w.spec & VM_SPEC_WATER_REPAIR) == 0u ||
                                 water_share_safe(f, w, vis, ws.shift, px, py, nid, hit, t))) {
        // shade_water_sec (resolve.wgsl:1247-1259): the block's legs
        const WaterCtx x = water_ctx(w, f, L, ci, vx, vy, vz, nid, hit, rd, t);
        const uint64_t h = (uint64_t)(py >> ws.shift) * ws.hw + (px >> ws.shift);
        color = water_compose(f, L, x, from_half4(ws.refr[h]), from_half4(ws.refl[h]));
      } else {
        color = shade_water(w, f, L, ci, vx, vy, vz, nid, hit, rd, t);
      }
    }
    if (PART == 0 && (!EXTRA || surface_debug(L) == 0u)) {   // water: the fog blend follows (k_resolve_blend)
      const float wet = underwater ? water_path(f, t, rd) : 0.0f;
      const float alpha = 1.0f - transmittance_from(f, cam.y + wet * rd.y, t - wet, rd);
      const float shaft = underwater ? 1.0f : sun_shaft(f, L, cam, rd, t, alpha, px, py);
      color = mix3(color, sky_base(f, L, rd, shaft), alpha);
      if (underwater) color = underwater_tail(w, f, color, rd, t);
    }
  }
  out[pix] = make_float4(color.x, color.y, color.z, 1.0f);
}

// The fog terms of the water and glass pixels (the blend of every surface
// lane, resolve.wgsl:1440-1466: fog opacity, sun shafts, sky behind), on the
// issue-bound chain beside the water and glass lanes, so that their long
// per-pixel chains end at the surface colour; k_resolve_blend applies them.
__global__ void __launch_bounds__(128, 12) k_resolve_fog(const __grid_constant__ vm_frame f,
                                                        const __grid_constant__ DevWorld w,
                                                        const __grid_constant__ Look L,
                                                        const unsigned long long* __restrict__ vis,
                                                        const uint8_t* __restrict__ lane, float4* __restrict__ fog) {
  const uint32_t px = blockIdx.x * 32u + threadIdx.x, py = blockIdx.y * 4u + threadIdx.y;
  if (px >= f.res[0] || py >= f.res[1]) return;
  const uint64_t pix = (uint64_t)py * f.res[0] + px;
  const uint32_t ln = lane[pix];
  if (ln != LANE_WATER && ln != LANE_GLASS && ln != LANE_WATER_OWN) return;
  const KeyParts k = split_key(vis[pix]);
  const F3 cam = ld3(f.cam_pos);
  const F3 rd = ray_dir(f, (float)px + 0.5f, (float)py + 0.5f);
  const float t = hit_t(f, ld_chunk(w, k.ci), k.vx, k.vy, k.vz, k.mx, k.my, k.mz, k.nid, rd);
  const bool underwater = (f.flags & VM_FLAG_UNDERWATER) != 0u;
  const float wet = underwater ? water_path(f, t, rd) : 0.0f;
  const float alpha = 1.0f - transmittance_from(f, cam.y + wet * rd.y, t - wet, rd);
  const float shaft = underwater ? 1.0f : sun_shaft(f, L, cam, rd, t, alpha, px, py);
  const F3 sky = sky_base(f, L, rd, shaft);
  fog[pix] = make_float4(sky.x, sky.y, sky.z, alpha);
}

// The fog blend of the water and glass pixels, once their lanes are done
// (and, in an underwater frame, the camera ray's own tail).
__global__ void __launch_bounds__(256) k_resolve_blend(const __grid_constant__ vm_frame f,
                                                       const __grid_constant__ DevWorld w,
                                                       const unsigned long long* __restrict__ vis,
                                                       const uint8_t* __restrict__ lane,
                                                       const float4* __restrict__ fog, float4* __restrict__ out) {
  const uint32_t pix = blockIdx.x * 256u + threadIdx.x;
  if (pix >= f.res[0] * f.res[1]) return;
  const uint32_t ln = lane[pix];
  if (ln != LANE_WATER && ln != LANE_GLASS && ln != LANE_WATER_OWN) return;
  const float4 c = out[pix], g = fog[pix];
  F3 color = mix3(f3(c.x, c.y, c.z), f3(g.x, g.y, g.z), g.w);
  if ((f.flags & VM_FLAG_UNDERWATER) != 0u) {
    const uint32_t px = pix % f.res[0], py = pix / f.res[0];
    const KeyParts k = split_key(vis[pix]);
    const F3 rd = ray_dir(f, (float)px + 0.5f, (float)py + 0.5f);
    const float t = hit_t(f, ld_chunk(w, k.ci), k.vx, k.vy, k.vz, k.mx, k.my, k.mz, k.nid, rd);
    color = underwater_tail(w, f, color, rd, t);
  }
  out[pix] = make_float4(color.x, color.y, color.z, 1.0f);
}

// heat (resolve.wgsl:36-44): the iteration heat map of a FLAG_HEATMAP frame
// (resolve.wgsl:1389-1394), every pixel's summed march iterations / 300.
__global__ void __launch_bounds__(256) k_resolve_heat(const __grid_constant__ vm_frame f,
                                                      const uint32_t* __restrict__ dbg, float4* __restrict__ out) {
  const uint32_t pix = blockIdx.x * 256u + threadIdx.x;
  if (pix >= f.res[0] * f.res[1]) return;
  const float t = clampf((float)dbg[pix] / 300.0f, 0.0f, 1.0f);
  const F3 c = {smoothstep(0.35f, 0.85f, t), smoothstep(0.0f, 0.45f, t) - smoothstep(0.65f, 1.0f, t),
                1.0f - smoothstep(0.0f, 0.45f, t)};
  out[pix] = make_float4(wpow(c.x, 2.2f), wpow(c.y, 2.2f), wpow(c.z, 2.2f), 1.0f);
}

cudaError_t launch_resolve_heat(const vm_frame& f, const uint32_t* dbg, float4* out, cudaStream_t s) {
  const uint32_t npix = f.res[0] * f.res[1];
  k_resolve_heat<<<(npix + 255u) / 256u, 256, 0, s>>>(f, dbg, out);
  return cudaGetLastError();
}

cudaError_t launch_resolve(const vm_frame& f, const DevWorld& w, const Look& L, const unsigned long long* vis,
                           const float* mask, const float* dist, bool soft_rays, uint32_t water_sec_shift,
                           uint16_t* leg_refr, uint16_t* leg_refl, uint8_t* lane, uint32_t* lists, float* light_ao,
                           float4* fog, float4* out, int sms, cudaStream_t s, const cudaStream_t lane_stream[3],
                           const cudaEvent_t lane_event[4]) {
  // The lanes write disjoint pixels.  The water lane (its legs, then the
  // pixels) and the glass lane cover a few clustered pixels with long serial
  // traces, which leave most SMs idle: they run on streams of their own,
  // forked from s and joined back into it, beside the sky / opaque lanes.
  const uint32_t npix = f.res[0] * f.res[1];
  uint32_t* glass_list = lists;
  uint32_t* own_list = lists + npix;
  uint32_t* counts = lists + 2u * (uint64_t)npix;
  const dim3 block(32, 4), grid((f.res[0] + 31u) / 32u, (f.res[1] + 3u) / 4u);
  const bool split_water = leg_refr != nullptr && water_sec_shift == 1u;
  const bool decide = split_water && (w.spec & VM_SPEC_WATER_REPAIR) != 0u;
  cudaError_t e = cudaMemsetAsync(counts, 0, 2 * sizeof(uint32_t), s);
  if (e != cudaSuccess) return e;
  if (decide) k_resolve_lanes<true><<<grid, block, 0, s>>>(f, w, vis, lane, glass_list, own_list, counts);
  else k_resolve_lanes<false><<<grid, block, 0, s>>>(f, w, vis, lane, glass_list, own_list, counts);
  if ((e = cudaEventRecord(lane_event[0], s)) != cudaSuccess) return e;
  for (int i = 0; i < 3 && e == cudaSuccess; ++i) e = cudaStreamWaitEvent(lane_stream[i], lane_event[0], 0);
  if (e != cudaSuccess) return e;
  const unsigned resident = (unsigned)max(sms, 1) * 8u;
  if (decide) k_resolve_list<1><<<resident, 128, 0, lane_stream[2]>>>(f, w, L, vis, own_list, counts + 1, out);
  if ((w.spec & VM_SPEC_GLASS) != 0u)
    k_resolve_list<0><<<resident, 128, 0, lane_stream[1]>>>(f, w, L, vis, glass_list, counts, out);
  WaterSec ws{nullptr, nullptr, water_sec_shift, 0u, decide};
  const cudaStream_t sw = lane_stream[0];
  if (leg_refr != nullptr) {
    const uint32_t span = 1u << water_sec_shift;
    const uint32_t hw = (f.res[0] + span - 1u) >> water_sec_shift, hh = (f.res[1] + span - 1u) >> water_sec_shift;
    k_water_legs<<<dim3((hw + 15) / 16, (hh + 7) / 8), dim3(16, 8), 0, sw>>>(
        f, w, L, vis, lane, water_sec_shift, (ushort4*)leg_refr, (ushort4*)leg_refl);
    ws = {(const ushort4*)leg_refr, (const ushort4*)leg_refl, water_sec_shift, hw, decide};
  }
  const bool extra = (f.flags & (VM_FLAG_UNDERWATER | VM_FLAG_PROBE_TAP | VM_FLAG_PROBE_AMBIENT)) != 0u ||
                     surface_debug(L) != 0u;
  if (extra) k_resolve<2, true><<<grid, block, 0, sw>>>(f, w, L, vis, mask, dist, lane, soft_rays, ws, nullptr, out);
  else k_resolve<2, false><<<grid, block, 0, sw>>>(f, w, L, vis, mask, dist, lane, soft_rays, ws, nullptr, out);
  if (light_ao != nullptr) k_resolve_light<<<grid, block, 0, s>>>(f, w, L, vis, lane, out, light_ao);
  if (extra) {
    k_resolve<0, true><<<grid, block, 0, s>>>(f, w, L, vis, mask, dist, lane, soft_rays, ws, light_ao, out);
    k_resolve<1, true><<<grid, block, 0, s>>>(f, w, L, vis, mask, dist, lane, soft_rays, ws, nullptr, out);
  } else {
    k_resolve<0, false><<<grid, block, 0, s>>>(f, w, L, vis, mask, dist, lane, soft_rays, ws, light_ao, out);
    k_resolve<1, false><<<grid, block, 0, s>>>(f, w, L, vis, mask, dist, lane, soft_rays, ws, nullptr, out);
  }
  const bool blend = surface_debug(L) == 0u;   // the debug views skip the fog and the underwater tail
  if (blend) k_resolve_fog<<<grid, block, 0, s>>>(f, w, L, vis, lane, fog);
  e = cudaGetLastError();
  for (int i = 0; i < 3 && e == cudaSuccess; ++i) {
    e = cudaEventRecord(lane_event[1 + i], lane_stream[i]);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(s, lane_event[1 + i], 0);
  }
  if (e != cudaSuccess) return e;
  if (blend) k_resolve_blend<<<(npix + 255u) / 256u, 256, 0, s>>>(f, w, vis, lane, fog, out);
  return cudaGetLastError();
}

}  // namespace vmk
