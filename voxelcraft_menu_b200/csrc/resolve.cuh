// The engine's resolve of opaque surfaces and sky: lane 0 of the resolve pass
// (resolve.wgsl:1378-1466 with RESOLVE_LANE 0), whose surface colour is
// shade_hit_legacy_cached (resolve.wgsl:1537-1788), the engine's default
// (SPEC_COMPACT_SHADE_HIT off), and whose sky is sky_color
// (common.wgsl:1484-1530).  Water and glass pixels belong to the engine's
// other resolve lanes.
//
// Material inputs are plain device buffers instead of textures: the block
// atlas (the engine's Rgba8UnormSrgb array, 16x16, 4 mips) decoded to linear
// float on upload, the block face table, the RGBA16F probe field and the
// shaft pass's envelope.  Texture filtering is restated from the sampling
// equations of the texture units (mag / min / mipmap filter, clamp-to-edge
// and repeat addressing) in float arithmetic, so the kernel and the oracle
// agree up to the last bits of the transcendental functions.
//
// Compiled with the march's float contract (--fmad=false): block lookups
// and voxel indices must match the march exactly.  The colour arithmetic
// (fog, sky, clouds, shafts, light curves, shading) runs at the accuracy
// WGSL specifies for the engine's own shaders instead (wdiv / wexp / wlog /
// wpow below), on the SM's approximate reciprocal, exp2 and log2 units.
// The larger helpers (sky,
// cloud octaves, biome noise, light samples, texture filters, shafts) stay
// out of line: inlined at every call site the kernel's code outgrew the
// instruction cache and its warps stalled on instruction fetch.
#pragma once
#include <cuda_fp16.h>
#include "march_device.cuh"
#include "water.cuh"

namespace vmd {

// The resolve's material inputs on the device.
struct Look {
  const float4* atlas; uint32_t atlas_layers;   // linear RGBA, mips 16, 8, 4, 2 one after the other, [layer][y][x]
  const uint32_t* faces; uint32_t n_faces;      // block_faces: id * 8 + normal_id -> layer | perm << 16
  const ushort4* probes;                        // RGBA16F probe field (x, slab * 128 + y, z), or null: all 1.0
  const float* shaft;                           // the shaft envelope, VM_SHAFT_DIM^2 floats, or null: terrain open
  const float2* grad;                           // (cos, sin) of the 32 simplex gradient angles
  uint32_t spec_hi;                             // the engine's FLAG_HI_* word (the resolve's overrides)
};

// WGSL's accuracy for the engine's shader arithmetic: x / y within 2.5 ULP
// (__fdividef: an approximate reciprocal and a multiply, 2 ULP for |y| below
// 2^126), exp within 3 + 2|x| ULP (__expf), log within 2^-21 absolute on
// [0.5, 2] and 3 ULP elsewhere (__logf), and pow inheriting its accuracy
// from exp2(y * log2(x)) (__powf computes exactly that).  IEEE division and
// CUDA's expf / logf / powf are several times the instructions and buy no
// accuracy the engine's own colours have.
__device__ __forceinline__ float wdiv(float a, float b) { return __fdividef(a, b); }
__device__ __forceinline__ F3 wdiv3(F3 a, float b) { return {wdiv(a.x, b), wdiv(a.y, b), wdiv(a.z, b)}; }
__device__ __forceinline__ float wexp(float x) { return __expf(x); }
__device__ __forceinline__ float wlog(float x) { return __logf(x); }
__device__ __forceinline__ float wpow(float x, float y) { return __powf(x, y); }
// smoothstep with WGSL's division (the march's smoothstep stays IEEE: its
// results decide which legs are traced)
__device__ __forceinline__ float wsmooth(float e0, float e1, float x) {
  const float t = fminf(fmaxf(wdiv(x - e0, e1 - e0), 0.0f), 1.0f);
  return t * t * (3.0f - 2.0f * t);
}

constexpr uint32_t ATLAS_SIZE = VM_ATLAS_SIZE, ATLAS_MIPS = VM_ATLAS_MIPS;
constexpr uint32_t PROBE_NX = VM_PROBE_NX, PROBE_NY = VM_PROBE_NY, PROBE_NZ = VM_PROBE_NZ;

__device__ __forceinline__ float mixf(float a, float b, float t) { return a * (1.0f - t) + b * t; }   // WGSL mix
__device__ __forceinline__ F3 mix3(F3 a, F3 b, float t) { return {mixf(a.x, b.x, t), mixf(a.y, b.y, t), mixf(a.z, b.z, t)}; }
__device__ __forceinline__ F3 mix3v(F3 a, F3 b, F3 t) { return {mixf(a.x, b.x, t.x), mixf(a.y, b.y, t.y), mixf(a.z, b.z, t.z)}; }
__device__ __forceinline__ float clampf(float x, float lo, float hi) { return fminf(fmaxf(x, lo), hi); }
__device__ __forceinline__ float fractf(float x) { return x - floorf(x); }
__device__ __forceinline__ F3 add_s(F3 a, float s) { return {a.x + s, a.y + s, a.z + s}; }

// ---------------------------------------------------------------------------
// fog and sky: common.wgsl:1332-1396

__device__ __forceinline__ float transmittance_from(const vm_frame& f, float y0, float s, F3 rd) {
  const float lambda = f.fog_falloff;
  const float x = clampf(lambda * s * rd.y, -60.0f, 60.0f);
  float path = s;
  if (fabsf(x) > 1e-4f) path = wdiv(s * (1.0f - wexp(-x)), x);
  const float rho = f.fog_density * wexp(-clampf(lambda * (y0 - f.fog_height), -60.0f, 60.0f));
  return wexp(-clampf(rho * path, 0.0f, 60.0f));
}

__device__ __forceinline__ F3 scatter_tint() { return {1.0000f, 0.4770f, 0.1474f}; }

__device__ __forceinline__ float hg_gain(float cos_t, float g) {
  const float g2 = g * g;
  const float d = 1.0f + g2 - 2.0f * g * cos_t;
  return wdiv(1.0f - g2, wpow(fmaxf(d, 1e-4f), 1.5f));
}

__device__ __forceinline__ F3 scatter_lobe(const vm_frame& f, F3 rd) {
  const float sd = dot(rd, ld3(f.sun_dir));
  return scatter_tint() * (hg_gain(sd, f.fog_g) * f.fog_scatter * f.daylight);
}

constexpr uint32_t HI_SKY_SPECULAR = 1u, HI_SHORE_WET = 8u, HI_CAUSTICS = 64u, HI_TINT_BALANCE = 512u,
                   HI_SKY_LOOK = 1024u, HI_SKY_COOL = 2048u, HI_FOLIAGE_RICH = 8192u, HI_CANOPY_RELIEF = 16384u,
                   HI_LEGACY_LIGHTING = 1048576u;

__device__ __forceinline__ F3 sky_horizon(const Look& L, float day) {
  const F3 day_h = (L.spec_hi & HI_SKY_COOL) ? f3(0.4074f, 0.6057f, 0.9150f) : f3(0.4480f, 0.6210f, 0.8900f);
  return mix3(f3(0.0049f, 0.0060f, 0.0134f), day_h, day);
}
__device__ __forceinline__ F3 sky_zenith(const Look& L, float day) {
  const F3 day_z = (L.spec_hi & HI_SKY_COOL) ? f3(0.0385f, 0.1892f, 0.8600f) : f3(0.0637f, 0.2140f, 0.8276f);
  return mix3(f3(0.0008f, 0.0015f, 0.0039f), day_z, day);
}

static __device__ __noinline__ F3 sky_base(const vm_frame& f, const Look& L, F3 rd, float shaft) {
  const float day = f.daylight;
  const float up = clampf(rd.y, 0.0f, 1.0f);
  const F3 horizon = sky_horizon(L, day);
  const F3 zenith = sky_zenith(L, day);
  F3 c = mix3(horizon, zenith, wpow(up, 0.55f));
  const float sd = dot(rd, ld3(f.sun_dir));
  c = c + f3(1.0f, 0.8276f, 0.5225f) * wsmooth(0.9975f, 0.9990f, sd) * fmaxf(day, 0.2f);
  c = c + scatter_lobe(f, rd) * shaft;
  const bool look = (L.spec_hi & HI_SKY_LOOK) != 0u;
  if (look && f.haze_warm > 0.0f) {
    const float band = wpow(1.0f - up, 3.0f);
    const float toward = 0.35f + 0.65f * wpow(fmaxf(sd, 0.0f), 4.0f);
    c = c + scatter_tint() * (band * toward * f.haze_warm * day * 0.22f);
  }
  if (look && f.zenith_deep > 0.0f) {
    const float z = wpow(up, 0.55f);
    c = c * mix3(f3(1.0f, 1.0f, 1.0f), f3(0.80f, 0.90f, 1.16f), f.zenith_deep * z * day);
  }
  return mix3(c, horizon * 0.26f, wsmooth(0.0f, -0.35f, rd.y));
}

// ---------------------------------------------------------------------------
// clouds: common.wgsl:1422-1556

constexpr float CLOUD_SOFT = 0.14f, CLOUD_DEEP = 0.55f, CLOUD_FADE = 3.0e4f, CLOUD_MAX = 1.0e5f,
                CLOUD_PATCH_SPAN = 6.0f, SUN_ANGLE = 0.0093f;

__device__ __forceinline__ float cloud_lattice(int32_t cx, int32_t cy) {
  const uint32_t h = hash_u32((uint32_t)cx ^ (hash_u32((uint32_t)cy) * 0x9e3779b9u));
  return (float)(h >> 8u) * (1.0f / 16777216.0f);
}

__device__ __forceinline__ float cloud_noise(float px, float py) {
  const float ix = floorf(px), iy = floorf(py);
  const float fx = px - ix, fy = py - iy;
  const float wx = fx * fx * fx * (fx * (fx * 6.0f - 15.0f) + 10.0f);
  const float wy = fy * fy * fy * (fy * (fy * 6.0f - 15.0f) + 10.0f);
  const int32_t cx = __float2int_rz(ix), cy = __float2int_rz(iy);
  const int32_t cx1 = (int32_t)((uint32_t)cx + 1u), cy1 = (int32_t)((uint32_t)cy + 1u);
  const float a = cloud_lattice(cx, cy), b = cloud_lattice(cx1, cy);
  const float d = cloud_lattice(cx, cy1), e = cloud_lattice(cx1, cy1);
  return mixf(mixf(a, b, wx), mixf(d, e, wx), wy);
}

static __device__ __noinline__ float cloud_fbm(float px, float py, float fp) {
  float freq = 1.0f, amp = 1.0f, sum = 0.0f, norm = 0.0f;
#pragma unroll 1
  for (int i = 0; i < 4; ++i) {
    const float w = amp * (1.0f - wsmooth(0.25f, 0.5f, fp * freq));
    if (w > 0.0f) {
      sum += w * cloud_noise(px * freq, py * freq);
      norm += w;
    }
    freq *= 2.0f;
    amp *= 0.5f;
  }
  if (norm <= 0.0f) return 0.5f;
  return wdiv(sum, norm);
}

__device__ __forceinline__ float cloud_shade(const vm_frame& f, F3 p, float fp) {
  if (f.cloud_shadow <= 0.0f || f.cloud_cover <= 0.0f) return 1.0f;
  const float dy = f.cloud_height - p.y;
  if (dy * f.sun_dir[1] <= 0.0f) return 1.0f;
  const float t = wdiv(dy, f.sun_dir[1]);
  if (t > CLOUD_MAX) return 1.0f;
  const float qx = p.x + f.sun_dir[0] * t, qz = p.z + f.sun_dir[2] * t;
  const float drift = f.time * f.cloud_speed;
  const float n = cloud_fbm(wdiv(qx + 0.94f * drift, f.cloud_scale), wdiv(qz + 0.34f * drift, f.cloud_scale),
                            wdiv(fmaxf(fp, t * SUN_ANGLE), f.cloud_scale));
  const float thr = 1.0f - f.cloud_cover;
  return 1.0f - wsmooth(thr, thr + CLOUD_SOFT, n) * f.cloud_shadow;
}

__device__ __forceinline__ F3 cloud_radiance(const vm_frame& f, const Look& L, float dens, float depth, F3 rd) {
  const float day = f.daylight;
  const float thick = rd.y < 0.0f ? 0.0f : depth;
  const float warm = 1.0f - wsmooth(0.02f, 0.30f, f.sun_dir[1]);
  const F3 sun_tint = mix3(f3(1.0f, 1.0f, 1.0f), scatter_tint(), warm * 0.72f);
  const bool cool = (L.spec_hi & HI_SKY_COOL) != 0u;
  const F3 lit = cool ? f3(1.0f, 1.0f, 1.0f) : f3(1.0000f, 0.9575f, 0.8963f);
  const F3 base = cool ? f3(0.4420f, 0.4880f, 0.6010f) : f3(0.4854f, 0.5312f, 0.6462f);
  const F3 day_c = mix3(lit * sun_tint, base, thick);
  const F3 glow = scatter_tint() * (hg_gain(dot(rd, ld3(f.sun_dir)), 0.82f) * 0.055f * day * (1.0f - dens));
  return mix3(f3(0.0021f, 0.0026f, 0.0052f), day_c, day) + glow;
}

static __device__ __noinline__ F3 sky_color(const vm_frame& f, const Look& L, F3 ro, F3 rd, float travelled, float shaft) {
  const F3 base = sky_base(f, L, rd, shaft);
  if (f.cloud_cover <= 0.0f) return base;
  const float dy = f.cloud_height - ro.y;
  if (dy * rd.y <= 0.0f) return base;
  const float t = wdiv(dy, rd.y);
  if (t > CLOUD_MAX) return base;
  const float px = ro.x + rd.x * t, pz = ro.z + rd.z * t;
  const float px_angle = 2.0f * f.tan_half_fov / (float)f.res[1] * exp2f(f.mip_bias);
  const float fp = wdiv((travelled + t) * px_angle, fabsf(rd.y) * f.cloud_scale);
  const float drift = f.time * f.cloud_speed;
  const float qx = px + 0.94f * drift, qz = pz + 0.34f * drift;
  const float n = cloud_fbm(wdiv(qx, f.cloud_scale), wdiv(qz, f.cloud_scale), fp);
  float thr = 1.0f - f.cloud_cover;
  const bool look = (L.spec_hi & HI_SKY_LOOK) != 0u;
  if (look && f.cloud_patch > 0.0f) {
    const float span = f.cloud_scale * CLOUD_PATCH_SPAN;
    const float m = cloud_fbm(wdiv(qx, span), wdiv(qz, span), wdiv(fp, CLOUD_PATCH_SPAN));
    thr = clampf(thr + (m - 0.5f) * f.cloud_patch, 0.0f, 0.99f);
  }
  const float dens = wsmooth(thr, thr + CLOUD_SOFT, n);
  if (dens <= 0.0f) return base;
  float depth = wsmooth(thr, thr + CLOUD_DEEP, n);
  if (look && f.cloud_relief > 0.0f) {
    const float ax0 = f.sun_dir[0] + 1.0e-3f, az0 = f.sun_dir[2];
    const float al = sqrtf(ax0 * ax0 + az0 * az0);
    const float ax = wdiv(ax0, al), az = wdiv(az0, al);
    const float step = wdiv(8.0f + f.sun_dir[1] * 48.0f, f.cloud_scale);
    const float ns = cloud_fbm(wdiv(qx, f.cloud_scale) + ax * step, wdiv(qz, f.cloud_scale) + az * step, fp);
    depth = clampf(depth + (ns - n) * (2.2f * f.cloud_relief), 0.0f, 1.0f);
  }
  const float reach = 1.0f - wsmooth(CLOUD_FADE, CLOUD_MAX, t);
  const float a = dens * reach * transmittance_from(f, ro.y, t, rd);
  return mix3(base, cloud_radiance(f, L, dens, depth, rd), a);
}

// ---------------------------------------------------------------------------
// terrain shafts and sun shafts: common.wgsl:1557-1643

__device__ __forceinline__ float shaft_at(const Look& L, uint32_t x, uint32_t y) {
  return __ldg(L.shaft + (uint64_t)y * VM_SHAFT_DIM + x);
}

static __device__ __noinline__ float terrain_shade(const vm_frame& f, const Look& L, F3 p) {
  if (L.shaft == nullptr) return 1.0f;
  const float tx = wdiv(p.x - f.shaft_origin[0], f.shaft_texel) - 0.5f;
  const float tz = wdiv(p.z - f.shaft_origin[1], f.shaft_texel) - 0.5f;
  const float hi = (float)VM_SHAFT_DIM - 1.0f;
  const float cx = clampf(tx, 0.0f, hi), cz = clampf(tz, 0.0f, hi);
  const float f0x = floorf(cx), f0z = floorf(cz);
  const float frx = cx - f0x, frz = cz - f0z;
  const uint32_t i0x = __float2uint_rz(f0x), i0z = __float2uint_rz(f0z);
  const uint32_t i1x = min(i0x + 1u, VM_SHAFT_DIM - 1u), i1z = min(i0z + 1u, VM_SHAFT_DIM - 1u);
  const float a = shaft_at(L, i0x, i0z), b = shaft_at(L, i1x, i0z);
  const float c0 = shaft_at(L, i0x, i1z), d = shaft_at(L, i1x, i1z);
  const float e = mixf(mixf(a, b, frx), mixf(c0, d, frx), frz);
  return wsmooth(e - f.shaft_soft, e + f.shaft_soft, p.y);
}

__device__ __forceinline__ float dither(const vm_frame& f, uint32_t px, uint32_t py) {
  const float p0 = (float)px + 5.588238f * (float)f.frame_index;
  const float p1 = (float)py;
  return fractf(52.9829189f * fractf(p0 * 0.06711056f + p1 * 0.00583715f));
}

static __device__ __noinline__ float sun_shaft(const vm_frame& f, const Look& L, F3 ro, F3 rd, float dist, float alpha,
                                           uint32_t px, uint32_t py) {
  const bool terrain = (f.flags & VM_FLAG_TERRAIN_SHAFTS) != 0u;
  const bool deck = f.cloud_shadow > 0.0f && f.cloud_cover > 0.0f;
  if (f.godray_strength <= 0.0f) return 1.0f;
  if (!deck && !terrain) return 1.0f;
  const F3 lobe = scatter_lobe(f, rd);
  const float imp = wsmooth(0.0040f, 0.0120f, fmaxf(fmaxf(lobe.x, lobe.y), lobe.z) * alpha);
  if (imp <= 0.0f) return 1.0f;
  const float d = fminf(dist, f.godray_dist);
  if (d <= 0.0f) return 1.0f;
  const float opac = 1.0f - transmittance_from(f, ro.y, d, rd);
  if (opac <= 1e-6f) return 1.0f;
  const float lambda = f.fog_falloff;
  const float rho0 = f.fog_density * wexp(-clampf(lambda * (ro.y - f.fog_height), -60.0f, 60.0f));
  const float k = lambda * rd.y;
  const float off = dither(f, px, py);
  const float px_angle = 2.0f * f.tan_half_fov / (float)f.res[1] * exp2f(f.mip_bias);
  float sum = 0.0f;
  for (uint32_t i = 0; i < f.godray_steps; ++i) {
    const float u = wdiv((float)i + off, (float)f.godray_steps);
    const float path = wdiv(-wlog(1.0f - u * opac), rho0);
    float s = path;
    const float kp = k * path;
    if (fabsf(kp) > 1e-4f) s = wdiv(-wlog(fmaxf(1.0f - kp, 1e-6f)), k);
    s = clampf(s, 0.0f, d);
    const F3 p = ro + rd * s;
    float v = cloud_shade(f, p, s * px_angle);
    if (terrain) v = v * terrain_shade(f, L, p);
    sum += v;
  }
  const float vis = wdiv(sum, (float)f.godray_steps);
  float covered = 1.0f;
  if (d < dist) {
    const float full = 1.0f - transmittance_from(f, ro.y, dist, rd);
    if (full > 1e-6f) covered = fminf(wdiv(opac, full), 1.0f);
  }
  return fmaxf(mixf(1.0f, vis, imp * f.godray_strength * covered), 0.0f);
}

// ---------------------------------------------------------------------------
// light: common.wgsl:977-1096, resolve.wgsl:30-55

constexpr uint32_t LIGHT_OPEN_SKY = 0xF000u;

__device__ __forceinline__ uint32_t light_at(const DevWorld& w, const Chunk& c, int32_t x, int32_t y, int32_t z) {
  if ((c.light_flags & 1u) != 0u) return c.light_base;
  if (x < 0 || y < 0 || z < 0 || x > 63 || y > 63 || z > 63) return LIGHT_OPEN_SKY;
  const uint32_t ux = x, uy = y, uz = z;
  const uint32_t cell = (ux >> 2) | ((uy >> 2) << 4) | ((uz >> 2) << 8);
  const uint32_t entry = ld_brick(w, (uint64_t)c.light_base + cell);
  if ((entry & VM_UNIFORM_BIT) != 0u) return entry & 0xFFFFu;
  const uint32_t vb = cell_bit(ux & 3u, uy & 3u, uz & 3u);
  const uint32_t wd = ld_brick(w, (uint64_t)entry + (vb >> 1));
  return (wd >> ((vb & 1u) * 16u)) & 0xFFFFu;
}

// voxel_occludes: common.wgsl:942-975
__device__ __forceinline__ bool voxel_occludes(const DevWorld& w, const Chunk& c, int32_t x, int32_t y, int32_t z) {
  if (!voxel_occupied(w, c, x, y, z)) return false;
  if ((c.attr_flags & (VM_ATTR_HAS_WATER | VM_ATTR_HAS_FOLIAGE)) != 0u) {
    const uint32_t b = block_at(w, c, (uint32_t)x, (uint32_t)y, (uint32_t)z);
    return b != VM_WATER && !is_tuft(b);
  }
  return true;
}

// world_sample: common.wgsl:1015-1032 (light word, occluding bit)
static __device__ __noinline__ uint2 world_sample(const DevWorld& w, const vm_frame& f, F3 p) {
  uint64_t gi;
  if (!grid_rel(f, ffloor_i(p.x * INV64), ffloor_i(p.y * INV64), ffloor_i(p.z * INV64), &gi))
    return make_uint2(LIGHT_OPEN_SKY, 0u);
  const uint32_t ci = ld_grid(w, gi);
  if (ci == VM_NO_CHUNK) return make_uint2(LIGHT_OPEN_SKY, 0u);
  const Chunk c = ld_chunk(w, ci);
  const Scale s = make_scale(c.vs);
  const int32_t vx = ffloor_i(sdiv(p.x - c.origin[0], s));
  const int32_t vy = ffloor_i(sdiv(p.y - c.origin[1], s));
  const int32_t vz = ffloor_i(sdiv(p.z - c.origin[2], s));
  return make_uint2(light_at(w, c, vx, vy, vz), voxel_occludes(w, c, vx, vy, vz) ? 1u : 0u);
}

// gather_face: common.wgsl:1034-1096.  The nine air voxels of a face's 3x3
// neighbourhood inside one chunk: occupancy (only water cleared, unlike
// voxel_occludes, which also clears tufts) and light word.  The samples walk
// a 3x3 square, so the L1 node, leaf mask and light cell of the previous
// sample are kept, as the engine's loop keeps them.
static __device__ __noinline__ void gather_face(const DevWorld& w, const Chunk& c, int32_t bx, int32_t by, int32_t bz,
                                                int32_t tax, int32_t tay, int32_t taz, int32_t tbx, int32_t tby,
                                                int32_t tbz, uint2* out) {
  const uint32_t root_lo = c.root[0], root_hi = c.root[1];
  const bool root_full = (c.root[2] & VM_FULL_BIT) != 0u;
  const uint32_t root_ptr = c.root[2] & VM_PTR_MASK;
  const bool light_uniform = (c.light_flags & 1u) != 0u;
  const bool has_water = (c.attr_flags & VM_ATTR_HAS_WATER) != 0u;
  uint32_t l1_key = 0xFFFFFFFFu, leaf_key = 0xFFFFFFFFu, brick_key = 0xFFFFFFFFu;
  uint4 l1 = make_uint4(0u, 0u, 0u, 0u);
  uint2 leaf = make_uint2(0u, 0u);
  uint32_t brick = 0u;
  for (int i = 0; i < 9; ++i) {
    const int32_t da = i % 3 - 1, db = i / 3 - 1;
    const uint32_t ux = (uint32_t)(bx + tax * da + tbx * db), uy = (uint32_t)(by + tay * da + tby * db),
                   uz = (uint32_t)(bz + taz * da + tbz * db);
    bool solid = false;
    const uint32_t l1b = cell_bit(ux >> 4, uy >> 4, uz >> 4);
    if (mask_has(root_lo, root_hi, l1b)) {
      if (root_full) {
        solid = true;
      } else {
        if (l1b != l1_key) {
          l1_key = l1b;
          l1 = ld_inner(w, (uint64_t)root_ptr + mask_below(root_lo, root_hi, l1b));
          leaf_key = 0xFFFFFFFFu;
        }
        const uint32_t lfb = cell_bit((ux >> 2) & 3u, (uy >> 2) & 3u, (uz >> 2) & 3u);
        if ((l1.z & VM_FULL_BIT) != 0u) {
          solid = true;
        } else if (mask_has(l1.x, l1.y, lfb)) {
          if (lfb != leaf_key) {
            leaf_key = lfb;
            leaf = ld_leaf(w, (uint64_t)(l1.z & VM_PTR_MASK) + mask_below(l1.x, l1.y, lfb));
          }
          solid = mask_has(leaf.x, leaf.y, cell_bit(ux & 3u, uy & 3u, uz & 3u));
        }
      }
    }
    if (solid && has_water) solid = block_at(w, c, ux, uy, uz) != VM_WATER;
    uint32_t packed = c.light_base;
    if (!light_uniform) {
      const uint32_t cell = (ux >> 2) | ((uy >> 2) << 4) | ((uz >> 2) << 8);
      if (cell != brick_key) {
        brick_key = cell;
        brick = ld_brick(w, (uint64_t)c.light_base + cell);
      }
      if ((brick & VM_UNIFORM_BIT) != 0u) {
        packed = brick & 0xFFFFu;
      } else {
        const uint32_t vb = cell_bit(ux & 3u, uy & 3u, uz & 3u);
        packed = (ld_brick(w, (uint64_t)brick + (vb >> 1)) >> ((vb & 1u) * 16u)) & 0xFFFFu;
      }
    }
    out[i] = make_uint2(packed, solid ? 1u : 0u);
  }
}

__device__ __forceinline__ float light_sky(uint32_t p) { return (float)(p >> 12u); }
__device__ __forceinline__ F3 light_block_rgb(uint32_t p) {
  return {(float)((p >> 8u) & 0xFu), (float)((p >> 4u) & 0xFu), (float)(p & 0xFu)};
}
__device__ __forceinline__ float light_block_level(uint32_t p) {
  const F3 c = light_block_rgb(p);
  return fmaxf(c.x, fmaxf(c.y, c.z));
}
__device__ __forceinline__ float light_curve(float level) {
  const float l = wdiv(level, 15.0f);
  return l * l * (0.6f + 0.4f * l);
}
__device__ __forceinline__ F3 light_curve3(F3 level) {
  const F3 l = wdiv3(level, 15.0f);
  return l * l * add_s(l * 0.4f, 0.6f);
}
__device__ __forceinline__ F3 block_ambient(F3 blk, float sk, F3 sky) {
  const float bk = fmaxf(blk.x, fmaxf(blk.y, blk.z));
  const F3 tint = wdiv3(blk, fmaxf(bk, 1e-4f));
  return mix3(sky, tint, wdiv(bk, fmaxf(sk + bk, 1e-4f))) * fmaxf(sk, bk);
}
__device__ __forceinline__ F3 block_tint() { return {1.0000f, 0.6500f, 0.3200f}; }

// sky_ambient_tint / surface_sky_fill: resolve.wgsl:1-5, 73-89 (SPEC_SKY_TINT
// on, FLAG_SKY_TINT of the frame)
__device__ __forceinline__ F3 sky_ambient_tint(const vm_frame& f, const Look& L, F3 n) {
  const F3 sky_tint = {0.6038f, 0.7084f, 1.0000f};
  if ((f.flags & VM_FLAG_SKY_TINT) == 0u) return sky_tint;
  const float day = f.daylight;
  const F3 horizon = mix3(f3(0.0049f, 0.0060f, 0.0134f), f3(0.4480f, 0.6210f, 0.8900f), day);
  const F3 zenith = mix3(f3(0.0008f, 0.0015f, 0.0039f), f3(0.0637f, 0.2140f, 0.8276f), day);
  const float wgt = n.y < -0.5f ? 0.0f : (n.y > 0.5f ? 0.78431373f : 0.58578900f);
  F3 c = mix3(horizon, zenith, wgt);
  c = c + scatter_tint() * (f.fog_scatter * day * 4.0f * fmaxf(dot(n, ld3(f.sun_dir)), 0.0f));
  const F3 ref = {0.14658824f, 0.30178431f, 0.84105882f};
  const F3 t = sky_tint * f3(wpow(wdiv(c.x, ref.x), 2.5f), wpow(wdiv(c.y, ref.y), 2.5f),
                             wpow(wdiv(c.z, ref.z), 2.5f));
  const float luma = 0.2126f * t.x + 0.7152f * t.y + 0.0722f * t.z;
  return t * wdiv(0.70721556f, fmaxf(luma, 1e-6f));
}
__device__ __forceinline__ bool lighting_repair(const Look& L) { return (L.spec_hi & HI_LEGACY_LIGHTING) == 0u; }
// SURFACE_DEBUG: (spec_hi >> 23) & 7 (FLAG_HI_DEBUG_A..C, mod.rs make_spec)
__host__ __device__ __forceinline__ uint32_t surface_debug(const Look& L) { return (L.spec_hi >> 23) & 7u; }
static __device__ __noinline__ F3 surface_sky_fill(const vm_frame& f, const Look& L, F3 n) {
  const F3 sky = sky_ambient_tint(f, L, n);
  if (!lighting_repair(L)) return sky;
  return sky * (0.60f * mixf(0.35f, 1.0f, clampf(n.y * 0.5f + 0.5f, 0.0f, 1.0f)));
}

// ---------------------------------------------------------------------------
// texture sampling

// The atlas (Rgba8UnormSrgb, 16x16 layers, 4 mips) through the engine's
// sampler (mag nearest, min and mipmap linear, clamp to edge) at an explicit
// level: level <= 0 magnifies (nearest texel of mip 0), otherwise the two
// mips around the level are sampled bilinearly and blended.
__device__ __forceinline__ uint64_t atlas_mip_base(uint32_t layers, uint32_t mip) {
  uint64_t base = 0;
  for (uint32_t m = 0; m < mip; ++m) base += (uint64_t)layers * (ATLAS_SIZE >> m) * (ATLAS_SIZE >> m);
  return base;
}
__device__ __forceinline__ float4 atlas_texel(const Look& L, uint64_t base, uint32_t size, uint32_t layer, int32_t x,
                                              int32_t y) {
  x = min(max(x, 0), (int32_t)size - 1);
  y = min(max(y, 0), (int32_t)size - 1);
  return __ldg(L.atlas + base + ((uint64_t)layer * size + (uint32_t)y) * size + (uint32_t)x);
}
__device__ __forceinline__ float4 mix4(float4 a, float4 b, float t) {
  return make_float4(mixf(a.x, b.x, t), mixf(a.y, b.y, t), mixf(a.z, b.z, t), mixf(a.w, b.w, t));
}
__device__ __forceinline__ float4 atlas_bilinear(const Look& L, uint32_t mip, uint32_t layer, float u, float v) {
  const uint32_t size = ATLAS_SIZE >> mip;
  const uint64_t base = atlas_mip_base(L.atlas_layers, mip);
  const float x = u * (float)size - 0.5f, y = v * (float)size - 0.5f;
  const float x0 = floorf(x), y0 = floorf(y);
  const float ax = x - x0, ay = y - y0;
  const int32_t ix = ffloor_i(x0), iy = ffloor_i(y0);
  const int32_t ix1 = (int32_t)((uint32_t)ix + 1u), iy1 = (int32_t)((uint32_t)iy + 1u);
  const float4 t00 = atlas_texel(L, base, size, layer, ix, iy), t10 = atlas_texel(L, base, size, layer, ix1, iy);
  const float4 t01 = atlas_texel(L, base, size, layer, ix, iy1), t11 = atlas_texel(L, base, size, layer, ix1, iy1);
  return mix4(mix4(t00, t10, ax), mix4(t01, t11, ax), ay);
}
static __device__ __noinline__ float4 atlas_sample(const Look& L, float u, float v, uint32_t layer, float lod) {
  layer = min(layer, L.atlas_layers - 1u);   // an array index past the last layer reads the last one
  if (!(lod > 0.0f)) {
    const int32_t x = ffloor_i(u * (float)ATLAS_SIZE), y = ffloor_i(v * (float)ATLAS_SIZE);
    return atlas_texel(L, 0, ATLAS_SIZE, layer, x, y);
  }
  const float d = fminf(lod, (float)(ATLAS_MIPS - 1));
  const float dl = floorf(d);
  const float delta = d - dl;
  const uint32_t m0 = __float2uint_rz(dl);
  const float4 a = atlas_bilinear(L, m0, layer, u, v);
  if (!(delta > 0.0f) || m0 + 1u >= ATLAS_MIPS) return a;
  return mix4(a, atlas_bilinear(L, m0 + 1u, layer, u, v), delta);
}

// The probe field (Rgba16Float, 128 x 768 x 128) through the probe sampler
// (linear; repeat in u and w, clamp to edge in v).
__device__ __forceinline__ float4 probe_texel(const Look& L, int32_t x, int32_t y, int32_t z) {
  x = ((x % (int32_t)PROBE_NX) + (int32_t)PROBE_NX) % (int32_t)PROBE_NX;
  z = ((z % (int32_t)PROBE_NZ) + (int32_t)PROBE_NZ) % (int32_t)PROBE_NZ;
  y = min(max(y, 0), (int32_t)PROBE_NY - 1);
  const ushort4 h = __ldg(L.probes + ((uint64_t)(uint32_t)z * PROBE_NY + (uint32_t)y) * PROBE_NX + (uint32_t)x);
  return make_float4(__half2float(__ushort_as_half(h.x)), __half2float(__ushort_as_half(h.y)),
                     __half2float(__ushort_as_half(h.z)), __half2float(__ushort_as_half(h.w)));
}
static __device__ __noinline__ float4 probe_field(const Look& L, F3 p, uint32_t nid) {
  if (L.probes == nullptr) return make_float4(1.0f, 1.0f, 1.0f, 1.0f);
  const uint32_t slab = nid >= VM_NORMAL_CROSS_A ? 3u : nid;
  const F3 t = p * 0.25f;
  const float y = clampf(t.y, 0.5f, 127.5f);
  const float u = t.x * (1.0f / 128.0f);
  const float v = ((float)slab * 128.0f + y) * (1.0f / 768.0f);
  const float w = t.z * (1.0f / 128.0f);
  const float x = u * (float)PROBE_NX - 0.5f, yy = v * (float)PROBE_NY - 0.5f, z = w * (float)PROBE_NZ - 0.5f;
  const float x0 = floorf(x), y0 = floorf(yy), z0 = floorf(z);
  const float ax = x - x0, ay = yy - y0, az = z - z0;
  const int32_t ix = ffloor_i(x0), iy = ffloor_i(y0), iz = ffloor_i(z0);
  float4 s[2];
#pragma unroll
  for (int dz = 0; dz < 2; ++dz) {
    const float4 a = mix4(probe_texel(L, ix, iy, iz + dz), probe_texel(L, ix + 1, iy, iz + dz), ax);
    const float4 b = mix4(probe_texel(L, ix, iy + 1, iz + dz), probe_texel(L, ix + 1, iy + 1, iz + dz), ax);
    s[dz] = mix4(a, b, ay);
  }
  return mix4(s[0], s[1], az);
}

// probe_tap (resolve.wgsl:120-127, PROBE_TAPS = 1): the probe field through
// the engine's linear sampler (linear filtering, clamp to edge on every
// axis) at fract(p / (PROBE_DIM * PROBE_SPACING)).
__device__ __forceinline__ float4 probe_texel_clamped(const Look& L, int32_t x, int32_t y, int32_t z) {
  return probe_texel(L, min(max(x, 0), (int32_t)PROBE_NX - 1), y, min(max(z, 0), (int32_t)PROBE_NZ - 1));
}
static __device__ __noinline__ F3 probe_tap(const Look& L, F3 p) {
  if (L.probes == nullptr) return {1.0f, 1.0f, 1.0f};
  const float inv_span = 1.0f / ((float)PROBE_NX * 4.0f);
  const float u = fractf(p.x * inv_span), v = fractf(p.y * inv_span), w = fractf(p.z * inv_span + 0.0f);
  const float x = u * (float)PROBE_NX - 0.5f, yy = v * (float)PROBE_NY - 0.5f, z = w * (float)PROBE_NZ - 0.5f;
  const float x0 = floorf(x), y0 = floorf(yy), z0 = floorf(z);
  const float ax = x - x0, ay = yy - y0, az = z - z0;
  const int32_t ix = ffloor_i(x0), iy = ffloor_i(y0), iz = ffloor_i(z0);
  float4 s[2];
#pragma unroll
  for (int dz = 0; dz < 2; ++dz) {
    const float4 a = mix4(probe_texel_clamped(L, ix, iy, iz + dz), probe_texel_clamped(L, ix + 1, iy, iz + dz), ax);
    const float4 b =
        mix4(probe_texel_clamped(L, ix, iy + 1, iz + dz), probe_texel_clamped(L, ix + 1, iy + 1, iz + dz), ax);
    s[dz] = mix4(a, b, ay);
  }
  const float4 r = mix4(s[0], s[1], az);
  return f3(1.0f, 1.0f, 1.0f) * f3(r.x, r.y, r.z);
}

// ---------------------------------------------------------------------------
// surface material: resolve.wgsl:129-165, 166-285

__device__ __forceinline__ void face_uv(uint32_t nid, F3 local, float* u, float* v) {
  if (nid >= VM_NORMAL_CROSS_A) { *u = local.x; *v = 1.0f - local.y; return; }
  const uint32_t axis = nid >> 1u;
  if (axis == 0u) { *u = local.z; *v = 1.0f - local.y; }
  else if (axis == 1u) { *u = local.x; *v = local.z; }
  else { *u = local.x; *v = 1.0f - local.y; }
  if (nid == 1u || nid == 4u) *u = 1.0f - *u;
}

__device__ __forceinline__ uint32_t perm_key(F3 box_min, uint32_t nid) {
  const int32_t cx = ffloor_i(floorf(box_min.x)), cy = ffloor_i(floorf(box_min.y)), cz = ffloor_i(floorf(box_min.z));
  return hash_u32(((uint32_t)cx * 0x9e3779b9u) ^ ((uint32_t)cy * 0x85ebca6bu) ^ ((uint32_t)cz * 0xc2b2ae35u) ^
                  (nid * 0x27d4eb2fu));
}

__device__ __forceinline__ void permute_uv(float* u, float* v, uint32_t pclass, uint32_t h) {
  const bool d4 = pclass == 2u;
  float px = *u, py = *v;
  if (d4 && (h & 1u) != 0u) { const float t = px; px = py; py = t; }
  if (pclass != 0u && (h & 2u) != 0u) px = 1.0f - px;
  if (d4 && (h & 4u) != 0u) py = 1.0f - py;
  *u = px; *v = py;
}

__device__ __forceinline__ float hash_alpha(F3 p) {
  const int32_t qx = ffloor_i(floorf(p.x * 64.0f)), qy = ffloor_i(floorf(p.y * 64.0f)), qz = ffloor_i(floorf(p.z * 64.0f));
  uint32_t h = ((uint32_t)qx * 73856093u) ^ ((uint32_t)qy * 19349663u) ^ ((uint32_t)qz * 83492791u);
  h = h ^ (h >> 13u);
  h = h * 1274126177u;
  return (float)((h >> 8u) & 0xFFFFFFu) / 16777216.0f;
}

// biome noise: OpenSimplex2 2D (resolve.wgsl:180-257); the cos / sin of the
// gradient angles come from a table made once on the host.
__device__ __forceinline__ float simplex_grad(const Look& L, uint32_t seed, uint32_t xp, uint32_t yp, float xd, float yd) {
  const uint32_t h = (seed ^ xp ^ yp) * 0x27d4eb2du;
  const int32_t hs = (int32_t)h;
  const uint32_t idx = (uint32_t)((hs ^ (hs >> 15)) & 254);
  const uint32_t k = idx < 240u ? ((idx % 48u) >> 1u) : 24u + ((idx - 240u) >> 1u);
  const float2 cs = __ldg(L.grad + k);
  return xd * cs.x + yd * cs.y;
}
__device__ __forceinline__ int32_t biome_fast_floor(float f) {
  const int32_t i = __float2int_rz(f);
  return f >= 0.0f ? i : i - 1;
}
static __device__ __noinline__ float biome_noise(const Look& L, int32_t seed_i, float freq, float px, float pz) {
  const uint32_t seed = (uint32_t)seed_i;
  const float sqrt3 = 1.7320508075688772f;
  const float g2 = (3.0f - sqrt3) / 6.0f;
  const float f2 = 0.5f * (sqrt3 - 1.0f);
  float x = px * freq, y = pz * freq;
  const float s = (x + y) * f2;
  x = x + s; y = y + s;
  const int32_t i0 = biome_fast_floor(x), j0 = biome_fast_floor(y);
  const float xi = x - (float)i0, yi = y - (float)j0;
  const float t = (xi + yi) * g2;
  const float x0 = xi - t, y0 = yi - t;
  const uint32_t PX = 501125321u, PY = 1136930381u;
  const uint32_t i = (uint32_t)i0 * PX, j = (uint32_t)j0 * PY;
  const float a = 0.5f - x0 * x0 - y0 * y0;
  float n0 = 0.0f;
  if (a > 0.0f) n0 = (a * a) * (a * a) * simplex_grad(L, seed, i, j, x0, y0);
  const float c = (2.0f * (1.0f - 2.0f * g2) * (1.0f / g2 - 2.0f)) * t +
                  ((-2.0f * (1.0f - 2.0f * g2) * (1.0f - 2.0f * g2)) + a);
  float n2 = 0.0f;
  if (c > 0.0f) {
    const float x2 = x0 + (2.0f * g2 - 1.0f), y2 = y0 + (2.0f * g2 - 1.0f);
    n2 = (c * c) * (c * c) * simplex_grad(L, seed, i + PX, j + PY, x2, y2);
  }
  float n1 = 0.0f;
  if (y0 > x0) {
    const float x1 = x0 + g2, y1 = y0 + (g2 - 1.0f);
    const float b = 0.5f - x1 * x1 - y1 * y1;
    if (b > 0.0f) n1 = (b * b) * (b * b) * simplex_grad(L, seed, i, j + PY, x1, y1);
  } else {
    const float x1 = x0 + (g2 - 1.0f), y1 = y0 + g2;
    const float b = 0.5f - x1 * x1 - y1 * y1;
    if (b > 0.0f) n1 = (b * b) * (b * b) * simplex_grad(L, seed, i + PX, j, x1, y1);
  }
  return (n0 + n1 + n2) * 99.83685446303647f;
}
__device__ __forceinline__ F3 biome_band_weights(float n) {
  const float hot = wsmooth(0.22f - 0.18f, 0.22f + 0.18f, n);
  const float cold = 1.0f - wsmooth(-0.22f - 0.18f, -0.22f + 0.18f, n);
  return {cold, 1.0f - cold - hot, hot};
}
__device__ __forceinline__ F3 biome_tint(const vm_frame& f, const Look& L, float x, float z) {
  const float temperature = biome_noise(L, (int32_t)((uint32_t)f.tint_seed + 7u), f.tint_freq_t, x, z);
  const float humidity = biome_noise(L, (int32_t)((uint32_t)f.tint_seed + 8u), f.tint_freq_h, x, z);
  const F3 wt = biome_band_weights(temperature), wh = biome_band_weights(humidity);
  const F3 plains = (L.spec_hi & HI_TINT_BALANCE) ? f3(0.935f, 1.067f, 0.892f) : f3(1.0f, 1.0f, 1.0f);
  const F3 forest = {0.664f, 1.045f, 1.000f}, savanna = {1.842f, 0.935f, 0.793f}, desert = {2.096f, 0.957f, 0.699f};
  const F3 taiga = {0.832f, 0.935f, 2.096f}, tundra = {0.755f, 0.893f, 2.812f};
  const F3 dry = tundra * wt.x + plains * wt.y + desert * wt.z;
  const F3 mid = taiga * wt.x + plains * wt.y + savanna * wt.z;
  const F3 wet = taiga * wt.x + forest * wt.y + forest * wt.z;
  return dry * wh.x + mid * wh.y + wet * wh.z;
}

__device__ __forceinline__ float schlick_ground(float cos_i) {
  const float m = clampf(1.0f - cos_i, 0.0f, 1.0f);
  const float m2 = m * m;
  const float top = fmaxf(1.0f - 0.9f, 0.04f);
  return 0.04f + (top - 0.04f) * m2 * m2 * m;
}

__device__ __forceinline__ float face_shade(uint32_t nid) {
  switch (nid) {
    case 3u: return 1.00f;
    case 2u: return 0.50f;
    case 4u: case 5u: return 0.80f;
    case 6u: case 7u: return 0.90f;
    default: return 0.62f;
  }
}

// ---------------------------------------------------------------------------
// shade_hit_legacy (resolve.wgsl:289-585) and its cached form
// (resolve.wgsl:1537-1788): lit_in >= 0 is the frame's sun visibility of a
// primary hit (the cached form), lit_in < 0 traces shadow_ray from the hit
// over shadow_dist (the secondary legs).  smooth: the 3x3 smooth light with
// AO, else the single light sample of the voxel in front of the face.
// pre: the hit's light terms when a stage computed them, else null.  EXTRA:
// the frame may use the probe-tap / probe-ambient variants or a surface debug
// view (without it their branches are compiled out).
struct LightTerms { F3 amb; float sky_sm, ao; };   // ambient colour, smoothed sky light, AO
template <bool EXTRA>
__device__ __noinline__ F3 shade_surface(const DevWorld& w, const vm_frame& f, const Look& L, uint32_t ci, uint32_t vx,
                                         uint32_t vy, uint32_t vz, uint32_t id, uint32_t nid, F3 hit, F3 rd, float dist,
                                         float shadow_dist, bool smooth, bool do_spec, float lit_in,
                                         const LightTerms* pre);

}  // namespace vmd
