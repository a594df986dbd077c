// Per-ray stages shared by the march kernels: key decoding, the shadow ray
// set-up of shadow_guide and the one water / glass secondary ray per hit.
#pragma once
#include "march_device.cuh"
#include "water.cuh"

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

// Glass is its own surface (no sun-shadow ray of its own, a transmission
// leg) only with SPEC_GLASS (shadow.wgsl:18, resolve.wgsl:1440); without it
// glass blocks shade as opaque blocks.
__device__ __forceinline__ bool is_glass_leg(uint32_t spec, uint32_t id) {
  return (spec & VM_SPEC_GLASS) != 0u && id == VM_GLASS;
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
  if (id == VM_WATER || (is_glass_leg(w.spec, id))) return false;
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

// Soft shadows (VM_SPEC_SOFT_RAYS): the s-th jittered sun direction of
// pixel (px, py) at the frame's frame_index.  Tangent basis of the sun
// direction from a fixed up vector, one of VM_SOFT_ROTATIONS rotations of the
// disk pattern per pixel (the engine's hash_u32 of pixel and frame), offset
// added in the tangent plane, normalised (v / sqrt(dot)).
__device__ static const float g_soft_disk[VM_SOFT_ROTATIONS][VM_SOFT_SAMPLES][2] = VM_SOFT_DISK_INIT;
__device__ __forceinline__ bool soft_shadows(uint32_t spec) { return (spec & VM_SPEC_SOFT_RAYS) != 0u; }
__device__ __forceinline__ F3 soft_sun_dir(const vm_frame& f, uint32_t px, uint32_t py, uint32_t s) {
  const F3 sun = ld3(f.sun_dir);
  const F3 up = fabsf(sun.y) < 0.99f ? f3(0.0f, 1.0f, 0.0f) : f3(1.0f, 0.0f, 0.0f);
  const F3 c = cross(sun, up);
  const float lc = sqrtf(dot(c, c));
  const F3 tg = {c.x / lc, c.y / lc, c.z / lc};
  const F3 bt = cross(tg, sun);
  const uint32_t r = hash_u32((px * 73856093u) ^ (py * 19349663u) ^ (f.frame_index * 83492791u)) &
                     (VM_SOFT_ROTATIONS - 1u);
  const F3 v = (sun + tg * g_soft_disk[r][s][0]) + bt * g_soft_disk[r][s][1];
  const float l = sqrtf(dot(v, v));
  return {v.x / l, v.y / l, v.z / l};
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
  const bool water = id == VM_WATER, glass = is_glass_leg(w.spec, id);
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

// The reflect leg of a water hit (water_reflect_leg, resolve.wgsl:1044-1058,
// scheduled by water_sec resolve.wgsl:1526-1528): gated by FLAG_WATER_REFLECT
// and reflect_detail > 0 (resolve.wgsl:1099); from hit + n * SURFACE_EPS (the
// face normal) along water_ctx's mirror_t (water.cuh: the face normal's
// reflection, or the wave normal's on a waved +Y face), 768 voxels, water
// transparent.
__device__ __forceinline__ bool water_reflects(const vm_frame& f, float t) {
  if ((f.flags & VM_FLAG_WATER_REFLECT) == 0u) return false;
  return 1.0f - smoothstep(VM_WATER_REFLECT_NEAR, VM_WATER_REFLECT_FAR, t) > 0.0f;
}
template <bool COUNT, bool TUFTS = false>
__device__ __forceinline__ SecRay reflect_ray(const DevWorld& w, const vm_frame& f, F3 hit, F3 rd, uint32_t nid,
                                              float t, Traffic* tr) {
  SecRay s;
  s.o = hit + normal_of(nid) * VM_SURFACE_EPS;
  s.d = water_mirror_t<COUNT, TUFTS>(w, f, nid, hit, rd, t, tr);
  s.max_dist = VM_WATER_REFLECT_DIST;
  s.water = true;
  return s;
}
template <bool TUFTS>
__device__ __forceinline__ bool reflect_setup(const DevWorld& w, const vm_frame& f, unsigned long long key,
                                              uint32_t px, uint32_t py, SecRay* s) {
  if (key == 0ull) return false;
  const KeyParts k = split_key(key);
  const Chunk c = ld_chunk(w, k.ci);
  if (block_at(w, c, k.vx, k.vy, k.vz) != VM_WATER) return false;
  const F3 rd = ray_dir(f, (float)px + 0.5f, (float)py + 0.5f);
  const float t = hit_t(f, c, k.vx, k.vy, k.vz, k.mx, k.my, k.mz, k.nid, rd);
  if (!water_reflects(f, t)) return false;
  *s = reflect_ray<false, TUFTS>(w, f, ld3(f.cam_pos) + rd * t, rd, k.nid, t, nullptr);
  return true;
}

template <bool COUNT, bool TUFTS>
__device__ __forceinline__ void secondary_trace(const DevWorld& w, const vm_frame& f, const SecRay& s,
                                                unsigned long long* out_key, float* out_t, Traffic* tr) {
  const WorldHit h = s.water ? trace_world<true, COUNT, TUFTS>(w, f, s.o, s.d, s.max_dist, tr)
                             : trace_world<false, COUNT, TUFTS>(w, f, s.o, s.d, s.max_dist, tr);
  unsigned long long k = (1ull << 63) | (s.water ? 0ull : (1ull << 61));
  if (h.hit)
    k |= (1ull << 62) | ((unsigned long long)h.normal << 37) | ((unsigned long long)h.ci << 24) |
         (unsigned long long)((h.vx << 16) | (h.vy << 8) | h.vz);
  *out_key = k;
  *out_t = h.t;
}

}  // namespace vmk
