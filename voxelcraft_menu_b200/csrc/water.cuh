// The water surface of a hit: the reflect direction of water_ctx
// (resolve.wgsl:1078-1166), which on a waved surface comes from the wave
// field (wave_octave / wave_field / wave_normal, resolve.wgsl:902-975) with
// its anisotropic filter, the shoal-depth damping (a short downward
// trace_world) and the optical roughness that pulls the normal back to the
// face normal.  Compiled with the march's float contract; cos and exp are
// CUDA's, the oracle uses the host's, so on a waved surface with a positive
// reflect slope the direction can differ in its last bits.  With the
// engine's default slope of 0 the traced normal is the face normal whatever
// the wave field is, and the direction is exact.
#pragma once
#include "march_device.cuh"

namespace vmd {

constexpr float WAVE_TAU = 6.28318531f;
constexpr float WAVE_GRAZE_MIN = 1e-3f;
constexpr float SHOAL_DEPTH = 6.0f;
constexpr float WAVE_FILTER_K = 1.0f;

// one octave: slope vector and the unresolved slope variance it leaves
__device__ __forceinline__ F3 wave_octave(float px_, float pz_, float dx, float dz, float lambda, float slope,
                                          float phase, float px, float vhx, float vhz, float kk, bool aniso) {
  float fade;
  if (aniso) {
    const float d = dx * vhx + dz * vhz;
    const float ext = px * sqrtf(1.0f + kk * d * d);
    const float u = ext / lambda;
    fade = expf(-WAVE_FILTER_K * u * u);
  } else {
    fade = smoothstep(2.0f, 4.0f, lambda / fmaxf(px, 1e-4f));
  }
  const float s = slope * fade * cosf(WAVE_TAU / lambda * (px_ * dx + pz_ * dz) + phase);
  return {dx * s, dz * s, 0.5f * slope * slope * (1.0f - fade * fade)};
}

// the octaves of wave_field (resolve.wgsl:944-965): direction x, z, the
// wavelength divisor, the amplitude share and the phase rate; FLAG_WAVE_FILL's
// eight, else the base four
static __constant__ float WAVE_FILL_OCTAVES[8][5] = {
    {-0.438371f, 0.898794f, 1.0f, 0.3086f, 1.0000f},    {-0.927184f, 0.374607f, 1.3934f, 0.2584f, 1.1804f},
    {-0.190809f, 0.981627f, 1.9417f, 0.2163f, 1.3934f}, {-0.669131f, 0.743145f, 2.7056f, 0.1810f, 1.6449f},
    {0.121869f, 0.992546f, 3.7700f, 0.1515f, 1.9417f},  {0.694658f, 0.719340f, 5.2533f, 0.1269f, 2.2920f},
    {0.970296f, 0.241922f, 7.3201f, 0.1062f, 2.7056f},  {0.438371f, 0.898794f, 10.2000f, 0.0889f, 3.1937f}};
static __constant__ float WAVE_BASE_OCTAVES[4][5] = {{0.913089f, 0.407760f, 1.0f, 0.42f, 1.0000f},
                                                     {-0.388685f, 0.921371f, 2.17f, 0.27f, 1.4731f},
                                                     {-0.980382f, -0.197108f, 4.71f, 0.19f, 2.1703f},
                                                     {0.477328f, -0.878725f, 10.20f, 0.12f, 3.1937f}};

// wave_field: the sum of the octaves (8 with FLAG_WAVE_FILL, else 4).  The
// loop stays rolled: unrolled, its transcendentals made the kernels that
// shade water outgrow the instruction cache.
__device__ __forceinline__ F3 wave_field(const vm_frame& f, float x, float z, float px, float vhx, float vhz, float kk,
                                         bool aniso, float shoal) {
  const float l0 = f.wave_scale;
  const float a = f.wave_amp * shoal;
  const float ph = f.time * f.wave_speed * WAVE_TAU;
  const bool fill = (f.flags & VM_FLAG_WAVE_FILL) != 0u;
  const float (*tab)[5] = fill ? WAVE_FILL_OCTAVES : WAVE_BASE_OCTAVES;
  const int n = fill ? 8 : 4;
  F3 s = {0.0f, 0.0f, 0.0f};
#pragma unroll 1
  for (int i = 0; i < n; ++i) {
    const float lambda = i == 0 ? l0 : l0 / tab[i][2];
    s = s + wave_octave(x, z, tab[i][0], tab[i][1], lambda, a * tab[i][3], ph * tab[i][4], px, vhx, vhz, kk, aniso);
  }
  return s;
}

__device__ __forceinline__ F3 unit(F3 v) {   // WGSL normalize: v / sqrt(dot(v, v))
  const float l = sqrtf(dot(v, v));
  return {v.x / l, v.y / l, v.z / l};
}

// The direction water_reflect_leg traces from a water hit (water_ctx's
// mirror_t): reflect(rd, nt), with nt the wave normal for FLAG_WAVES on a +Y
// face, limited by wave_reflect_slope and pulled to the face normal by the
// optical roughness; a waved direction never points below the horizon.
template <bool COUNT, bool TUFTS = false>
__device__ __forceinline__ F3 water_mirror_t(const DevWorld& w, const vm_frame& f, uint32_t nid, F3 hit, F3 rd,
                                             float t, Traffic* tr) {
  const F3 n = normal_of(nid);
  F3 nt = n;
  float unresolved = 0.0f;
  const bool waved = (f.flags & VM_FLAG_WAVES) != 0u && nid == VM_NORMAL_PY;
  if (waved) {
    const float px_world = fmaxf(t, 1e-3f) * 2.0f * f.tan_half_fov / (float)f.res[1];
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
      const WorldHit dh = trace_world<true, COUNT, TUFTS>(w, f, dro, f3(0.001f, -0.999999f, 0.001f), SHOAL_DEPTH, tr);
      shoal = smoothstep(0.0f, SHOAL_DEPTH, dh.hit ? dh.t : SHOAL_DEPTH);
    }
    const F3 wf = wave_field(f, hit.x, hit.z, px_world, vhx, vhz, kk, aniso, shoal);
    unresolved = fmaxf(wf.z, 0.0f);
    const float gl = sqrtf(wf.x * wf.x + wf.y * wf.y);
    const float lim = fminf(1.0f, f.wave_reflect_slope / fmaxf(gl, 1e-6f));
    nt = unit(f3(-(wf.x * lim), 1.0f, -(wf.y * lim)));   // wave_normal
  }
  const float rough = fminf(fmaxf(1.0f - expf(-8.0f * unresolved), 0.0f), 1.0f);
  nt = unit(nt * (1.0f - rough) + n * rough);              // normalize(mix(nt, n, rough))
  F3 m = reflect(rd, nt);
  if (waved) m = unit(f3(m.x, fmaxf(m.y, 0.0f), m.z));
  return m;
}

}  // namespace vmd
