// Host-side material inputs of the resolve for callers without the engine's:
// a block atlas, the block face table, a probe field, the shaft envelope of a
// recipe's terrain and the frame's look parameters.  An engine passes its own
// atlas, face table, probe field and shaft pass output to vm_upload_*; these
// exist for the tests, the benchmarks and the smoke check.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "vm_types.h"
#include "recipe.h"
#include "../../include/voxmarch.h"
#include "../../include/voxmarch_world.h"

namespace {

// Face layers of every block id, in normal order -x, +x, -y, +y, -z, +z, and
// the perm class of every layer: the engine's block table
// (src/block.rs:37-131, 144-182; `column(side, bottom, top)`), kept alike
// because the face word is part of the resolve's input format.
enum : uint32_t {
  T_STONE, T_DIRT, T_GRASS_TOP, T_GRASS_SIDE, T_SAND, T_GRAVEL, T_LOG_SIDE, T_LOG_TOP, T_LEAVES, T_PLANKS, T_COBBLE,
  T_GLASS, T_GLOWSTONE, T_BEDROCK, T_WATER, T_SNOW, T_PODZOL, T_PINE_LEAVES, T_LICHEN, T_TALL_GRASS, T_MEADOW_TOP,
  T_AMBER_LAMP, T_AZURE_LAMP, T_VERDANT_LAMP, T_MEADOW_SIDE, T_GRASS_TALL, T_REEDS, T_COUNT
};
static_assert(T_COUNT == VM_TEX_COUNT, "atlas layer count");

struct Faces { uint32_t side, bottom, top; bool column; };
constexpr Faces all(uint32_t t) { return {t, t, t, false}; }
constexpr Faces column(uint32_t side, uint32_t bottom, uint32_t top) { return {side, bottom, top, true}; }
const Faces BLOCK_FACES[VM_BLOCK_COUNT] = {
    all(0), all(T_STONE), all(T_DIRT), column(T_GRASS_SIDE, T_DIRT, T_GRASS_TOP), all(T_SAND), all(T_GRAVEL),
    column(T_LOG_SIDE, T_LOG_TOP, T_LOG_TOP), all(T_LEAVES), all(T_PLANKS), all(T_COBBLE), all(T_GLASS),
    all(T_GLOWSTONE), all(T_BEDROCK), all(T_WATER), all(T_SNOW), all(T_PODZOL), all(T_PINE_LEAVES), all(T_LICHEN),
    all(T_TALL_GRASS), column(T_GRASS_SIDE, T_DIRT, T_MEADOW_TOP), all(T_AMBER_LAMP), all(T_AZURE_LAMP),
    all(T_VERDANT_LAMP), column(T_MEADOW_SIDE, T_DIRT, T_MEADOW_TOP), all(T_GRASS_TALL), all(T_REEDS)};

uint32_t perm_class(uint32_t layer) {
  switch (layer) {
    case T_DIRT: case T_GRASS_TOP: case T_SAND: case T_PODZOL: case T_LEAVES: case T_PINE_LEAVES: case T_MEADOW_TOP:
      return 2u;   // D4
    case T_MEADOW_SIDE: case T_GRASS_SIDE:
      return 1u;   // FLIP_U
    default:
      return 0u;
  }
}

uint32_t hash2(uint32_t x, uint32_t y, uint32_t s) { return vmr::mix32(x * 0x8da6b343u ^ vmr::mix32(y * 0xd8163841u ^ s)); }
float unit01(uint32_t h) { return (float)(h >> 8) * (1.0f / 16777216.0f); }

float to_linear(uint8_t u) {
  const float c = (float)u / 255.0f;
  return c <= 0.04045f ? c / 12.92f : powf((c + 0.055f) / 1.055f, 2.4f);
}
uint8_t to_srgb(float c) {
  const float s = c <= 0.0031308f ? c * 12.92f : 1.055f * powf(c, 1.0f / 2.4f) - 0.055f;
  return (uint8_t)std::min(255.0f, std::max(0.0f, s * 255.0f + 0.5f));
}

// A layer's texel (mip 0): base colour, value noise of two scales, a darker
// seam pattern for a few layers, and the alpha the resolve reads: the tint
// mask of tinted surfaces (grass tops, leaves, meadows) or the coverage of the
// cross-quad tufts.
void texel(uint32_t layer, uint32_t x, uint32_t y, uint32_t seed, uint8_t* out) {
  static const float base[T_COUNT][3] = {
      {0.50f, 0.50f, 0.50f}, {0.53f, 0.38f, 0.26f}, {0.36f, 0.62f, 0.24f}, {0.50f, 0.42f, 0.28f},
      {0.86f, 0.80f, 0.58f}, {0.48f, 0.46f, 0.44f}, {0.42f, 0.31f, 0.18f}, {0.68f, 0.55f, 0.34f},
      {0.22f, 0.48f, 0.16f}, {0.70f, 0.54f, 0.32f}, {0.52f, 0.52f, 0.52f}, {0.85f, 0.93f, 0.97f},
      {0.95f, 0.80f, 0.45f}, {0.22f, 0.22f, 0.24f}, {0.10f, 0.30f, 0.55f}, {0.92f, 0.94f, 0.98f},
      {0.40f, 0.26f, 0.14f}, {0.14f, 0.32f, 0.18f}, {0.48f, 0.52f, 0.40f}, {0.30f, 0.58f, 0.20f},
      {0.40f, 0.62f, 0.22f}, {0.95f, 0.70f, 0.35f}, {0.40f, 0.62f, 0.95f}, {0.55f, 0.92f, 0.45f},
      {0.45f, 0.55f, 0.26f}, {0.28f, 0.55f, 0.18f}, {0.46f, 0.52f, 0.24f}};
  const uint32_t s = seed * 0x9e3779b9u + layer * 0x632be5abu;
  const float fine = unit01(hash2(x, y, s));
  const float coarse = unit01(hash2(x >> 2, y >> 2, s ^ 0x5bd1e995u));
  float v = 0.72f + 0.28f * fine + 0.22f * coarse;
  if ((layer == T_PLANKS && (y & 3u) == 0u) || (layer == T_COBBLE && coarse < 0.25f) ||
      (layer == T_LOG_SIDE && (x % 5u) == 0u))
    v *= 0.7f;
  for (int c = 0; c < 3; ++c) out[c] = (uint8_t)std::min(255.0f, std::max(0.0f, base[layer][c] * v * 255.0f));
  uint8_t a = 0;
  switch (layer) {
    case T_GRASS_TOP: case T_LEAVES: case T_PINE_LEAVES: case T_MEADOW_TOP: case T_MEADOW_SIDE:
      a = 255;
      break;
    case T_GRASS_SIDE:
      a = y < 3u + (hash2(x, 0, s) & 1u) ? 255 : 0;   // the grass rim of the side face
      break;
    case T_TALL_GRASS: case T_GRASS_TALL: case T_REEDS: {
      // blades: columns of random height, thinning toward their tips
      const uint32_t top = 4u + hash2(x, 1u, s) % 10u;
      const bool blade = (hash2(x, 2u, s) & 3u) != 0u && y >= top;
      a = blade ? (uint8_t)(255.0f * std::min(1.0f, 0.4f + 0.1f * (float)(y - top))) : 0;
      break;
    }
    default:
      a = 0;
  }
  out[3] = a;
}

}  // namespace

extern "C" {

uint64_t vmw_atlas_bytes(uint32_t layers) {
  uint64_t texels = 0;
  for (uint32_t m = 0; m < VM_ATLAS_MIPS; ++m) texels += (uint64_t)layers * (VM_ATLAS_SIZE >> m) * (VM_ATLAS_SIZE >> m);
  return texels * 4;
}

int vmw_build_atlas(uint32_t seed, uint8_t* out) {
  if (!out) return VM_E_INVALID;
  const uint32_t L = VM_TEX_COUNT, S = VM_ATLAS_SIZE;
  uint8_t* level = out;
  for (uint32_t l = 0; l < L; ++l)
    for (uint32_t y = 0; y < S; ++y)
      for (uint32_t x = 0; x < S; ++x) texel(l, x, y, seed, level + ((l * S + y) * S + x) * 4);
  // each further mip: the 2x2 box average, colour averaged in linear light
  uint32_t size = S;
  for (uint32_t m = 1; m < VM_ATLAS_MIPS; ++m) {
    uint8_t* next = level + (size_t)L * size * size * 4;
    const uint32_t half = size / 2;
    for (uint32_t l = 0; l < L; ++l)
      for (uint32_t y = 0; y < half; ++y)
        for (uint32_t x = 0; x < half; ++x) {
          float acc[4] = {0, 0, 0, 0};
          for (uint32_t d = 0; d < 4; ++d) {
            const uint8_t* p = level + ((l * size + 2 * y + (d >> 1)) * size + 2 * x + (d & 1u)) * 4;
            for (int c = 0; c < 3; ++c) acc[c] += to_linear(p[c]);
            acc[3] += (float)p[3] / 255.0f;
          }
          uint8_t* q = next + ((l * half + y) * half + x) * 4;
          for (int c = 0; c < 3; ++c) q[c] = to_srgb(acc[c] * 0.25f);
          q[3] = (uint8_t)std::min(255.0f, acc[3] * 0.25f * 255.0f + 0.5f);
        }
    level = next;
    size = half;
  }
  return VM_OK;
}

int vmw_block_faces(uint32_t* out, uint32_t n) {
  if (!out || n < VM_BLOCK_COUNT * 8u) return VM_E_INVALID;
  for (uint32_t b = 0; b < VM_BLOCK_COUNT; ++b) {
    const Faces& f = BLOCK_FACES[b];
    const uint32_t layers[8] = {f.side, f.side, f.bottom, f.top, f.side, f.side, f.side, f.side};
    for (uint32_t i = 0; i < 8; ++i) out[b * 8 + i] = layers[i] | (perm_class(layers[i]) << 16);
  }
  return VM_OK;
}

int vmw_probe_field(uint32_t seed, uint16_t* out) {
  if (!out) return VM_E_INVALID;
  // values in [0.55, 1], constant over 8^3 texel cells, as binary16
  const uint64_t n = (uint64_t)VM_PROBE_NX * VM_PROBE_NY * VM_PROBE_NZ;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < (int64_t)n; ++i) {
    const uint32_t x = (uint32_t)(i % VM_PROBE_NX), y = (uint32_t)((i / VM_PROBE_NX) % VM_PROBE_NY);
    const uint32_t z = (uint32_t)(i / ((uint64_t)VM_PROBE_NX * VM_PROBE_NY));
    for (uint32_t c = 0; c < 4; ++c) {
      const float v = 0.55f + 0.45f * vmr::unit(vmr::hash3((int32_t)(x >> 3), (int32_t)(y >> 3), (int32_t)(z >> 3),
                                                           seed * 4u + c));
      // binary16 of a normal float in [0.5, 1]: rebias the exponent, keep 10 mantissa bits
      uint32_t bits;
      memcpy(&bits, &v, 4);
      const uint32_t e = ((bits >> 23) & 0xFFu) - 127u + 15u;
      out[i * 4 + c] = (uint16_t)((e << 10) | ((bits >> 13) & 0x3FFu));
    }
  }
  return VM_OK;
}

int vmw_shaft_envelope(const vmw_recipe* r, const float* sun_dir, const float* origin, float texel, float* out) {
  if (!r || !sun_dir || !origin || !out || !(texel > 0.0f)) return VM_E_INVALID;
  // the terrain's sun envelope: at each texel, the highest point of the
  // height field seen toward the sun, lowered by the sun's slope over the
  // distance (the terrain shadow line of the shaft pass); 256 texels of reach
  const uint32_t D = VM_SHAFT_DIM;
  std::vector<float> h((size_t)D * D);
#pragma omp parallel for schedule(static)
  for (int64_t z = 0; z < (int64_t)D; ++z)
    for (uint32_t x = 0; x < D; ++x) {
      const int32_t wx = (int32_t)floorf(origin[0] + ((float)x + 0.5f) * texel);
      const int32_t wz = (int32_t)floorf(origin[1] + ((float)z + 0.5f) * texel);
      const bool inside = wx >= 0 && wz >= 0 && wx < (int32_t)r->size[0] && wz < (int32_t)r->size[2];
      h[(size_t)z * D + x] = inside ? (float)vmr::column_height(*r, wx, wz) : 0.0f;
    }
  const float horiz = std::max(sqrtf(sun_dir[0] * sun_dir[0] + sun_dir[2] * sun_dir[2]), 1e-3f);
  const float dx = sun_dir[0] / horiz, dz = sun_dir[2] / horiz, slope = sun_dir[1] / horiz;
  const auto sample = [&](float x, float z) {
    const float cx = std::min(std::max(x, 0.0f), (float)(D - 1)), cz = std::min(std::max(z, 0.0f), (float)(D - 1));
    const uint32_t x0 = (uint32_t)cx, z0 = (uint32_t)cz;
    const uint32_t x1 = std::min(x0 + 1u, D - 1u), z1 = std::min(z0 + 1u, D - 1u);
    const float fx = cx - (float)x0, fz = cz - (float)z0;
    const float a = h[(size_t)z0 * D + x0] * (1 - fx) + h[(size_t)z0 * D + x1] * fx;
    const float b = h[(size_t)z1 * D + x0] * (1 - fx) + h[(size_t)z1 * D + x1] * fx;
    return a * (1 - fz) + b * fz;
  };
#pragma omp parallel for schedule(static)
  for (int64_t z = 0; z < (int64_t)D; ++z)
    for (uint32_t x = 0; x < D; ++x) {
      float best = h[(size_t)z * D + x];
      for (uint32_t m = 1; m <= 256; ++m)
        best = std::max(best, sample((float)x + dx * (float)m, (float)z + dz * (float)m) - (float)m * texel * slope);
      out[(size_t)z * D + x] = best;
    }
  return VM_OK;
}

void vmw_look_defaults(vm_frame* f, int32_t seed) {
  if (!f) return;
  // the engine's default fog, clouds, god rays, tint and shaft parameters
  // (src/render/mod.rs:504-582 defaults as the frame carries them,
  // src/config.rs:276-380, src/biome.rs:59-60, src/shaft.rs:5-9)
  f->fog_density = 5.0e-4f;
  f->fog_falloff = 1.0f / 64.0f;
  f->fog_scatter = 0.020f;
  f->fog_g = 0.80f;
  f->fog_height = f->sea_level;
  f->ambient = 0.08f;
  f->cloud_cover = 0.45f;
  f->cloud_height = 448.0f;
  f->cloud_scale = 320.0f;
  f->cloud_speed = 3.0f;
  f->godray_strength = 1.0f;
  f->godray_steps = 4;
  f->godray_dist = 4096.0f;
  f->cloud_shadow = 0.85f;
  f->tint_strength = 1.0f;
  f->tint_seed = seed;
  f->tint_freq_t = 0.00055f;
  f->tint_freq_h = 0.0007f;
  f->shaft_texel = 4.0f;
  f->shaft_soft = 4.0f;
  // the envelope window centred on the camera (src/shaft.rs:53-58, 104-109)
  const int32_t half = (int32_t)VM_SHAFT_DIM / 2;
  f->shaft_origin[0] = (float)(((int32_t)floorf(f->cam_pos[0] / 4.0f) - half) * 4);
  f->shaft_origin[1] = (float)(((int32_t)floorf(f->cam_pos[2] / 4.0f) - half) * 4);
}

}  // extern "C"
