// ORACLE — test infrastructure only.
//
// The engine's block atlas restated in C++: build_atlas, texel and
// downsample of src/textures.rs:9-351 and the mip chain make_atlas uploads
// (src/render/mod.rs:2159-2210): 27 layers of 16x16 Rgba8UnormSrgb texels,
// mips 16, 8, 4, 2.  The tests feed it to the resolve and to the tuft cross
// quads as the engine's own atlas, beside the library's procedural one.
// Unpinned: the engine has no golden atlas bytes, and its Rust cannot run
// here; the restatement follows the source's arithmetic (f32, libm sinf /
// powf / sqrtf, `as u8` truncating and saturating).

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace {

enum : uint32_t {
  STONE, DIRT, GRASS_TOP, GRASS_SIDE, SAND, GRAVEL, LOG_SIDE, LOG_TOP, LEAVES, PLANKS, COBBLE, GLASS, GLOWSTONE,
  BEDROCK, WATER, SNOW, PODZOL, PINE_LEAVES, LICHEN, TALL_GRASS, MEADOW_TOP, AMBER_LAMP, AZURE_LAMP, VERDANT_LAMP,
  MEADOW_SIDE, GRASS_TALL, REEDS, COUNT
};
constexpr uint32_t SIZE = 16;

struct Px { uint8_t c[4]; };

// `(v as f32) as u8`: truncation toward zero, saturating at 0 and 255
uint8_t as_u8(float v) {
  if (!(v > 0.0f)) return 0;
  if (v >= 255.0f) return 255;
  return (uint8_t)v;
}

float hash(uint32_t x, uint32_t y, uint32_t seed) {   // src/textures.rs:9-16
  uint32_t h = (x * 0x8da6b343u) ^ (y * 0xd8163841u) ^ (seed * 0xcb1ab31fu);
  h ^= h >> 13;
  h *= 0x5bd1e995u;
  h ^= h >> 15;
  return (float)(h & 0xFFFFu) / 65535.0f;
}

Px px(const float* c, float v) {   // src/textures.rs:18-21
  Px p;
  for (int i = 0; i < 3; ++i) p.c[i] = as_u8(std::min(std::max(c[i] * v, 0.0f), 1.0f) * 255.0f);
  p.c[3] = 0;
  return p;
}
Px pxt(const float* c, float v) {
  Px p = px(c, v);
  p.c[3] = 255;
  return p;
}
Px px3(float r, float g, float b, float v) { const float c[3] = {r, g, b}; return px(c, v); }
Px pxt3(float r, float g, float b, float v) { const float c[3] = {r, g, b}; return pxt(c, v); }

const float GRASS[3] = {0.36f, 0.62f, 0.24f};
constexpr float MEADOW_SHADE = 0.59f;

float blob(uint32_t x, uint32_t y, uint32_t seed) {   // src/textures.rs:33-41
  const int32_t d[5][2] = {{0, 0}, {1, 0}, {0, 1}, {-1, 0}, {0, -1}};
  float acc = 0.0f;
  for (const auto& o : d) {
    const uint32_t xx = (uint32_t)((((int32_t)x + o[0]) % 16 + 16) % 16);
    const uint32_t yy = (uint32_t)((((int32_t)y + o[1]) % 16 + 16) % 16);
    acc += hash(xx / 2, yy / 2, seed);
  }
  return acc / 5.0f;
}

Px lamp(uint32_t x, uint32_t y, float n, uint32_t seed, const float* core, const float* body) {
  if (blob(x, y, seed) > 0.55f) return px(core, 1.0f);
  return px(body, 0.85f + 0.2f * n);
}

struct Blade { float root, tip, h; };

// a tuft layer: blades bending from root to tip (quadratic, or straight
// stalks), half width shrinking toward the tip
Px tuft(uint32_t x, uint32_t y, float n, const Blade* blades, int count, float w0, float w1, bool straight,
        const float* base, const float* grow, float shade) {
  const float fx = (float)x + 0.5f;
  const float ry = (float)(SIZE - 1 - y);
  float tip_frac = -1.0f;
  for (int i = 0; i < count; ++i) {
    const Blade& b = blades[i];
    if (ry > b.h) continue;
    const float s = ry / b.h;
    const float cx = straight ? b.root + (b.tip - b.root) * s : b.root + (b.tip - b.root) * s * s;
    const float half = w0 - w1 * s;
    if (fabsf(fx - cx) <= half) tip_frac = std::max(tip_frac, s);
  }
  if (tip_frac < 0.0f) return Px{{0, 0, 0, 0}};
  const float c[3] = {base[0] + grow[0] * tip_frac, base[1] + grow[1] * tip_frac, base[2] + grow[2] * tip_frac};
  Px p = px(c, shade + 0.3f * n);
  p.c[3] = 255;
  return p;
}

// texel: src/textures.rs:51-290
Px texel(uint32_t layer, uint32_t x, uint32_t y, float water_mottle, bool tint_balance) {
  const float n = hash(x, y, layer * 31u + 7u);
  switch (layer) {
    case STONE: return px3(0.50f, 0.50f, 0.50f, 0.78f + 0.28f * blob(x, y, 1));
    case DIRT: return px3(0.53f, 0.38f, 0.26f, 0.75f + 0.35f * n);
    case GRASS_TOP: return pxt(GRASS, 0.78f + 0.32f * n);
    case GRASS_SIDE: {
      const uint32_t edge = 3u + (uint32_t)(hash(x, 0, 99) * 2.5f);
      if (y < edge) return pxt(GRASS, 0.78f + 0.32f * n);
      return px3(0.53f, 0.38f, 0.26f, 0.75f + 0.35f * n);
    }
    case SAND: {
      Px p = px3(0.86f, 0.80f, 0.58f, 0.86f + 0.16f * n);
      if (tint_balance) return pxt3(p.c[0] / 255.0f, p.c[1] / 255.0f, p.c[2] / 255.0f, 1.0f);
      return p;
    }
    case GRAVEL: return px3(0.48f, 0.46f, 0.44f, 0.65f + 0.5f * blob(x, y, 5));
    case LOG_SIDE: {
      const float stripe = 0.8f + 0.2f * (sinf((float)x * 1.7f) * 0.5f + 0.5f) + 0.1f * n;
      return px3(0.42f, 0.31f, 0.18f, stripe);
    }
    case LOG_TOP: {
      const float cx = (float)x - 7.5f, cy = (float)y - 7.5f;
      const float r = sqrtf(cx * cx + cy * cy);
      const float ring = 0.75f + 0.25f * (sinf(r * 1.9f) * 0.5f + 0.5f) + 0.05f * n;
      if (r > 7.2f) return px3(0.42f, 0.31f, 0.18f, 0.9f);
      return px3(0.72f, 0.58f, 0.36f, ring);
    }
    case LEAVES:
      if (hash(x, y, 4) < 0.35f) return pxt3(0.16f, 0.36f, 0.12f, 0.9f + 0.2f * n);
      return pxt3(0.24f, 0.52f, 0.18f, 0.85f + 0.3f * n);
    case PLANKS: {
      const uint32_t plank = (y / 4) % 2;
      const bool seam = y % 4 == 0 || x == (plank * 8 + 3) % 16;
      if (seam) return px3(0.55f, 0.42f, 0.25f, 0.6f);
      return px3(0.72f, 0.56f, 0.33f, 0.88f + 0.2f * n);
    }
    case COBBLE: {
      const float b = blob(x, y, 9);
      if (b < 0.36f) return px3(0.30f, 0.30f, 0.30f, 0.9f);
      return px3(0.56f, 0.56f, 0.56f, 0.75f + 0.35f * b);
    }
    case GLASS: {
      const bool border = x == 0 || y == 0 || x == 15 || y == 15;
      const bool streak = (x + y) % 9 == 0;
      if (border) return px3(0.80f, 0.90f, 0.95f, 0.9f);
      if (streak) return px3(0.90f, 0.96f, 1.0f, 0.95f);
      return px3(0.70f, 0.85f, 0.92f, 0.95f);
    }
    case GLOWSTONE: {
      const float core[3] = {1.0f, 0.95f, 0.65f}, body[3] = {0.80f, 0.62f, 0.30f};
      return lamp(x, y, n, 13, core, body);
    }
    case BEDROCK: return px3(0.30f, 0.30f, 0.32f, 0.5f + 0.9f * blob(x, y, 21));
    case WATER: return px3(0.10f, 0.34f, 0.42f, (1.0f - 0.5f * water_mottle) + water_mottle * blob(x, y, 33));
    case SNOW: return px3(0.88f, 0.91f, 0.97f, 0.94f + 0.10f * blob(x, y, 41));
    case PODZOL: return px3(0.34f, 0.23f, 0.13f, 0.78f + 0.34f * n);
    case PINE_LEAVES:
      if (hash(x, y, 6) < 0.40f) return pxt3(0.09f, 0.24f, 0.17f, 0.9f + 0.2f * n);
      return pxt3(0.15f, 0.36f, 0.24f, 0.85f + 0.3f * n);
    case LICHEN: {
      if (hash(x, y, 8) < 0.30f) return px3(0.47f, 0.47f, 0.44f, 0.82f + 0.3f * n);
      Px p = px3(0.45f, 0.50f, 0.38f, 0.80f + 0.32f * blob(x, y, 17));
      if (tint_balance) return pxt3(p.c[0] / 255.0f, p.c[1] / 255.0f, p.c[2] / 255.0f, 1.0f);
      return p;
    }
    case TALL_GRASS: {
      static const Blade b[6] = {{1.5f, 0.4f, 12.0f}, {4.0f, 5.2f, 15.0f}, {6.5f, 5.8f, 9.0f},
                                 {8.5f, 9.9f, 14.0f}, {11.0f, 10.2f, 11.0f}, {13.5f, 14.6f, 13.0f}};
      const float base[3] = {0.13f, 0.30f, 0.10f}, grow[3] = {0.12f, 0.30f, 0.06f};
      return tuft(x, y, n, b, 6, 1.15f, 0.85f, false, base, grow, 0.85f);
    }
    case MEADOW_TOP: return pxt(GRASS, (0.78f + 0.32f * n) * MEADOW_SHADE);
    case MEADOW_SIDE: {
      const uint32_t edge = 3u + (uint32_t)(hash(x, 0, 99) * 2.5f);
      if (y < edge) return pxt(GRASS, (0.78f + 0.32f * n) * MEADOW_SHADE);
      return px3(0.53f, 0.38f, 0.26f, (0.75f + 0.35f * n) * MEADOW_SHADE);
    }
    case GRASS_TALL: {
      static const Blade b[7] = {{1.0f, 0.2f, 15.0f}, {3.0f, 4.4f, 16.0f}, {5.5f, 4.9f, 13.0f}, {7.5f, 8.6f, 15.0f},
                                 {9.5f, 8.9f, 14.0f}, {11.5f, 12.8f, 16.0f}, {14.0f, 13.2f, 14.0f}};
      const float base[3] = {0.14f, 0.33f, 0.09f}, grow[3] = {0.30f, 0.26f, 0.07f};
      return tuft(x, y, n, b, 7, 1.2f, 0.8f, false, base, grow, 0.82f);
    }
    case REEDS: {
      static const Blade b[5] = {{2.0f, 2.7f, 16.0f}, {5.0f, 4.6f, 15.0f}, {7.8f, 8.4f, 16.0f},
                                 {10.6f, 10.1f, 14.0f}, {13.6f, 14.1f, 16.0f}};
      const float base[3] = {0.20f, 0.28f, 0.10f}, grow[3] = {0.16f, 0.16f, 0.06f};
      return tuft(x, y, n, b, 5, 0.85f, 0.25f, true, base, grow, 0.80f);
    }
    case AMBER_LAMP: {
      const float core[3] = {1.0f, 0.78f, 0.42f}, body[3] = {0.74f, 0.34f, 0.10f};
      return lamp(x, y, n, 41, core, body);
    }
    case AZURE_LAMP: {
      const float core[3] = {0.68f, 0.88f, 1.0f}, body[3] = {0.14f, 0.34f, 0.80f};
      return lamp(x, y, n, 43, core, body);
    }
    case VERDANT_LAMP: {
      const float core[3] = {0.74f, 1.0f, 0.58f}, body[3] = {0.18f, 0.62f, 0.20f};
      return lamp(x, y, n, 47, core, body);
    }
    default: return Px{{255, 0, 255, 0}};
  }
}

float srgb_to_linear(uint8_t u) {   // src/textures.rs:304-311
  const float c = (float)u / 255.0f;
  return c <= 0.04045f ? c / 12.92f : powf((c + 0.055f) / 1.055f, 2.4f);
}
uint8_t linear_to_srgb(float c) {   // src/textures.rs:313-320
  const float s = c <= 0.0031308f ? c * 12.92f : 1.055f * powf(c, 1.0f / 2.4f) - 0.055f;
  return as_u8(std::min(std::max(s, 0.0f), 1.0f) * 255.0f + 0.5f);
}

}  // namespace

extern "C" {

// The atlas as make_atlas uploads it: mip 0 of every layer ([layer][y][x]
// RGBA), then mips 8, 4, 2, each the downsample of the one before
// (src/textures.rs:322-350).  out: 27 * 340 * 4 bytes.
void or_build_atlas(float water_mottle, int tint_balance, uint8_t* out) {
  uint8_t* level = out;
  for (uint32_t l = 0; l < COUNT; ++l)
    for (uint32_t y = 0; y < SIZE; ++y)
      for (uint32_t x = 0; x < SIZE; ++x) {
        const Px p = texel(l, x, y, water_mottle, tint_balance != 0);
        memcpy(level + ((l * SIZE + y) * SIZE + x) * 4, p.c, 4);
      }
  uint32_t size = SIZE;
  for (uint32_t mip = 1; mip < 4; ++mip) {
    uint8_t* next = level + (size_t)COUNT * size * size * 4;
    const uint32_t half = size / 2;
    for (uint32_t l = 0; l < COUNT; ++l)
      for (uint32_t y = 0; y < half; ++y)
        for (uint32_t x = 0; x < half; ++x) {
          uint8_t* o = next + ((l * half + y) * half + x) * 4;
          for (int c = 0; c < 4; ++c) {
            float acc = 0.0f;
            const uint32_t d[4][2] = {{0, 0}, {1, 0}, {0, 1}, {1, 1}};
            for (const auto& e : d) {
              const uint8_t v = level[((l * size + y * 2 + e[1]) * size + x * 2 + e[0]) * 4 + c];
              acc += c == 3 ? (float)v / 255.0f : srgb_to_linear(v);
            }
            acc = acc / 4.0f;
            o[c] = c == 3 ? as_u8(std::min(std::max(acc, 0.0f), 1.0f) * 255.0f + 0.5f) : linear_to_srgb(acc);
          }
        }
    level = next;
    size = half;
  }
}

}  // extern "C"
