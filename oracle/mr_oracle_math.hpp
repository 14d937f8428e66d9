// CPU oracle - TEST INFRASTRUCTURE ONLY. Nothing in the product links this.
// Math primitives restated from the reference (paths relative to the
// reference project). Compiled with -ffp-contract=off.
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>
#include <algorithm>

namespace orc {

struct V3 { float x, y, z; };
static inline V3 v3(float x, float y, float z) { return V3{x, y, z}; }
static inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
static inline V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
static inline V3 operator*(V3 a, V3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
static inline V3 operator*(V3 a, float b) { return {a.x * b, a.y * b, a.z * b}; }
static inline V3 operator/(V3 a, float b) { return {a.x / b, a.y / b, a.z / b}; }
static inline V3 operator+(V3 a, float b) { return {a.x + b, a.y + b, a.z + b}; }
static inline V3 operator-(V3 a, float b) { return {a.x - b, a.y - b, a.z - b}; }
static inline V3 operator-(V3 a) { return {-a.x, -a.y, -a.z}; }
static inline float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline V3 cross(V3 a, V3 b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
static inline V3 normalize(V3 v) { float l = std::sqrt(dot(v, v)); return {v.x / l, v.y / l, v.z / l}; }
static inline float length(V3 v) { return std::sqrt(dot(v, v)); }
static inline V3 vmin(V3 a, V3 b) { return {std::min(a.x, b.x), std::min(a.y, b.y), std::min(a.z, b.z)}; }
static inline V3 vmax(V3 a, V3 b) { return {std::max(a.x, b.x), std::max(a.y, b.y), std::max(a.z, b.z)}; }
// core/vector.cu:29 lerp(a,b,v) = a*(1-v) + b*v
static inline float lerp(float a, float b, float v) { return a * (1.0f - v) + b * v; }

// core/vector.cu:19 inv(): zero components map to 999999999.
static inline V3 inv(V3 a) {
  return {a.x == 0 ? 999999999.0f : 1 / a.x, a.y == 0 ? 999999999.0f : 1 / a.y,
          a.z == 0 ? 999999999.0f : 1 / a.z};
}
// core/vector.cu:41-58: entry distance to the box +-0.4999 (or -1 on a miss).
static inline float ray_box_offset(V3 p, V3 dir) {
  V3 d = inv(dir);
  V3 bmax = {0.4999f, 0.4999f, 0.4999f};
  V3 to_axis = (-p) * d;
  V3 to_face = bmax * d;
  V3 d0 = to_axis + to_face, d1 = to_axis - to_face;
  V3 tmin = vmin(d0, d1), tmax = vmax(d0, d1);
  float tmi = std::max(tmin.x, std::max(tmin.y, tmin.z));
  float tma = std::min(tmax.x, std::min(tmax.y, tmax.z));
  return tma >= tmi ? std::max(tmi, 0.0f) : -1.0f;
}
// core/vector.cu:60-75: exit distance from the box +-0.5.
static inline float ray_box_distance(V3 p, V3 dir) {
  V3 d = inv(dir);
  V3 bmax = {0.5f, 0.5f, 0.5f};
  V3 to_axis = (-p) * d;
  V3 to_face = bmax * d;
  V3 d0 = to_axis + to_face, d1 = to_axis - to_face;
  V3 tmax = vmax(d0, d1);
  return std::min(tmax.x, std::min(tmax.y, tmax.z));
}
// core/vector.cu:205-209 (no 1/pi: the reference's convention). x^1.5 = x*sqrt(x).
static inline float hg_phase(float c, float g) {
  float g2 = g * g;
  float d = 1.0f + g2 - 2.0f * g * c;
  return ((1.0f - g2) / (d * std::sqrt(d))) * 0.25f;
}
// core/vector.cu:211-218
static inline float hg_sample_cos(float s, float g) {
  if (std::fabs(g) < 0.0001f) return s * 2.0f - 1.0f;
  float g2 = g * g;
  float t0 = (1 - g2) / (1 - g + 2 * g * s);
  return (1 + g2 - t0 * t0) / (2 * g);
}
static const float kTwoPi = 6.28318530718f;
// core/vector.cu:220-237
static inline V3 hg_sample_dir(float e0, float e1, V3 v, float g) {
  float ct = hg_sample_cos(e0, g);
  float phi = kTwoPi * e1;
  float st = std::sqrt(std::max(0.0f, 1.0f - ct * ct));
  V3 v2 = std::fabs(v.z) > 0.70710678f ? normalize(cross(v, v3(0, 1, 0)))
                                       : normalize(cross(v, v3(0, 0, 1)));
  V3 v3_ = cross(v2, v);
  return (v3_ * (st * std::cos(phi))) + (v2 * (st * std::sin(phi))) + (v * ct);
}
// core/vector.cu:190-203
static inline V3 uniform_sphere(float ex, float ey) {
  float phi = kTwoPi * ex;
  float ct = 1 - 2 * ey;
  float st = std::sqrt(1 - ct * ct);
  return {st * std::cos(phi), st * std::sin(phi), ct};
}

// ---- Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11) ----------------------
static inline void philox4x32_10(const uint32_t ctr_in[4], uint32_t k0, uint32_t k1,
                                 uint32_t out[4]) {
  uint32_t x0 = ctr_in[0], x1 = ctr_in[1], x2 = ctr_in[2], x3 = ctr_in[3];
  for (int r = 0; r < 10; ++r) {
    if (r) { k0 += 0x9E3779B9u; k1 += 0xBB67AE85u; }
    uint64_t p0 = (uint64_t)0xD2511F53u * x0;
    uint64_t p1 = (uint64_t)0xCD9E8D57u * x2;
    uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    uint32_t y0 = hi1 ^ x1 ^ k0, y2 = hi0 ^ x3 ^ k1;
    x0 = y0; x1 = lo1; x2 = y2; x3 = lo0;
  }
  out[0] = x0; out[1] = x1; out[2] = x2; out[3] = x3;
}
// Uniform in [2^-24, 1-2^-24]: ((x>>9) + 0.5) * 2^-23, exact in fp32.
static inline float u01(uint32_t x) { return ((float)(x >> 9) + 0.5f) * 1.1920928955078125e-7f; }

// Stream tags (word 3 of the counter).
enum { TAG_PT = 1, TAG_NN = 2, TAG_LUT = 3, TAG_GEN = 4, TAG_LABEL = 5, TAG_MISC = 6, TAG_ENV = 7 };

// One path's random stream: key (seed, 0), counter (a, b, block, tag);
// draw k is word k%4 of block k/4.
struct Rng {
  uint32_t ctr[4];
  uint32_t key;
  uint32_t buf[4];
  int used;
  Rng(uint32_t seed, uint32_t a, uint32_t b, uint32_t tag) {
    ctr[0] = a; ctr[1] = b; ctr[2] = 0; ctr[3] = tag; key = seed; used = 4;
  }
  float next() {
    if (used == 4) { philox4x32_10(ctr, key, 0u, buf); ctr[2]++; used = 0; }
    return u01(buf[used++]);
  }
};

// ---- 192-point stencil layout (core/vector.cu:299-400) ----------------------
struct StencilInfo { float offset; int mip; int type; int localindex; };
static inline StencilInfo stencil_info(int i) {
  const float ms = 0.6f;  // MsOffsetScale
  if (i < 8) return {1.0f / 256.0f * lerp(ms, 1.0f, 1.0f), 0, 5, i};
  if (i < 16) return {2.5f / 256.0f * lerp(ms, 1.0f, 0.8f), 1, 5, 8};
  if (i < 32) return {5.5f / 256.0f * lerp(ms, 1.0f, 0.6f), 2, 5, 8};
  if (i < 48) return {11.5f / 256.0f * lerp(ms, 1.0f, 0.4f), 3, 5, 8};
  if (i < 64) return {23.5f / 256.0f * lerp(ms, 1.0f, 0.2f), 4, 5, 8};
  if (i < 96) return {47.5f / 256.0f * ms, 5, 5, 8};
  if (i < 128) return {95.5f / 256.0f * ms, 6, 5, 8};
  if (i < 160) return {191.5f / 256.0f * ms, 7, 5, 8};
  if (i < 168) return {(float)(i - 160 + 1) / 256.0f, 0, 1, 8};
  if (i < 176) return {(8.5f + 1.0f + 2.0f * (float)(i - 168)) / 256.0f, 1, 1, 8};
  if (i < 184) return {(26.5f + 4.0f * (float)(i - 176)) / 256.0f, 2, 1, 8};
  if (i < 192) return {(60.5f + 8.0f * (float)(i - 184)) / 256.0f, 3, 1, 8};
  return {0.0f, 0, 1, 8};
}

}  // namespace orc
