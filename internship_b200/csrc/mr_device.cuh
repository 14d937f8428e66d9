// Device-side primitives of the MRPNN B200 renderer: vector math, the
// reference's ray-box / Henyey-Greenstein conventions, Philox4x32-10 streams
// and fp32 trilinear samplers over raw HBM grids.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace mr {

struct F3 { float x, y, z; };
__host__ __device__ __forceinline__ F3 f3(float x, float y, float z) { return F3{x, y, z}; }
__host__ __device__ __forceinline__ F3 operator+(F3 a, F3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__host__ __device__ __forceinline__ F3 operator-(F3 a, F3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__host__ __device__ __forceinline__ F3 operator*(F3 a, F3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
__host__ __device__ __forceinline__ F3 operator*(F3 a, float b) { return {a.x * b, a.y * b, a.z * b}; }
__host__ __device__ __forceinline__ F3 operator/(F3 a, float b) { return {a.x / b, a.y / b, a.z / b}; }
__host__ __device__ __forceinline__ F3 operator+(F3 a, float b) { return {a.x + b, a.y + b, a.z + b}; }
__host__ __device__ __forceinline__ F3 operator-(F3 a, float b) { return {a.x - b, a.y - b, a.z - b}; }
__host__ __device__ __forceinline__ F3 operator-(F3 a) { return {-a.x, -a.y, -a.z}; }
__host__ __device__ __forceinline__ float dot(F3 a, F3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__host__ __device__ __forceinline__ F3 cross(F3 a, F3 b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__host__ __device__ __forceinline__ F3 normalize(F3 v) {
  float l = sqrtf(dot(v, v));
  return {v.x / l, v.y / l, v.z / l};
}
__host__ __device__ __forceinline__ float length(F3 v) { return sqrtf(dot(v, v)); }
__host__ __device__ __forceinline__ F3 vmin(F3 a, F3 b) { return {fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z)}; }
__host__ __device__ __forceinline__ F3 vmax(F3 a, F3 b) { return {fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z)}; }
__host__ __device__ __forceinline__ float lerpf(float a, float b, float v) { return a * (1.0f - v) + b * v; }

// Reciprocal with the reference's zero convention (core/vector.cu:19).
__host__ __device__ __forceinline__ F3 inv3(F3 a) {
  return {a.x == 0 ? 999999999.0f : 1 / a.x, a.y == 0 ? 999999999.0f : 1 / a.y,
          a.z == 0 ? 999999999.0f : 1 / a.z};
}
// Entry distance into the box +-0.4999, -1 on a miss (core/vector.cu:41-58).
__host__ __device__ __forceinline__ float ray_box_offset(F3 p, F3 dir) {
  F3 d = inv3(dir);
  F3 to_axis = (-p) * d;
  F3 to_face = f3(0.4999f, 0.4999f, 0.4999f) * d;
  F3 d0 = to_axis + to_face, d1 = to_axis - to_face;
  F3 tmin = vmin(d0, d1), tmax = vmax(d0, d1);
  float tmi = fmaxf(tmin.x, fmaxf(tmin.y, tmin.z));
  float tma = fminf(tmax.x, fminf(tmax.y, tmax.z));
  return tma >= tmi ? fmaxf(tmi, 0.0f) : -1.0f;
}
// Exit distance from the box +-0.5 (core/vector.cu:60-75).
__host__ __device__ __forceinline__ float ray_box_distance(F3 p, F3 dir) {
  F3 d = inv3(dir);
  F3 to_axis = (-p) * d;
  F3 to_face = f3(0.5f, 0.5f, 0.5f) * d;
  F3 d0 = to_axis + to_face, d1 = to_axis - to_face;
  F3 tmax = vmax(d0, d1);
  return fminf(tmax.x, fminf(tmax.y, tmax.z));
}
// HG phase without 1/pi (the reference's convention, core/vector.cu:205-209).
__host__ __device__ __forceinline__ float hg_phase(float c, float g) {
  float g2 = g * g;
  float d = 1.0f + g2 - 2.0f * g * c;
  return ((1.0f - g2) / (d * sqrtf(d))) * 0.25f;
}
__host__ __device__ __forceinline__ float hg_sample_cos(float s, float g) {
  if (fabsf(g) < 0.0001f) return s * 2.0f - 1.0f;
  float g2 = g * g;
  float t0 = (1 - g2) / (1 - g + 2 * g * s);
  return (1 + g2 - t0 * t0) / (2 * g);
}
constexpr float kTwoPi = 6.28318530718f;
// HG-distributed direction around v (core/vector.cu:220-237).
__host__ __device__ __forceinline__ F3 hg_sample_dir(float e0, float e1, F3 v, float g) {
  float ct = hg_sample_cos(e0, g);
  float phi = kTwoPi * e1;
  float st = sqrtf(fmaxf(0.0f, 1.0f - ct * ct));
  F3 v2 = fabsf(v.z) > 0.70710678f ? normalize(cross(v, f3(0, 1, 0))) : normalize(cross(v, f3(0, 0, 1)));
  F3 w = cross(v2, v);
  float sp, cp;
  sincosf(phi, &sp, &cp);
  return (w * (st * cp)) + (v2 * (st * sp)) + (v * ct);
}
__host__ __device__ __forceinline__ F3 uniform_sphere(float ex, float ey) {
  float phi = kTwoPi * ex;
  float ct = 1 - 2 * ey;
  float st = sqrtf(1 - ct * ct);
  float sp, cp;
  sincosf(phi, &sp, &cp);
  return {st * cp, st * sp, ct};
}

// srp = scatterrate^4 per channel (core/radiancePredict.cu:388).
__host__ __device__ __forceinline__ F3 srp_of(F3 sr) {
  return f3((sr.x * sr.x) * (sr.x * sr.x), (sr.y * sr.y) * (sr.y * sr.y), (sr.z * sr.z) * (sr.z * sr.z));
}

// ---- Philox4x32-10 (Salmon et al., SC'11) -------------------------------------
__host__ __device__ __forceinline__ void philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                                                       uint32_t k0, uint32_t k1, uint32_t out[4]) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    if (r) { k0 += 0x9E3779B9u; k1 += 0xBB67AE85u; }
#ifdef __CUDA_ARCH__
    uint32_t hi0 = __umulhi(0xD2511F53u, c0), lo0 = 0xD2511F53u * c0;
    uint32_t hi1 = __umulhi(0xCD9E8D57u, c2), lo1 = 0xCD9E8D57u * c2;
#else
    uint64_t p0 = (uint64_t)0xD2511F53u * c0, p1 = (uint64_t)0xCD9E8D57u * c2;
    uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
#endif
    uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
    c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
  }
  out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}
// Uniform in [2^-24, 1-2^-24], exact in fp32.
__host__ __device__ __forceinline__ float u01(uint32_t x) {
  return ((float)(x >> 9) + 0.5f) * 1.1920928955078125e-7f;
}

enum StreamTag : uint32_t { TAG_PT = 1, TAG_NN = 2, TAG_LUT = 3, TAG_GEN = 4, TAG_LABEL = 5, TAG_MISC = 6, TAG_ENV = 7 };

// A path's random stream: key (seed, 0), counter (a, b, block, tag); draw k is
// word k%4 of block k/4. Four draws per Philox call, kept in registers.
struct Rng {
  uint32_t a, b, blk, tag, key;
  uint32_t w0, w1, w2, w3;
  int left;
  __device__ __forceinline__ void init(uint32_t seed, uint32_t a_, uint32_t b_, uint32_t tag_) {
    a = a_; b = b_; blk = 0; tag = tag_; key = seed; left = 0;
  }
  __device__ __forceinline__ float next() {
    if (left == 0) {
      uint32_t o[4];
      philox4x32_10(a, b, blk, tag, key, 0u, o);
      w0 = o[0]; w1 = o[1]; w2 = o[2]; w3 = o[3];
      ++blk;
      left = 4;
    }
    uint32_t x = w0;
    w0 = w1; w1 = w2; w2 = w3;
    --left;
    return u01(x);
  }
};

// ---- samplers over raw grids (index (x*res+y)*res+z) --------------------------
// Trilinear, zero outside (cudaAddressModeBorder + linear filter semantics in
// fp32, core/volume.cu:675-703).
__device__ __forceinline__ float tri_border(const float* __restrict__ d, int res, F3 uv) {
  float px = uv.x * res - 0.5f, py = uv.y * res - 0.5f, pz = uv.z * res - 0.5f;
  float fx = floorf(px), fy = floorf(py), fz = floorf(pz);
  int x = (int)fx, y = (int)fy, z = (int)fz;
  float wx = px - fx, wy = py - fy, wz = pz - fz;
  bool x0 = (unsigned)x < (unsigned)res, x1 = (unsigned)(x + 1) < (unsigned)res;
  bool y0 = (unsigned)y < (unsigned)res, y1 = (unsigned)(y + 1) < (unsigned)res;
  bool z0 = (unsigned)z < (unsigned)res, z1 = (unsigned)(z + 1) < (unsigned)res;
  size_t r = (size_t)res;
  size_t bx0 = (size_t)x * r * r, bx1 = bx0 + r * r;
  size_t by0 = (size_t)y * r, by1 = by0 + r;
  float c000 = (x0 && y0 && z0) ? __ldg(d + bx0 + by0 + z) : 0.0f;
  float c001 = (x0 && y0 && z1) ? __ldg(d + bx0 + by0 + z + 1) : 0.0f;
  float c010 = (x0 && y1 && z0) ? __ldg(d + bx0 + by1 + z) : 0.0f;
  float c011 = (x0 && y1 && z1) ? __ldg(d + bx0 + by1 + z + 1) : 0.0f;
  float c100 = (x1 && y0 && z0) ? __ldg(d + bx1 + by0 + z) : 0.0f;
  float c101 = (x1 && y0 && z1) ? __ldg(d + bx1 + by0 + z + 1) : 0.0f;
  float c110 = (x1 && y1 && z0) ? __ldg(d + bx1 + by1 + z) : 0.0f;
  float c111 = (x1 && y1 && z1) ? __ldg(d + bx1 + by1 + z + 1) : 0.0f;
  return lerpf(lerpf(lerpf(c000, c001, wz), lerpf(c010, c011, wz), wy),
               lerpf(lerpf(c100, c101, wz), lerpf(c110, c111, wz), wy), wx);
}
// The four texels of the 2 x 2 footprint whose first texel is (i, j) (layer
// `layer` of a layered texture), unfiltered: with unnormalised coordinates
// (i + 1, j + 1) the footprint is texels i, i+1 and j, j+1 exactly, and the
// address mode supplies out-of-range texels. tld4 returns them in the order
// (i, j+1), (i+1, j+1), (i+1, j), (i, j); the result is reordered to
// {(i, j), (i+1, j), (i, j+1), (i+1, j+1)}.
__device__ __forceinline__ float4 gather_a2d(cudaTextureObject_t t, int layer, float fi, float fj) {
  float a, b, c, d;
  asm("tld4.r.a2d.v4.f32.f32 {%0, %1, %2, %3}, [%4, {%5, %6, %7, %8}];"
      : "=f"(a), "=f"(b), "=f"(c), "=f"(d)
      : "l"(t), "r"(layer), "f"(fi + 1.0f), "f"(fj + 1.0f), "f"(0.0f));
  return make_float4(d, c, a, b);
}
__device__ __forceinline__ float4 gather_2d(cudaTextureObject_t t, float fi, float fj) {
  float a, b, c, d;
  asm("tld4.r.2d.v4.f32.f32 {%0, %1, %2, %3}, [%4, {%5, %6}];"
      : "=f"(a), "=f"(b), "=f"(c), "=f"(d)
      : "l"(t), "f"(fi + 1.0f), "f"(fj + 1.0f));
  return make_float4(d, c, a, b);
}

// tri_border over a layered copy of the grid (layer x, texel (z, y), border
// address mode), through two texture gathers: the same corner values (except
// subnormal ones, which the texture unit reads as 0) and the same arithmetic.
__device__ __forceinline__ float tri_border_tex(cudaTextureObject_t t, int res, F3 uv) {
  float px = uv.x * res - 0.5f, py = uv.y * res - 0.5f, pz = uv.z * res - 0.5f;
  float fx = floorf(px), fy = floorf(py), fz = floorf(pz);
  int x = (int)fx;
  float wx = px - fx, wy = py - fy, wz = pz - fz;
  const float4 z4 = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  const float4 a = (unsigned)x < (unsigned)res ? gather_a2d(t, x, fz, fy) : z4;
  const float4 b = (unsigned)(x + 1) < (unsigned)res ? gather_a2d(t, x + 1, fz, fy) : z4;
  return lerpf(lerpf(lerpf(a.x, a.y, wz), lerpf(a.z, a.w, wz), wy),
               lerpf(lerpf(b.x, b.y, wz), lerpf(b.z, b.w, wz), wy), wx);
}
// Trilinear, clamp to edge (the TR tables, core/volume.cu:1412-1417).
__device__ __forceinline__ float tri_clamp(const float* __restrict__ d, int res, F3 uv) {
  float px = uv.x * res - 0.5f, py = uv.y * res - 0.5f, pz = uv.z * res - 0.5f;
  float fx = floorf(px), fy = floorf(py), fz = floorf(pz);
  int x = (int)fx, y = (int)fy, z = (int)fz;
  float wx = px - fx, wy = py - fy, wz = pz - fz;
  int m = res - 1;
  int xa = min(max(x, 0), m), xb = min(max(x + 1, 0), m);
  int ya = min(max(y, 0), m), yb = min(max(y + 1, 0), m);
  int za = min(max(z, 0), m), zb = min(max(z + 1, 0), m);
  size_t r = (size_t)res;
  size_t bxa = (size_t)xa * r * r, bxb = (size_t)xb * r * r, bya = (size_t)ya * r, byb = (size_t)yb * r;
  float c000 = __ldg(d + bxa + bya + za), c001 = __ldg(d + bxa + bya + zb);
  float c010 = __ldg(d + bxa + byb + za), c011 = __ldg(d + bxa + byb + zb);
  float c100 = __ldg(d + bxb + bya + za), c101 = __ldg(d + bxb + bya + zb);
  float c110 = __ldg(d + bxb + byb + za), c111 = __ldg(d + bxb + byb + zb);
  return lerpf(lerpf(lerpf(c000, c001, wz), lerpf(c010, c011, wz), wy),
               lerpf(lerpf(c100, c101, wz), lerpf(c110, c111, wz), wy), wx);
}
// 2-D bilinear with clamp addressing over lut[i + j*w].
__device__ __forceinline__ float bilinear_clamp(const float* __restrict__ d, int w, int h, float u, float v) {
  float px = u * w - 0.5f, py = v * h - 0.5f;
  float fx = floorf(px), fy = floorf(py);
  int x = (int)fx, y = (int)fy;
  float wx = px - fx, wy = py - fy;
  int x0 = min(max(x, 0), w - 1), x1 = min(max(x + 1, 0), w - 1);
  int y0 = min(max(y, 0), h - 1), y1 = min(max(y + 1, 0), h - 1);
  float a = lerpf(__ldg(d + x0 + y0 * w), __ldg(d + x1 + y0 * w), wx);
  float b = lerpf(__ldg(d + x0 + y1 * w), __ldg(d + x1 + y1 * w), wx);
  return lerpf(a, b, wy);
}

// ---- 192-point descriptor stencil layout (core/vector.cu:299-400) -------------
struct StencilInfo { float offset; int mip; int type; int localindex; };
__host__ __device__ __forceinline__ StencilInfo stencil_info(int i) {
  const float ms = 0.6f;
  if (i < 8) return {1.0f / 256.0f * lerpf(ms, 1.0f, 1.0f), 0, 5, i};
  if (i < 16) return {2.5f / 256.0f * lerpf(ms, 1.0f, 0.8f), 1, 5, 8};
  if (i < 32) return {5.5f / 256.0f * lerpf(ms, 1.0f, 0.6f), 2, 5, 8};
  if (i < 48) return {11.5f / 256.0f * lerpf(ms, 1.0f, 0.4f), 3, 5, 8};
  if (i < 64) return {23.5f / 256.0f * lerpf(ms, 1.0f, 0.2f), 4, 5, 8};
  if (i < 96) return {47.5f / 256.0f * ms, 5, 5, 8};
  if (i < 128) return {95.5f / 256.0f * ms, 6, 5, 8};
  if (i < 160) return {191.5f / 256.0f * ms, 7, 5, 8};
  if (i < 168) return {(float)(i - 160 + 1) / 256.0f, 0, 1, 8};
  if (i < 176) return {(8.5f + 1.0f + 2.0f * (float)(i - 168)) / 256.0f, 1, 1, 8};
  if (i < 184) return {(26.5f + 4.0f * (float)(i - 176)) / 256.0f, 2, 1, 8};
  if (i < 192) return {(60.5f + 8.0f * (float)(i - 184)) / 256.0f, 3, 1, 8};
  return {0.0f, 0, 1, 8};
}

// Offsets of the concatenated pyramid levels.
__host__ __device__ __forceinline__ size_t mip_offset(int k) {
  size_t o = 0;
  for (int j = 0; j < k; ++j) { size_t r = 256 >> j; o += r * r * r; }
  return o;
}
__host__ __device__ __forceinline__ size_t tr_offset(int k) {
  size_t o = 0;
  for (int j = 0; j < k; ++j) { size_t r = 128 >> j; o += r * r * r; }
  return o;
}
constexpr size_t kMipTotal = 16777216 + 2097152 + 262144 + 32768 + 4096 + 512 + 64 + 8 + 1;
constexpr size_t kTrTotal = 2097152 + 262144 + 32768 + 4096 + 512 + 64 + 8 + 1;
constexpr int kLut = 512;

}  // namespace mr
