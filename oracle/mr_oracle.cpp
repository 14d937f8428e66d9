// CPU oracle for the MRPNN cloud-rendering path - TEST INFRASTRUCTURE ONLY.
//
// A plain C++17 restatement of the reference's algorithm (citations are
// paths relative to the reference project). Only the tests, the smoke check
// and the CPU-baseline leg of bench.py load this library; the product never
// does. The random-number source is Philox4x32-10 with the stream layout the
// CUDA kernels use, so oracle and kernels follow the same paths.
#include "mr_oracle_math.hpp"

#include <omp.h>

#include <atomic>
#include <cstring>
#include <vector>

#include "../include/mrpnn_b200.h"
#include "../include/mrpnn_weights.h"

using namespace orc;

namespace {

// ---- samplers -------------------------------------------------------------
// core/volume.cu:675-703 trilinear with zero border; normalized coordinates
// with texel centres at (i+0.5)/res (the cudaFilterModeLinear convention).
inline float tap_border(const float* d, int res, int x, int y, int z) {
  if (x < 0 || y < 0 || z < 0 || x >= res || y >= res || z >= res) return 0.0f;
  return d[((size_t)x * res + y) * res + z];
}
inline float tri_border(const float* d, int res, V3 uv) {
  float px = uv.x * res - 0.5f, py = uv.y * res - 0.5f, pz = uv.z * res - 0.5f;
  float fx = std::floor(px), fy = std::floor(py), fz = std::floor(pz);
  int x = (int)fx, y = (int)fy, z = (int)fz;
  float wx = px - fx, wy = py - fy, wz = pz - fz;
  float c000 = tap_border(d, res, x, y, z), c001 = tap_border(d, res, x, y, z + 1);
  float c010 = tap_border(d, res, x, y + 1, z), c011 = tap_border(d, res, x, y + 1, z + 1);
  float c100 = tap_border(d, res, x + 1, y, z), c101 = tap_border(d, res, x + 1, y, z + 1);
  float c110 = tap_border(d, res, x + 1, y + 1, z), c111 = tap_border(d, res, x + 1, y + 1, z + 1);
  return lerp(lerp(lerp(c000, c001, wz), lerp(c010, c011, wz), wy),
              lerp(lerp(c100, c101, wz), lerp(c110, c111, wz), wy), wx);
}
// Clamp-to-edge addressing (the TR tables are bound with cudaAddressModeClamp,
// core/volume.cu:1412-1417; host reader SampleClamp :704-722).
inline float tap_clamp(const float* d, int res, int x, int y, int z) {
  x = std::max(std::min(x, res - 1), 0);
  y = std::max(std::min(y, res - 1), 0);
  z = std::max(std::min(z, res - 1), 0);
  return d[((size_t)x * res + y) * res + z];
}
inline float tri_clamp(const float* d, int res, V3 uv) {
  float px = uv.x * res - 0.5f, py = uv.y * res - 0.5f, pz = uv.z * res - 0.5f;
  float fx = std::floor(px), fy = std::floor(py), fz = std::floor(pz);
  int x = (int)fx, y = (int)fy, z = (int)fz;
  float wx = px - fx, wy = py - fy, wz = pz - fz;
  float c000 = tap_clamp(d, res, x, y, z), c001 = tap_clamp(d, res, x, y, z + 1);
  float c010 = tap_clamp(d, res, x, y + 1, z), c011 = tap_clamp(d, res, x, y + 1, z + 1);
  float c100 = tap_clamp(d, res, x + 1, y, z), c101 = tap_clamp(d, res, x + 1, y, z + 1);
  float c110 = tap_clamp(d, res, x + 1, y + 1, z), c111 = tap_clamp(d, res, x + 1, y + 1, z + 1);
  return lerp(lerp(lerp(c000, c001, wz), lerp(c010, c011, wz), wy),
              lerp(lerp(c100, c101, wz), lerp(c110, c111, wz), wy), wx);
}
// 2-D bilinear, clamp addressing, lut[i + j*W] (u -> i, v -> j).
inline float bilinear_clamp(const float* d, int w, int h, float u, float v) {
  float px = u * w - 0.5f, py = v * h - 0.5f;
  float fx = std::floor(px), fy = std::floor(py);
  int x = (int)fx, y = (int)fy;
  float wx = px - fx, wy = py - fy;
  int x0 = std::max(std::min(x, w - 1), 0), x1 = std::max(std::min(x + 1, w - 1), 0);
  int y0 = std::max(std::min(y, h - 1), 0), y1 = std::max(std::min(y + 1, h - 1), 0);
  float a = lerp(d[x0 + y0 * w], d[x1 + y0 * w], wx);
  float b = lerp(d[x0 + y1 * w], d[x1 + y1 * w], wx);
  return lerp(a, b, wy);
}

inline size_t mip_offset(int k) { size_t o = 0; for (int j = 0; j < k; ++j) { size_t r = 256 >> j; o += r * r * r; } return o; }
inline size_t tr_offset(int k) { size_t o = 0; for (int j = 0; j < k; ++j) { size_t r = 128 >> j; o += r * r * r; } return o; }

struct Vol {
  const float* density; int res; float max_density;
  const float* mips;  // concatenated levels 0..8
  const float* tr;    // concatenated levels 0..7
  const float* lut;   // 512 x 512
};

struct Scene {
  float alpha, g, tr_scale;
  V3 scatter, light_dir, light_color, env;
  int max_bounces;
};

// Environment map set by orc_set_env (w x h RGBA, row 0 straight up); empty
// = the constant env colour.
static std::vector<float> g_env;
static int g_env_w = 0, g_env_h = 0;

// SkyBox (core/render.cuh:57-61): the map at u = atan2(-d.z, d.x) / 2pi + 1/2,
// v = acos(d.y) / pi, bilinear with wrap, times the env scale.
static V3 sky(const Scene& sc, V3 d) {
  if (g_env.empty()) return sc.env;
  const int w = g_env_w, h = g_env_h;
  const float u = std::atan2(-d.z, d.x) * (float)(0.5 / 3.1415926) + 0.5f;
  const float v = std::acos(std::max(std::min(d.y, 1.0f), -1.0f)) * (float)(1.0 / 3.1415926);
  const float x = u * (float)w - 0.5f, y = v * (float)h - 0.5f;
  const float x0 = std::floor(x), y0 = std::floor(y);
  const float fx = x - x0, fy = y - y0;
  int i0 = (int)x0 % w, j0 = (int)y0 % h;
  if (i0 < 0) i0 += w;
  if (j0 < 0) j0 += h;
  const int i1 = i0 + 1 == w ? 0 : i0 + 1, j1 = j0 + 1 == h ? 0 : j0 + 1;
  auto px = [&](int i, int j, int c) { return g_env[((size_t)j * w + i) * 4 + c]; };
  auto lf = [](float a, float b, float t) { return a * (1.0f - t) + b * t; };
  float r[3];
  for (int c = 0; c < 3; ++c) r[c] = lf(lf(px(i0, j0, c), px(i1, j0, c), fx), lf(px(i0, j1, c), px(i1, j1, c), fx), fy);
  return v3(r[0] * sc.env.x, r[1] * sc.env.y, r[2] * sc.env.z);
}

inline V3 f3(const mr_float3& a) { return v3(a.x, a.y, a.z); }

// ---- delta tracking ---------------------------------------------------------
struct Tracker {
  const Vol& vol;
  const Scene& sc;
  uint64_t fetches = 0;
  uint64_t caps = 0;
  float density(V3 pos) { ++fetches; return tri_border(vol.density, vol.res, pos + 0.5f); }

  // core/render.cuh:138-172 DeterminateNextVertex (Woodcock free flight).
  bool next_vertex(Rng& rng, float alpha, float g, V3 pos, V3 dir, float dis, V3& npos, V3& ndir) {
    float smax = vol.max_density * alpha;
    float t = 0;
    int loop = 0;
    bool capped = true;
    while (loop++ < 10000) {
      float rk = rng.next();
      t -= std::log(1 - rk) / smax;
      if (t > dis) { npos = v3(0, 0, 0); ndir = v3(0, 0, 0); return false; }
      rk = rng.next();
      float d = density(pos + (dir * t));
      float s = d * alpha;
      if (s / smax > rk) { capped = false; break; }
      if (d < 0) t -= d;
    }
    if (capped) ++caps;
    float e0 = rng.next();
    float e1 = rng.next();
    ndir = hg_sample_dir(e0, e1, dir, g);
    npos = (dir * t) + pos;
    return true;
  }

  // core/render.cuh:93-136 Tr: ratio tracking while tr > 0.5, then delta tracking.
  float transmittance(Rng& rng, V3 pos, V3 dir, float dis, float alpha) {
    float smax = vol.max_density * alpha;
    float tr = 1, t = 0;
    int loop = 0;
    while (loop++ < 10000 && tr > 0.5f) {
      float rk = rng.next();
      t -= std::log(1 - rk) / smax * sc.tr_scale;
      if (t > dis) break;
      float d = density(pos + (dir * t));
      float s = d * alpha;
      tr *= 1 - std::max(0.0f, s / smax);
      if (d < 0) t -= d;
    }
    while (loop++ < 10000 && tr > 0.001f) {
      float rk = rng.next();
      t -= std::log(1 - rk) / smax * sc.tr_scale;
      if (t > dis) break;
      float d = density(pos + (dir * t));
      float s = d * alpha;
      if (rng.next() < std::max(0.0f, s / smax)) { tr = 0; break; }
      if (d < 0) t -= d;
    }
    if (loop > 10000) ++caps;
    return tr;
  }

  // core/render.cuh:200-258 CalculateRadiance (one sample). Returns radiance;
  // *first_t = distance to the first scattering vertex or -1.
  V3 radiance(Rng& rng, V3 ori, V3 dir, float* first_t) {
    dir = normalize(dir);
    V3 L = normalize(sc.light_dir);
    float t = -1;
    float dis = ray_box_offset(ori, dir);
    if (dis < 0) { *first_t = t; return sky(sc, dir); }
    V3 res = v3(0, 0, 0);
    V3 pos = ori + dir * dis;
    V3 rd = dir;
    V3 rate = v3(1, 1, 1);
    for (int s = 0; s < sc.max_bounces; ++s) {
      V3 np, nd;
      float maxd = ray_box_distance(pos, rd);
      bool hit = next_vertex(rng, sc.alpha, sc.g, pos, rd, maxd, np, nd);
      if (!hit) { res = res + sky(sc, rd) * rate; break; }
      if (s == 0) t = length(ori - np);
      pos = np;
      rate = rate * sc.scatter;
      maxd = ray_box_distance(pos, L);
      float ph = hg_phase(dot(rd, L), sc.g);
      res = res + (sc.light_color * rate) * (transmittance(rng, pos, L, maxd, sc.alpha) * ph);
      rd = nd;
    }
    *first_t = t;
    return res;
  }
};

// Camera ray of pixel (row, col): core/volume.cu:155-163 with the row-major
// W x H indexing this build defines (u from the column, v from the row).
inline V3 camera_dir(const mr_render_params& p, int row, int col, float jx, float jy) {
  float u = 1.0f - ((float)col + jx) / (float)p.width;
  float v = 1.0f - ((float)row + jy) / (float)p.height;
  V3 fwd = normalize(-f3(p.ori));
  V3 d = fwd + (f3(p.right) * (u * 2 - 1)) + (f3(p.up) * (v * 2 - 1));
  return normalize(d);
}

Scene make_scene(const mr_render_params& p) {
  Scene s;
  s.alpha = p.alpha; s.g = p.g; s.tr_scale = p.tr_scale;
  s.scatter = f3(p.scatter_rate); s.light_dir = f3(p.light_dir);
  s.light_color = f3(p.light_color); s.env = f3(p.env_color);
  s.max_bounces = p.max_bounces;
  return s;
}

// ---- network (core/radiancePredict.cu:11-238, 240-294, 370-485) -------------
struct Net {
  const float* w[MR_W_COUNT];
  explicit Net(const float* blob) {
    size_t off = 0;
#define MR_BIND(name, n) w[MR_W_##name] = blob + off; off += (n);
    MR_WEIGHT_LIST(MR_BIND)
#undef MR_BIND
  }
};

inline float relu(float x) { return x >= 0.0f ? x : 0.0f; }
// AVGMAX (radiancePredict.cu:21-33)
inline void avgmax(const float* in, float* out, int len, int at, int wa, int wm) {
  float s = 0.0f, m = -10000.0f;
  for (int i = 0; i < len; ++i) { s += in[at + i]; m = std::max(m, in[at + i]); }
  out[wa] = s / (float)len;
  out[wm] = m;
}
// LinearReLU_Unbias (:58-72)
inline void lin_relu_nobias(const float* in, float* out, int from, int to, int ra, int wa, const float* W) {
  for (int i = 0; i < to; ++i) {
    float acc = 0.0f;
    for (int j = 0; j < from; ++j) acc += in[j + ra] * W[j + i * from];
    out[i + wa] = relu(acc);
  }
}
// LinearSm_Unbias (:74-86)
inline void lin_sigmoid_nobias(const float* in, float* out, int from, int to, int ra, int wa, const float* W) {
  for (int i = 0; i < to; ++i) {
    float acc = 0.0f;
    for (int j = 0; j < from; ++j) acc += in[j + ra] * W[j + i * from];
    out[i + wa] = 1.0f / (1.0f + std::exp(-acc));
  }
}
// LinearReLU (:41-56): bias added after the sum.
inline void lin_relu_bias_last(const float* in, float* out, int from, int to, int ra, int wa, const float* W, const float* B) {
  for (int i = 0; i < to; ++i) {
    float acc = 0.0f;
    for (int j = 0; j < from; ++j) acc += in[j + ra] * W[j + i * from];
    acc += B[i];
    out[i + wa] = relu(acc);
  }
}
// LinearReLU<Size> / LinearReLU_SFL<From,To> (:129-224): bias first, then the
// products in ascending input order.
inline void lin_relu(const float* in, float* out, int from, int to, int ra, int wa, const float* W, const float* B) {
  for (int i = 0; i < to; ++i) {
    float acc = B[i];
    for (int j = 0; j < from; ++j) acc += in[j + ra] * W[j + i * from];
    out[i + wa] = relu(acc);
  }
}

struct NetState {
  float xv[192], xs[192], xh[192];
  float a[160], b[160], c[160], a2[160], b2[160], c2[160];
  float pool[75], sew[16], sep[6], tmp[8], comb[128];
};

enum { POOL = 36, P_DI = 24, DI = 160 };

// SE / SERES block (macros at radiancePredict.cu:240-279). last < 0 = SE.
void se_block(NetState& s, const Net& n, int last, int from, int to, int size, int pid,
              int sew0, int sew1, int ww, int trw, int hgw) {
  avgmax(s.xv, s.pool, size, from, pid + 0, POOL + pid + 0);
  avgmax(s.xs, s.pool, size, from, pid + 1, POOL + pid + 1);
  avgmax(s.xh, s.pool, size, from, pid + 2, POOL + pid + 2);
  for (int i = 0; i < 3; ++i) { s.tmp[i] = s.pool[pid + i]; s.tmp[3 + i] = s.pool[POOL + pid + i]; }
  lin_relu_nobias(s.tmp, s.sew, 8, 8, 0, 0, n.w[sew0]);
  lin_sigmoid_nobias(s.sew, s.sep, 8, 3, 0, 0, n.w[sew1]);
  const float* srcs[3] = {s.xv, s.xs, s.xh};
  float* xs[3] = {s.a, s.b, s.c};
  float* ys[3] = {s.a2, s.b2, s.c2};
  int wid[3] = {ww, trw, hgw};
  for (int br = 0; br < 3; ++br) {
    for (int i = 0; i < size; ++i) xs[br][to + i] = srcs[br][from + i];
    for (int i = 0; i < size; ++i) xs[br][to + i] *= s.sep[br];
    if (last >= 0)
      for (int i = 0; i < size; ++i) xs[br][to + i] = xs[br][to + i] + ys[br][last + i];
    lin_relu(xs[br], ys[br], size, size, to, to, n.w[wid[br]], n.w[wid[br] + 1]);
  }
}
void add3(NetState& s, int from, int to, int size) {
  for (int i = 0; i < size; ++i) {
    s.a2[to + i] = s.a2[to + i] + s.xv[from + i];
    s.b2[to + i] = s.b2[to + i] + s.xs[from + i];
    s.c2[to + i] = s.c2[to + i] + s.xh[from + i];
  }
}
void rep3(NetState& s, int from, int to, int size) {
  std::memmove(s.a2 + from, s.a2 + to, size * sizeof(float));
  std::memcpy(s.a2 + to, s.xv + to, size * sizeof(float));
  std::memmove(s.b2 + from, s.b2 + to, size * sizeof(float));
  std::memcpy(s.b2 + to, s.xs + to, size * sizeof(float));
  std::memmove(s.c2 + from, s.c2 + to, size * sizeof(float));
  std::memcpy(s.c2 + to, s.xh + to, size * sizeof(float));
}

#define W_(name) MR_W_##name

// Head SC(p) (radiancePredict.cu:439-473) for one albedo channel.
float head(NetState& s, const Net& n, float srp_channel) {
  s.pool[POOL + POOL + 2] = srp_channel;
  std::memcpy(s.a, s.comb, 120 * sizeof(float));
  lin_relu_bias_last(s.pool, s.a, 3, 8, POOL + POOL, 120, n.w[W_(LGGSW)], n.w[W_(LGGSB)]);
  lin_relu_nobias(s.pool, s.sew, 75, 16, 0, 0, n.w[W_(LSEFin1W)]);
  lin_sigmoid_nobias(s.sew, s.sep, 16, 6, 0, 0, n.w[W_(LSEFin2W)]);
  for (int i = 0; i < 32; ++i) s.a[i] *= s.sep[0];
  for (int i = 0; i < 32; ++i) s.a[32 + i] *= s.sep[1];
  for (int i = 0; i < 32; ++i) s.a[64 + i] *= s.sep[2];
  for (int i = 0; i < 8; ++i) s.a[96 + i] *= s.sep[3];
  for (int i = 0; i < 8; ++i) s.a[104 + i] *= s.sep[4];
  for (int i = 0; i < 8; ++i) s.a[112 + i] *= s.sep[5];
  lin_relu(s.a, s.b, 128, 128, 0, 0, n.w[W_(LC0W)], n.w[W_(LC0B)]);
  lin_relu(s.b, s.a, 128, 64, 0, 0, n.w[W_(LC1W)], n.w[W_(LC1B)]);
  lin_relu(s.a, s.b, 64, 32, 0, 0, n.w[W_(LC2W)], n.w[W_(LC2B)]);
  lin_relu(s.b, s.a, 32, 16, 0, 0, n.w[W_(LXW)], n.w[W_(LXB)]);
  const int lx[12] = {W_(LX0W), W_(LX1W), W_(LX2W), W_(LX3W), W_(LX4W), W_(LX5W),
                      W_(LX6W), W_(LX7W), W_(LX8W), W_(LX9W), W_(LX10W), W_(LX11W)};
  for (int r = 0; r < 6; ++r) {
    lin_relu(s.a, s.b, 16, 16, 0, 0, n.w[lx[2 * r]], n.w[lx[2 * r] + 1]);
    lin_relu(s.b, s.c, 16, 16, 0, 0, n.w[lx[2 * r + 1]], n.w[lx[2 * r + 1] + 1]);
    for (int i = 0; i < 16; ++i) s.a[i] = s.a[i] + s.c[i];
  }
  lin_relu_bias_last(s.a, s.b, 16, 1, 0, 0, n.w[W_(LX12W)], n.w[W_(LX12B)]);
  return s.b[0];
}

// Trunks of RadiancePredict (radiancePredict.cu:385-437): fills s.comb and
// s.pool from the gathered arrays in s.xv/xs/xh.
void trunks(NetState& s, const Net& n, float g, float gamma) {
  s.tmp[6] = g;
  s.tmp[7] = gamma;
  s.pool[POOL + POOL] = g;
  s.pool[POOL + POOL + 1] = gamma;
  // main trunk (:396-421)
  se_block(s, n, -1, 0, 0, 8, 0, W_(LSE01W), W_(LSE02W), W_(L01W), W_(L_Tr01W), W_(L_Hg01W));
  add3(s, 0, 0, 8);
  se_block(s, n, 0, 8, 8, 8, 3, W_(LSE11W), W_(LSE12W), W_(L11W), W_(L_Tr11W), W_(L_Hg11W));
  rep3(s, 0, 8, 8);
  se_block(s, n, 0, 16, 16, 16, 6, W_(LSE21W), W_(LSE22W), W_(L21W), W_(L_Tr21W), W_(L_Hg21W));
  add3(s, 16, 16, 16);
  se_block(s, n, 16, 32, 32, 16, 9, W_(LSE31W), W_(LSE32W), W_(L31W), W_(L_Tr31W), W_(L_Hg31W));
  add3(s, 32, 32, 16);
  se_block(s, n, 32, 48, 48, 16, 12, W_(LSE41W), W_(LSE42W), W_(L41W), W_(L_Tr41W), W_(L_Hg41W));
  rep3(s, 32, 48, 16);
  se_block(s, n, 32, 64, 64, 32, 15, W_(LSE51W), W_(LSE52W), W_(L51W), W_(L_Tr51W), W_(L_Hg51W));
  add3(s, 64, 64, 32);
  se_block(s, n, 64, 96, 96, 32, 18, W_(LSE61W), W_(LSE62W), W_(L61W), W_(L_Tr61W), W_(L_Hg61W));
  add3(s, 96, 96, 32);
  se_block(s, n, 96, 128, 128, 32, 21, W_(LSE71W), W_(LSE72W), W_(L71W), W_(L_Tr71W), W_(L_Hg71W));
  add3(s, 128, 128, 32);
  lin_relu(s.a2, s.comb, 32, 32, 128, 0, n.w[W_(L81W)], n.w[W_(L81B)]);
  lin_relu(s.b2, s.comb, 32, 32, 128, 32, n.w[W_(L_Tr81W)], n.w[W_(L_Tr81B)]);
  lin_relu(s.c2, s.comb, 32, 32, 128, 64, n.w[W_(L_Hg81W)], n.w[W_(L_Hg81B)]);
  // light-direction trunk (:424-437)
  se_block(s, n, -1, DI + 0, 0, 8, P_DI + 0, W_(LDSE01W), W_(LDSE02W), W_(LD01W), W_(LD_Tr01W), W_(LD_Hg01W));
  add3(s, DI + 0, 0, 8);
  se_block(s, n, 0, DI + 8, 8, 8, P_DI + 3, W_(LDSE11W), W_(LDSE12W), W_(LD11W), W_(LD_Tr11W), W_(LD_Hg11W));
  add3(s, DI + 8, 8, 8);
  se_block(s, n, 8, DI + 16, 16, 8, P_DI + 6, W_(LDSE21W), W_(LDSE22W), W_(LD21W), W_(LD_Tr21W), W_(LD_Hg21W));
  add3(s, DI + 16, 16, 8);
  se_block(s, n, 16, DI + 24, 24, 8, P_DI + 9, W_(LDSE31W), W_(LDSE32W), W_(LD31W), W_(LD_Tr31W), W_(LD_Hg31W));
  add3(s, DI + 24, 24, 8);
  lin_relu(s.a2, s.comb, 8, 8, 24, 96, n.w[W_(LD41W)], n.w[W_(LD41B)]);
  lin_relu(s.b2, s.comb, 8, 8, 24, 104, n.w[W_(LD_Tr41W)], n.w[W_(LD_Tr41B)]);
  lin_relu(s.c2, s.comb, 8, 8, 24, 112, n.w[W_(LD_Hg41W)], n.w[W_(LD_Hg41B)]);
}

// Heads per distinct albedo channel and the output transform (:475-485).
// srp = scatterrate^4; channels with equal srp share one head evaluation
// (x^4 is monotonic on albedos >= 0, so this is the reference's rate test).
V3 heads(NetState& s, const Net& n, V3 srp) {
  float X = head(s, n, srp.x), Y, Z;
  if (srp.y == srp.x) Y = X; else Y = head(s, n, srp.y);
  if (srp.z == srp.x) Z = X;
  else if (srp.z == srp.y) Z = Y;
  else Z = head(s, n, srp.z);
  return v3(std::max(std::exp(X) - 1.0f, 0.0f) * srp.x, std::max(std::exp(Y) - 1.0f, 0.0f) * srp.y,
            std::max(std::exp(Z) - 1.0f, 0.0f) * srp.z);
}

inline V3 srp_of(V3 sr) {
  return v3((sr.x * sr.x) * (sr.x * sr.x), (sr.y * sr.y) * (sr.y * sr.y), (sr.z * sr.z) * (sr.z * sr.z));
}

// Network body of RadiancePredict given the gathered arrays;
// scatterrate = scatter_rate/1.001.
V3 network(NetState& s, const Net& n, float g, float gamma, V3 scatterrate) {
  trunks(s, n, g, gamma);
  return heads(s, n, srp_of(scatterrate));
}

// ---- descriptor gather (radiancePredict.cu:319-359, renderResources.cu:42-139)
struct Frame { V3 X, Y, Z, LX; };

inline float mip_density(const Vol& vol, int mip, V3 pos) {
  return tri_border(vol.mips + mip_offset(mip), 256 >> mip, pos + 0.5f);
}
inline float mip_tr(const Vol& vol, int mip, V3 pos) {
  return tri_clamp(vol.tr + tr_offset(mip), 128 >> mip, pos + 0.5f);
}
// ShadowTerm_TRTex (renderResources.cu:121-139), light colour 1.
inline float shadow_tr(const Vol& vol, V3 p, V3 L, int mip) {
  if (p.x < -0.5f || p.y < -0.5f || p.z < -0.5f || p.x > 0.5f || p.y > 0.5f || p.z > 0.5f) {
    float off = ray_box_offset(p, L);
    if (off >= 0) return mip_tr(vol, mip, p + L * off);
    return 1.0f;
  }
  return mip_tr(vol, mip, p);
}

void gather(NetState& s, const Vol& vol, const float* stencil, V3 pos, V3 L, const Frame& f,
            float alpha, float g) {
  const float kLutAngle = 3.1415926535f * 60.0f / 180.0f;
  int ri = 0;
  for (int i = 0; i < 192; ++i) {
    StencilInfo si = stencil_info(i);
    float layer = (float)si.mip + 0.1f;
    V3 p;
    if (si.type >= 4) {
      const float* sp = stencil + 3 * ri;
      ++ri;
      p = pos + ((f.X * sp[0] + f.Y * sp[1] + f.Z * sp[2]) * si.offset);
    } else {
      p = pos + L * si.offset;
    }
    int mip = (int)layer;
    s.xv[i] = std::log(1.0f + alpha * mip_density(vol, mip, p) / 64.0f);
    if (si.localindex == 0) {
      s.xh[i] = std::log(hg_phase(dot(f.X, L), g) + 1.0f);
    } else {
      V3 md = normalize(p - pos);
      float radius = (float)(1 << mip) / 256.0f;
      float angle = std::atan(0.5f * radius / si.offset);
      float c1 = dot(f.X, md), c2 = dot(f.LX, md);
      float u1 = c1 * 0.5f + 0.5f, u2 = c2 * 0.5f + 0.5f;
      float v = angle / kLutAngle;
      float h0 = bilinear_clamp(vol.lut, 512, 512, u1, v);
      float h1 = bilinear_clamp(vol.lut, 512, 512, u2, v);
      s.xh[i] = std::log(h0 * h1 + 1.0f);
    }
    s.xs[i] = shadow_tr(vol, p, f.LX, std::max(mip - 1, 0));
  }
}

// GetMatrixFromNormal (core/render.cuh:355-369), rejection capped at 64 tries.
void frame_from(Rng& rng, V3 v1, V3& a, V3& b, V3& c) {
  v1 = normalize(v1);
  for (int tries = 0; tries < 64; ++tries) {
    float ex = rng.next();
    float ey = rng.next();
    V3 r = uniform_sphere(ex, ey);
    if (std::fabs(dot(r, v1)) < 0.01f) continue;
    V3 v2 = normalize(cross(v1, r));
    a = v1; b = v2; c = cross(v2, v1);
    return;
  }
  V3 r = std::fabs(v1.x) < 0.5f ? v3(1, 0, 0) : v3(0, 1, 0);
  V3 v2 = normalize(cross(v1, r));
  a = v1; b = v2; c = cross(v2, v1);
}

// NNPredict<MRPNN> for one pixel (core/render.cuh:469-523) without the warp
// ballot (per-pixel results are identical). Returns radiance; *hit_t set.
V3 neural_pixel(Tracker& tk, const Net& net, const float* stencil, Rng& rng, V3 ori, V3 dir, float* hit_t) {
  const Scene& sc = tk.sc;
  dir = normalize(dir);
  V3 L = normalize(sc.light_dir);
  // GetSamplePoint (:174-198)
  bool active = false;
  V3 pos = v3(0, 0, 0);
  float dis = ray_box_offset(ori, dir);
  if (dis >= 0) {
    V3 sp = ori + dir * dis;
    float maxd = ray_box_distance(sp, dir);
    V3 p0, p1;
    active = tk.next_vertex(rng, sc.alpha, 0.0f, sp, dir, maxd, p0, p1);
    if (active) pos = p0;
  }
  Frame f;
  V3 ly, lz;
  frame_from(rng, dir, f.X, f.Y, f.Z);
  frame_from(rng, L, f.LX, ly, lz);
  if (!active) { *hit_t = -1; return sky(sc, dir); }
  NetState s;
  gather(s, tk.vol, stencil, pos, L, f, sc.alpha, sc.g);
  V3 scatterrate = sc.scatter / 1.001f;
  float gamma = std::acos(dot(f.X, f.LX));
  V3 pred = network(s, net, sc.g, gamma, scatterrate);
  float d2 = ray_box_distance(pos, f.LX);
  float ph = hg_phase(dot(f.X, f.LX), sc.g);
  float tr = tk.transmittance(rng, pos, f.LX, d2, sc.alpha) * ph;
  pred = pred + tr;
  *hit_t = length(ori - pos);
  return (pred * sc.light_color) * sc.scatter;
}

// ---- NNPredict<Type::marching_MRPNN> (core/render.cuh:371-461, 524-633) ----
static V3 m_normal(Tracker& tk, V3 p) {  // Normal, :371-387
  float dl = 0.02f;
  V3 n;
  int left = 10;
  do {
    auto neg = [&](V3 q) { return std::max(0.0f, -tk.density(q)); };
    n = v3(neg(p + v3(dl, 0, 0)) - neg(p - v3(dl, 0, 0)), neg(p + v3(0, dl, 0)) - neg(p - v3(0, dl, 0)),
           neg(p + v3(0, 0, dl)) - neg(p - v3(0, 0, dl)));
    dl += 0.01f;
  } while (n.x == 0.0f && n.y == 0.0f && n.z == 0.0f && left-- > 0);
  return normalize(n);
}
static float m_sat(float x) { return std::min(std::max(x, 0.0f), 1.0f); }
static float m_lerp(float a, float b, float t) { return a * (1.0f - t) + b * t; }
// BRDF (:428-461): GGX specular (F0 0.04, roughness 0.008) and the dielectric
// Fresnel reflectance (PhysicsFresnel, :410-419) in w.
static void m_brdf(V3 n, V3 v, V3 l, float ior, float* spec, float* fres) {
  const V3 h = normalize(l + v);
  const float shift = dot(n, v);
  if (shift < 0.0f) n = n + v * (-shift + 1e-5f);
  const float nv = m_sat(dot(n, v)), nl = m_sat(dot(n, l)), nh = m_sat(dot(n, h)), lh = m_sat(dot(l, h));
  const float r = 0.008f, a2 = r * r;
  const float dd = (nh * a2 - nh) * nh + 1.0f;
  const float D = 0.318309886183790671538f * a2 / (dd * dd + 1e-7f);
  const float k = (r + 0.01f) * (r + 0.01f) / 1.01f / 1.01f / 2.0f;
  const float G = (1e-5f + nl * nv) / (1e-5f + m_lerp(nl, 1.0f, k) * m_lerp(nv, 1.0f, k)) * 3.1415926f;
  const float t = 1.0f - lh;
  const float F = 0.04f + (1.0f - 0.04f) * (t * t * t * t * t);
  *spec = F * G * D * nl;
  const float ci = std::fabs(dot(v, n));
  const float si = std::sqrt(std::max(0.0f, 1.0f - ci * ci));
  const float st = si / ior;
  const float ct = std::sqrt(std::max(0.0f, 1.0f - st * st));
  const float r1 = (ior * ci - ct) / (ior * ci + ct);
  const float r2 = (ci - ior * ct) / (ci + ior * ct);
  *fres = (r1 * r1 + r2 * r2) / 2.0f;
}
static V3 m_refract(V3 i, V3 n, float eta) {
  const float ci = dot(i * -1.0f, n);
  const float c2 = 1.0f - eta * eta * (1.0f - ci * ci);
  const V3 t = i * eta + n * (eta * ci - std::sqrt(std::fabs(c2)));
  return t * (c2 > 0.0f ? 1.0f : 0.0f);
}
static V3 m_reflect(V3 i, V3 n) { return i - n * (dot(i, n) * 2.0f); }

V3 marching_pixel(Tracker& tk, const Net& net, const float* stencil, Rng& rng, V3 ori0, V3 dir, float ior,
                  float* hit_t) {
  const Scene& sc = tk.sc;
  dir = normalize(dir);
  const V3 L = normalize(sc.light_dir);
  Frame f;
  V3 ly, lz;
  frame_from(rng, dir, f.X, f.Y, f.Z);
  frame_from(rng, L, f.LX, ly, lz);
  const float offset = ray_box_offset(ori0, dir);
  bool go = offset >= 0.0f;
  V3 ori = ori0 + dir * offset;
  float dis = ray_box_distance(ori, dir);
  const int steps = 1024;
  float inv = dis / (float)(steps - 1);
  float trans = 1.0f, t = 0.0f, hit_dis = -1.0f, total_w = 0.0f;
  bool surfaced = !(ior > 0.0f);
  V3 ref = v3(0, 0, 0), pos = v3(0, 0, 0);
  for (int step = 0; go; ++step) {
    if (trans < 0.005f || t >= dis || step > steps * 2) break;
    const V3 sp = ori + dir * t;
    const float vd = tk.density(sp);
    if (vd > 0.0f && hit_dis == -1.0f) hit_dis = offset + t;
    t += std::max(inv, -vd);
    if (vd <= 0.0f) continue;
    if (!surfaced) {
      V3 n = m_normal(tk, sp);
      n = n - dir * std::max(0.0f, dot(n, dir) + 0.01f);
      float spec, fres;
      m_brdf(n, dir * -1.0f, L, ior, &spec, &fres);
      const float tr = tk.transmittance(rng, sp, L, ray_box_distance(sp, L), sc.alpha);
      ref = sc.light_color * (spec * tr);
      dir = rng.next() < fres ? m_reflect(dir, n) : m_refract(dir, n, 1.0f / ior);
      ori = sp;
      t = 0.0f;
      dis = ray_box_distance(ori, dir);
      inv = dis / (float)(steps - 1);
      frame_from(rng, dir, f.X, f.Y, f.Z);
      frame_from(rng, L, f.LX, ly, lz);
      surfaced = true;
    }
    const float tr_step = std::exp(-vd * sc.alpha * inv);
    const float w = trans * (1.0f - tr_step);
    total_w += w;
    if (rng.next() < w / total_w) pos = sp;
    trans *= tr_step;
  }
  const V3 skyc = sky(sc, dir);
  *hit_t = hit_dis;
  if (hit_dis < 0.0f) return ref + skyc;
  NetState s;
  gather(s, tk.vol, stencil, pos, L, f, sc.alpha, sc.g);
  const V3 scatterrate = sc.scatter / 1.001f;
  const float gamma = std::acos(dot(f.X, f.LX));
  V3 pred = network(s, net, sc.g, gamma, scatterrate);
  const float ph = hg_phase(dot(f.X, f.LX), sc.g);
  const float tr = tk.transmittance(rng, pos, f.LX, ray_box_distance(pos, f.LX), sc.alpha) * ph;
  pred = pred + tr;
  const V3 lit = pred * sc.light_color;
  return ref + lit * (1.0f - trans) + skyc * trans;
}

inline float u01_tag(uint32_t seed, uint32_t a, uint32_t b, uint32_t tag) {
  Rng r(seed, a, b, tag);
  return r.next();
}

}  // namespace

// =============================================================================
// C ABI (ctypes)
// =============================================================================
extern "C" {

// Environment map for the trackers (n = 0 clears it).
void orc_set_env(const float* rgba, int w, int h) {
  if (!rgba || w <= 0 || h <= 0) {
    g_env.clear();
    g_env_w = g_env_h = 0;
    return;
  }
  g_env.assign(rgba, rgba + (size_t)w * h * 4);
  g_env_w = w;
  g_env_h = h;
}

// The light of neural pass p->sample_offset with the environment map set
// (core/volume.cu:417-432): rate = 4e / (4e + max(light colour)), e =
// max(env colour); with probability rate (Philox(seed; pass, 0, 0, TAG_ENV)
// word 0) the direction is the R2 point (core/vector.cu:174-178) of the pass
// on the uniform sphere and the colour the map there (Image_host::Sample:
// bilinear, clamped, core/volume.hpp:22-42) * env * 4 / rate; otherwise the
// colour / (1 - rate). Writes light_dir[3], light_color[3].
void orc_select_env_light(const mr_render_params* p, float* light_dir, float* light_color) {
  V3 env = f3(p->env_color), lc = f3(p->light_color), L = f3(p->light_dir);
  V3 outL = L, outC = lc;
  const float e = std::max(env.x, std::max(env.y, env.z));
  const float m = std::max(lc.x, std::max(lc.y, lc.z));
  if (!g_env.empty() && e > 0.0f) {
    const float rate = e * 4.0f / (e * 4.0f + m);
    uint32_t ctr[4] = {p->sample_offset, 0u, 0u, (uint32_t)TAG_ENV}, o[4];
    philox4x32_10(ctr, p->seed, 0u, o);
    if (u01(o[0]) < rate) {
      const float g = 1.32471795724474602596f;
      const float ax = 1.0f / g, ay = 1.0f / (g * g);
      const float n = (float)p->sample_offset;
      float rx = ax * n + 0.5f, ry = ay * n + 0.5f;
      rx -= std::floor(rx);
      ry -= std::floor(ry);
      V3 d = uniform_sphere(rx, ry);
      const float u = std::atan2(-d.z, d.x) * (float)(0.5 / 3.1415926) + 0.5f;
      const float vv = std::acos(std::max(std::min(d.y, 1.0f), -1.0f)) * (float)(1.0 / 3.1415926);
      const int w = g_env_w, h = g_env_h;
      auto at = [&](int x, int y, int c) {
        x = std::min(std::max(x, 0), w - 1);
        y = std::min(std::max(y, 0), h - 1);
        return g_env[((size_t)y * w + x) * 4 + c];
      };
      const float pxf = u * (float)w - 0.5f, pyf = vv * (float)h - 0.5f;
      const int x = (int)std::floor(pxf), y = (int)std::floor(pyf);
      const float wx = pxf - (float)x, wy = pyf - (float)y;
      float c3[3];
      for (int c = 0; c < 3; ++c) {
        const float a0 = at(x, y, c) * (1.0f - wx) + at(x + 1, y, c) * wx;
        const float a1 = at(x, y + 1, c) * (1.0f - wx) + at(x + 1, y + 1, c) * wx;
        c3[c] = a0 * (1.0f - wy) + a1 * wy;
      }
      const float k = 4.0f / rate;
      outL = d;
      outC = v3(c3[0] * env.x * k, c3[1] * env.y * k, c3[2] * env.z * k);
    } else {
      outC = lc * (1.0f / (1.0f - rate));
    }
  }
  light_dir[0] = outL.x; light_dir[1] = outL.y; light_dir[2] = outL.z;
  light_color[0] = outC.x; light_color[1] = outC.y; light_color[2] = outC.z;
}

void orc_philox(const uint32_t* ctr, const uint32_t* key, uint32_t* out) {
  philox4x32_10(ctr, key[0], key[1], out);
}

// Xavier-uniform weights of the benchmark network (the workload definition
// the library's mr_weights_xavier draws): array a of the blob (declaration
// order of core/NNWeight.cuh), element e uses word e % 4 of
// Philox(seed, 0; a, e / 4, 0, TAG_MISC); weights uniform in
// +-sqrt(6 / (fan_in + fan_out)), biases 0. Fan-in / fan-out from the
// layer shapes of core/radiancePredict.cu:370-485.
void orc_weights_xavier(uint32_t seed, float* out) {
  struct Shape { int in, out; };
  auto shape = [](const char* name, int n) -> Shape {
    const size_t len = std::strlen(name);
    if (!std::strcmp(name, "LSEFin1W")) return {75, 16};
    if (!std::strcmp(name, "LSEFin2W")) return {16, 6};
    if (!std::strcmp(name, "LGGSW")) return {3, 8};
    if (!std::strcmp(name, "LC1W")) return {128, 64};
    if (!std::strcmp(name, "LC2W")) return {64, 32};
    if (!std::strcmp(name, "LXW")) return {32, 16};
    if (!std::strcmp(name, "LX12W")) return {16, 1};
    if (len > 4 && name[len - 2] == '2' && name[len - 1] == 'W' && n == 24) return {8, 3};
    const int k = (int)std::lround(std::sqrt((double)n));
    return {k, k};
  };
  int a = 0;
  size_t off = 0;
#define ORC_XAV(name, n)                                                            \
  {                                                                                 \
    const char* nm = #name;                                                         \
    const bool bias = nm[std::strlen(nm) - 1] == 'B';                               \
    const Shape sh = shape(nm, (n));                                                \
    const float lim = bias ? 0.0f : (float)std::sqrt(6.0 / (double)(sh.in + sh.out)); \
    for (int e = 0; e < (n); ++e) {                                                 \
      uint32_t ctr[4] = {(uint32_t)a, (uint32_t)(e >> 2), 0u, (uint32_t)TAG_MISC}, o[4]; \
      philox4x32_10(ctr, seed, 0u, o);                                              \
      out[off + e] = bias ? 0.0f : (2.0f * u01(o[e & 3]) - 1.0f) * lim;             \
    }                                                                               \
    off += (n);                                                                     \
    ++a;                                                                            \
  }
  MR_WEIGHT_LIST(ORC_XAV)
#undef ORC_XAV
}
void orc_uniforms(uint32_t seed, uint32_t a, uint32_t b, uint32_t tag, int n, float* out) {
  Rng r(seed, a, b, tag);
  for (int i = 0; i < n; ++i) out[i] = r.next();
}
float orc_hg(float c, float g) { return hg_phase(c, g); }
float orc_hg_sample_cos(float s, float g) { return hg_sample_cos(s, g); }
void orc_hg_sample_dir(float e0, float e1, const float* v, float g, float* out) {
  V3 r = hg_sample_dir(e0, e1, v3(v[0], v[1], v[2]), g);
  out[0] = r.x; out[1] = r.y; out[2] = r.z;
}
float orc_ray_box_offset(const float* p, const float* d) { return ray_box_offset(v3(p[0], p[1], p[2]), v3(d[0], d[1], d[2])); }
float orc_ray_box_distance(const float* p, const float* d) { return ray_box_distance(v3(p[0], p[1], p[2]), v3(d[0], d[1], d[2])); }
void orc_stencil_info(int i, float* offset, int* mip, int* type, int* localindex) {
  StencilInfo s = stencil_info(i);
  *offset = s.offset; *mip = s.mip; *type = s.type; *localindex = s.localindex;
}
float orc_sample_border(const float* d, int res, const float* uv) { return tri_border(d, res, v3(uv[0], uv[1], uv[2])); }
float orc_sample_clamp(const float* d, int res, const float* uv) { return tri_clamp(d, res, v3(uv[0], uv[1], uv[2])); }
float orc_sample_lut(const float* lut, float u, float v) { return bilinear_clamp(lut, 512, 512, u, v); }

// Update(): intended mip/variance pyramid (core/volume.cu:1228-1287, :775-827).
// mip0 = trilinear resample (zero border, negatives clamped) to 256^3;
// mip k+1 = 2x2x2 mean of mip k; var k+1 = max(0, E[x^2] - E[x]^2); var0 = 0.
// Returns the global majorant max(1e-5, max density) (:1219-1224).
float orc_build_mips(const float* density, int res, float* mips, float* var, int nthreads) {
  float md = 0.00001f;
  size_t n = (size_t)res * res * res;
  for (size_t i = 0; i < n; ++i) md = std::max(md, density[i]);
  std::vector<float> clamped(n);
  for (size_t i = 0; i < n; ++i) clamped[i] = std::max(0.0f, density[i]);
  float* m0 = mips;
#pragma omp parallel for num_threads(nthreads) schedule(static)
  for (int x = 0; x < 256; ++x)
    for (int y = 0; y < 256; ++y)
      for (int z = 0; z < 256; ++z) {
        V3 uv = v3(((float)x + 0.5f) / 256.0f, ((float)y + 0.5f) / 256.0f, ((float)z + 0.5f) / 256.0f);
        m0[((size_t)x * 256 + y) * 256 + z] = tri_border(clamped.data(), res, uv);
      }
  std::memset(var, 0, sizeof(float) * 256 * 256 * 256);
  for (int k = 0; k < 8; ++k) {
    int r = 256 >> k, nr = r >> 1;
    const float* src = mips + mip_offset(k);
    float* dm = mips + mip_offset(k + 1);
    float* dv = var + mip_offset(k + 1);
#pragma omp parallel for num_threads(nthreads) schedule(static)
    for (int x = 0; x < nr; ++x)
      for (int y = 0; y < nr; ++y)
        for (int z = 0; z < nr; ++z) {
          float s = 0.0f, s2 = 0.0f;
          for (int dx = 0; dx < 2; ++dx)
            for (int dy = 0; dy < 2; ++dy)
              for (int dz = 0; dz < 2; ++dz) {
                float v = src[((size_t)(2 * x + dx) * r + (2 * y + dy)) * r + (2 * z + dz)];
                s += v;
                s2 += v * v;
              }
          float mean = s / 8.0f;
          float variance = s2 / 8.0f - mean * mean;
          size_t o = ((size_t)x * nr + y) * nr + z;
          dm[o] = mean;
          dv[o] = std::max(0.0f, variance);
        }
  }
  return md;
}

// Fill_TR (core/volume.cu:1320-1345) for all 8 levels: level k (res 128>>k)
// marches 128 steps towards the light through mip k+1 with alpha/1.73^(k+1).
void orc_build_tr(const float* mips, float alpha, const float* light, float* tr, int nthreads) {
  V3 L = normalize(v3(light[0], light[1], light[2]));
  for (int k = 0; k < 8; ++k) {
    int r = 128 >> k;
    const float* src = mips + mip_offset(k + 1);
    float* dst = tr + tr_offset(k);
    float a = alpha / std::pow(1.73f, (float)k + 1.0f);
#pragma omp parallel for num_threads(nthreads) schedule(static)
    for (int x = 0; x < r; ++x)
      for (int y = 0; y < r; ++y)
        for (int z = 0; z < r; ++z) {
          V3 uv = v3(((float)x + 0.5f) / (float)r, ((float)y + 0.5f) / (float)r, ((float)z + 0.5f) / (float)r);
          V3 o = uv - 0.5f;
          float dis = ray_box_distance(o, L);
          float step = dis / 128.0f;
          V3 lp = o;
          float sum = 0.0f;
          for (int i = 0; i < 128; ++i) {
            lp = lp + L * step;
            sum = sum + tri_border(src, r, lp + 0.5f);
          }
          dst[((size_t)x * r + y) * r + z] = std::exp(-sum * a * step);
        }
  }
}

// Scrambled radical inverse (ScrambledRadicalInverse, core/volume.cu:1060-1076):
// digit d of a in base b is replaced by perm[d]; the tail of perm[0] digits
// adds perm[0] / (b - 1) of the last digit weight; clamped below 1.
static float scrambled_radical_inverse(uint32_t base, const uint8_t* perm, uint32_t a) {
  const float inv_base = 1.0f / (float)base;
  uint32_t rev = 0;
  float inv_bn = 1.0f;
  while (a) {
    uint32_t next = a / base;
    uint32_t digit = a - next * base;
    rev = rev * base + perm[digit];
    inv_bn *= inv_base;
    a = next;
  }
  return std::min(inv_bn * ((float)rev + inv_base * (float)perm[0] / (1.0f - inv_base)), 0.99999994f);
}
// The permutation-table entries of the Halton dimensions Fill_Hg draws
// (dims 0, 1, 2, 4 = bases 2, 3, 5, 11; core/volume.cu:956-958).
static const uint8_t kPerm2[2] = {0, 1}, kPerm3[3] = {2, 1, 0}, kPerm5[5] = {4, 1, 2, 3, 0},
                     kPerm11[11] = {8, 3, 5, 4, 7, 2, 6, 9, 1, 10, 0};
static inline float fracf(float f) { return f - (float)(long)f; }

// One texel of Fill_Hg (core/volume.cu:1082-1160): the average of HG over a
// ball of radius tan(angle_j) centred on direction cos_i at unit distance,
// 1024 scrambled Halton samples (dims 0,1,2 and 4) mixing HG-sampled chords
// and uniform ball points, shifted by the texel's offset bn.
static float hglut_texel(int i, int j, float g, float bn) {
  float costheta = (((float)i + 0.5f) / 512.0f) * 2.0f - 1.0f;
  float aa = ((float)j + 0.5f) / 512.0f;
  float angle = aa * 3.1415926535f * 60.0f / 180.0f;
  float hg = 0.0f;
  float R = std::tan(angle);
  V3 view = v3(1, 0, 0);
  V3 D = v3(costheta, std::sqrt(1.0f - costheta * costheta), 0.0f);
  float mis = 0.0f;
  {
    float p = R * R - 1 + D.x * D.x;
    if (p > 0) {
      float sdotl = g > 0 ? D.x : -D.x;
      float w = std::sqrt(p);
      float d0 = std::max(0.0f, sdotl - w) / R;
      float d1 = (sdotl + w) / R;
      float d = d1 * d1 * d1 - d0 * d0 * d0;
      mis = (d1 > d0) ? d : 0.0f;
    }
    mis = std::min(std::max(mis, 1e-8f), 1.0f);
    float a = std::fabs(g);
    a = a < 0.6f ? 0.0f : (a < 0.7f ? (a - 0.6f) * 9.0f : (std::pow((a - 0.7f) / 0.3f, 0.05f) * 0.1f + 0.9f));
    mis = 1.0f - 1.0f / (1.0f + a * mis / (1.0f - a));
  }
  for (int k = 0; k < 1024; ++k) {
    float r0 = fracf(scrambled_radical_inverse(2, kPerm2, k) + bn);
    float r1 = fracf(scrambled_radical_inverse(3, kPerm3, k) + bn);
    if (fracf(scrambled_radical_inverse(11, kPerm11, k) + bn) < mis) {
      V3 l = hg_sample_dir(r0, r1, view, g);
      float sdotl = dot(D, l);
      float p = R * R - 1 + sdotl * sdotl;
      if (p <= 0) continue;
      float w = std::sqrt(p);
      float d0 = sdotl - w;
      float d1 = (sdotl + w) / R;
      d0 = std::max(0.0f, d0) / R;
      float d = d1 * d1 * d1 - d0 * d0 * d0;
      hg += std::max(0.0f, d / 4);
    } else {
      float r2 = fracf(scrambled_radical_inverse(5, kPerm5, k) + bn);
      float theta = r0 * 2.0f * 3.1415926535f;
      float phi = std::acos(2.0f * r1 - 1.0f);
      float rr = std::cbrt(r2);
      float x = R * rr * std::sin(phi) * std::cos(theta);
      float y = R * rr * std::sin(phi) * std::sin(theta);
      float z = R * rr * std::cos(phi);
      V3 rp = v3(x, y, z) + D;
      hg += hg_phase(dot(normalize(rp), view), g);
    }
  }
  return hg / 1024.0f;
}

// The 512 x 512 table, lut[i + j*512], with the per-texel offset drawn from
// Philox (seed; i + 512 j, 0, TAG_LUT) where the reference draws it from curand.
void orc_build_hglut(float g, uint32_t seed, float* lut, int nthreads) {
#pragma omp parallel for num_threads(nthreads) schedule(static)
  for (int j = 0; j < 512; ++j)
    for (int i = 0; i < 512; ++i) lut[i + j * 512] = hglut_texel(i, j, g, u01_tag(seed, (uint32_t)(i + j * 512), 0, TAG_LUT));
}

// n texels (i = texel[k] % 512, j = texel[k] / 512) with given offsets bn[k]:
// evaluates the table's estimator with the offsets another generator drew.
void orc_hglut_texels(float g, const int32_t* texel, const float* bn, int n, float* out, int nthreads) {
#pragma omp parallel for num_threads(nthreads) schedule(static)
  for (int k = 0; k < n; ++k) out[k] = hglut_texel(texel[k] % 512, texel[k] / 512, g, bn[k]);
}

// Delta-tracking render (VolumeRender::Render, rt = PT). Pixel (row, col),
// sample s uses Philox stream (seed; row*W+col, sample_offset+s, ., TAG_PT):
// draws 0,1 jitter, then the path. Writes per-pixel sums and sums of squares
// of the radiance (W*H*3 each, fp64). Rows [row0, row1) only.
void orc_render_pt(const float* density, int res, float max_density, const mr_render_params* p,
                   int row0, int row1, double* sum, double* sumsq, uint64_t* counters, int nthreads) {
  Vol vol{density, res, max_density, nullptr, nullptr, nullptr};
  Scene sc = make_scene(*p);
  std::atomic<uint64_t> fetches{0}, caps{0};
#pragma omp parallel for num_threads(nthreads) schedule(dynamic, 1)
  for (int row = row0; row < row1; ++row) {
    Tracker tk{vol, sc};
    for (int col = 0; col < p->width; ++col) {
      size_t pix = (size_t)row * p->width + col;
      double acc[3] = {0, 0, 0}, acc2[3] = {0, 0, 0};
      for (int s = 0; s < p->spp; ++s) {
        Rng rng(p->seed, (uint32_t)pix, p->sample_offset + (uint32_t)s, TAG_PT);
        float jx = rng.next(), jy = rng.next();
        V3 dir = camera_dir(*p, row, col, jx, jy);
        float t;
        V3 L = tk.radiance(rng, f3(p->ori), dir, &t);
        L = vmax(L, v3(0, 0, 0));
        acc[0] += L.x; acc[1] += L.y; acc[2] += L.z;
        acc2[0] += (double)L.x * L.x; acc2[1] += (double)L.y * L.y; acc2[2] += (double)L.z * L.z;
      }
      for (int c = 0; c < 3; ++c) {
        sum[pix * 3 + c] = acc[c];
        if (sumsq) sumsq[pix * 3 + c] = acc2[c];
      }
    }
    fetches += tk.fetches;
    caps += tk.caps;
  }
  if (counters) { counters[0] = fetches.load(); counters[1] = caps.load(); }
}

// Neural render (rt = MRPNN), one primary sample per pixel with stream
// (seed; pixel, sample_offset, ., TAG_NN): draws 0,1 jitter, then
// GetSamplePoint, two frames, and the single-scatter Tr.
void orc_render_neural_dist(const float* density, int res, float max_density, const float* mips, const float* tr,
                            const float* lut, const float* weights, const float* stencil, const mr_render_params* p,
                            int row0, int row1, float* out_rgb, float* out_dist, int nthreads);
void orc_render_neural(const float* density, int res, float max_density, const float* mips,
                       const float* tr, const float* lut, const float* weights, const float* stencil,
                       const mr_render_params* p, int row0, int row1, float* out_rgb, int nthreads) {
  orc_render_neural_dist(density, res, max_density, mips, tr, lut, weights, stencil, p, row0, row1, out_rgb, nullptr,
                         nthreads);
}

// NNPredict<Type::marching_MRPNN> render, rows [row0, row1): the marching
// form with surface index of refraction `ior` (<= 0: no surface); the same
// per-pixel Philox stream as the neural render.
void orc_render_marching(const float* density, int res, float max_density, const float* mips, const float* tr,
                         const float* lut, const float* weights, const float* stencil, const mr_render_params* p,
                         float ior, int row0, int row1, float* out_rgb, int nthreads) {
  Vol vol{density, res, max_density, mips, tr, lut};
  Scene sc = make_scene(*p);
  Net net(weights);
#pragma omp parallel for num_threads(nthreads) schedule(dynamic, 1)
  for (int row = row0; row < row1; ++row) {
    Tracker tk{vol, sc};
    for (int col = 0; col < p->width; ++col) {
      size_t pix = (size_t)row * p->width + col;
      Rng rng(p->seed, (uint32_t)pix, p->sample_offset, TAG_NN);
      float jx = rng.next(), jy = rng.next();
      V3 dir = camera_dir(*p, row, col, jx, jy);
      float t;
      V3 L = marching_pixel(tk, net, stencil, rng, f3(p->ori), dir, ior, &t);
      L = vmax(L, v3(0, 0, 0));
      out_rgb[pix * 3 + 0] = L.x; out_rgb[pix * 3 + 1] = L.y; out_rgb[pix * 3 + 2] = L.z;
    }
  }
}

// Same, also writing each pixel's first-hit distance (< 0: no medium), the
// input of the interactive mode's reprojection.
void orc_render_neural_dist(const float* density, int res, float max_density, const float* mips, const float* tr,
                            const float* lut, const float* weights, const float* stencil, const mr_render_params* p,
                            int row0, int row1, float* out_rgb, float* out_dist, int nthreads) {
  Vol vol{density, res, max_density, mips, tr, lut};
  Scene sc = make_scene(*p);
  Net net(weights);
#pragma omp parallel for num_threads(nthreads) schedule(dynamic, 1)
  for (int row = row0; row < row1; ++row) {
    Tracker tk{vol, sc};
    for (int col = 0; col < p->width; ++col) {
      size_t pix = (size_t)row * p->width + col;
      Rng rng(p->seed, (uint32_t)pix, p->sample_offset, TAG_NN);
      float jx = rng.next(), jy = rng.next();
      V3 dir = camera_dir(*p, row, col, jx, jy);
      float t;
      V3 L = neural_pixel(tk, net, stencil, rng, f3(p->ori), dir, &t);
      L = vmax(L, v3(0, 0, 0));
      out_rgb[pix * 3 + 0] = L.x; out_rgb[pix * 3 + 1] = L.y; out_rgb[pix * 3 + 2] = L.z;
      if (out_dist) out_dist[pix] = t;
    }
  }
}

// Gather + network for n points with explicit frames (bypasses the RNG):
// pos n x 3, frame n x 12 (X, Y, Z, LX). Writes desc n x 576, aux n x 5 and,
// if out != NULL, the network output n x 3.
void orc_gather(const float* mips, const float* tr, const float* lut, const float* stencil,
                const float* pos, const float* frame, int n, float alpha, float g,
                const float* scatter_rate, const float* light_dir, float* desc, float* aux) {
  Vol vol{nullptr, 0, 0, mips, tr, lut};
  V3 L = normalize(v3(light_dir[0], light_dir[1], light_dir[2]));
  V3 sr = v3(scatter_rate[0], scatter_rate[1], scatter_rate[2]) / 1.001f;
#pragma omp parallel for schedule(static)
  for (int k = 0; k < n; ++k) {
    NetState s;
    const float* fr = frame + 12 * k;
    Frame f{v3(fr[0], fr[1], fr[2]), v3(fr[3], fr[4], fr[5]), v3(fr[6], fr[7], fr[8]), v3(fr[9], fr[10], fr[11])};
    gather(s, vol, stencil, v3(pos[3 * k], pos[3 * k + 1], pos[3 * k + 2]), L, f, alpha, g);
    std::memcpy(desc + 576 * k, s.xv, 192 * sizeof(float));
    std::memcpy(desc + 576 * k + 192, s.xs, 192 * sizeof(float));
    std::memcpy(desc + 576 * k + 384, s.xh, 192 * sizeof(float));
    float* ax = aux + 5 * k;
    ax[0] = g;
    ax[1] = std::acos(dot(f.X, f.LX));
    V3 srp = srp_of(sr);
    ax[2] = srp.x; ax[3] = srp.y; ax[4] = srp.z;
  }
}

// Network body on n descriptors (desc n x 576, aux n x 5 = g, gamma, srp.xyz).
void orc_predict(const float* weights, const float* desc, const float* aux, int n, float* out) {
  Net net(weights);
#pragma omp parallel for schedule(static)
  for (int k = 0; k < n; ++k) {
    NetState s;
    std::memcpy(s.xv, desc + 576 * k, 192 * sizeof(float));
    std::memcpy(s.xs, desc + 576 * k + 192, 192 * sizeof(float));
    std::memcpy(s.xh, desc + 576 * k + 384, 192 * sizeof(float));
    const float* ax = aux + 5 * k;
    trunks(s, net, ax[0], ax[1]);
    V3 r = heads(s, net, v3(ax[2], ax[3], ax[4]));
    out[3 * k + 0] = r.x; out[3 * k + 1] = r.y; out[3 * k + 2] = r.z;
  }
}

// Procedural cloud (same definition as oracle/cloud_np.py): Perlin improved
// noise fBm, normalised, thresholded, radial falloff; perm = 256 entries.
static inline float orc_fade(float t) { return t * t * t * (t * (t * 6.0f - 15.0f) + 10.0f); }
static inline float orc_grad(int h, float x, float y, float z) {
  h &= 15;
  float u = h < 8 ? x : y;
  float v = h < 4 ? y : (h == 12 || h == 14 ? x : z);
  return ((h & 1) ? -u : u) + ((h & 2) ? -v : v);
}
static float orc_perlin(const int* P, float x, float y, float z) {
  float fx = std::floor(x), fy = std::floor(y), fz = std::floor(z);
  int X = (int)fx & 255, Y = (int)fy & 255, Z = (int)fz & 255;
  x -= fx; y -= fy; z -= fz;
  float u = orc_fade(x), v = orc_fade(y), w = orc_fade(z);
  int A = P[X] + Y, AA = P[A] + Z, AB = P[A + 1] + Z, B = P[X + 1] + Y, BA = P[B] + Z, BB = P[B + 1] + Z;
  return lerp(lerp(lerp(orc_grad(P[AA], x, y, z), orc_grad(P[BA], x - 1, y, z), u),
                   lerp(orc_grad(P[AB], x, y - 1, z), orc_grad(P[BB], x - 1, y - 1, z), u), v),
              lerp(lerp(orc_grad(P[AA + 1], x, y, z - 1), orc_grad(P[BA + 1], x - 1, y, z - 1), u),
                   lerp(orc_grad(P[AB + 1], x, y - 1, z - 1), orc_grad(P[BB + 1], x - 1, y - 1, z - 1), u), v),
              w);
}
void orc_cloud(int res, const int* perm256, int octaves, float f0, float lac, float gain, float thr, float* out,
               int nthreads) {
  int P[512];
  for (int i = 0; i < 512; ++i) P[i] = perm256[i & 255];
#pragma omp parallel for num_threads(nthreads) schedule(static)
  for (int x = 0; x < res; ++x)
    for (int y = 0; y < res; ++y)
      for (int z = 0; z < res; ++z) {
        float px = ((float)x + 0.5f) / res, py = ((float)y + 0.5f) / res, pz = ((float)z + 0.5f) / res;
        float sum = 0.0f, norm = 0.0f, amp = 1.0f, f = f0;
        for (int o = 0; o < octaves; ++o) {
          sum += amp * orc_perlin(P, px * f, py * f, pz * f);
          norm += amp;
          amp *= gain;
          f *= lac;
        }
        float nv = 0.5f + 0.5f * sum / norm;
        float dx = px - 0.5f, dy = py - 0.5f, dz = pz - 0.5f;
        float r2 = 4.0f * (dx * dx + dy * dy + dz * dz);
        out[((size_t)x * res + y) * res + z] = std::max(0.0f, nv - thr) / (1.0f - thr) * std::max(0.0f, 1.0f - r2);
      }
}

// Training label GetSample (core/render.cuh:276-315): multiple-scattering
// radiance at pos along view dir, light L; stream (seed; k, sample, ., TAG_LABEL).
void orc_get_samples(const float* density, int res, float max_density, const float* pos,
                     const float* dir, const float* light, const float* alpha, const float* g,
                     const float* scatter, int n, int max_bounces, int spp, uint32_t seed,
                     double* out, int nthreads) {
  Vol vol{density, res, max_density, nullptr, nullptr, nullptr};
#pragma omp parallel for num_threads(nthreads) schedule(dynamic, 1)
  for (int k = 0; k < n; ++k) {
    Scene sc;
    sc.alpha = alpha[k]; sc.g = g[k]; sc.tr_scale = 1.0f;
    sc.scatter = v3(scatter[k], scatter[k], scatter[k]);
    sc.light_dir = v3(light[3 * k], light[3 * k + 1], light[3 * k + 2]);
    sc.light_color = v3(1, 1, 1); sc.env = g_env.empty() ? v3(0, 0, 0) : v3(1, 1, 1); sc.max_bounces = max_bounces;
    Tracker tk{vol, sc};
    V3 L = normalize(sc.light_dir);
    V3 d0 = v3(dir[3 * k], dir[3 * k + 1], dir[3 * k + 2]);
    double acc = 0.0;
    for (int s = 0; s < spp; ++s) {
      Rng rng(seed, (uint32_t)k, (uint32_t)s, TAG_LABEL);
      V3 sp = v3(pos[3 * k], pos[3 * k + 1], pos[3 * k + 2]);
      float e0 = rng.next(), e1 = rng.next();
      V3 rd = hg_sample_dir(e0, e1, d0, sc.g);
      float rate = 1.0f;
      float res_acc = 0.0f;
      for (int b = 0; b < max_bounces; ++b) {
        V3 np, nd;
        float dis = ray_box_distance(sp, rd);
        if (!tk.next_vertex(rng, sc.alpha, sc.g, sp, rd, dis, np, nd)) {
          res_acc = res_acc + rate * sky(sc, rd).x;  // SkyBox on escape (black without a map)
          break;
        }
        sp = np;
        rate = rate * 1.001f * scatter[k];
        dis = ray_box_distance(sp, L);
        float ph = hg_phase(dot(rd, L), sc.g);
        res_acc = res_acc + rate * (tk.transmittance(rng, sp, L, dis, sc.alpha) * ph);
        rd = nd;
      }
      acc += res_acc;
    }
    out[k] = acc / spp;
  }
}


// Training points (dataGen.cu:148-216 MeanFreePathSample on rays of
// GetDesiredCountSample), in ray order: per ray the stream (seed; r, 0, .,
// TAG_GEN), four draws for origin and direction, then per Woodcock vertex the
// free-flight draws and six more (keep, jitter, 3 offsets, view). Returns the
// number of points (<= cap written).
// `density` is the grid the Woodcock steps read: dataGen's host code samples
// VolumeRender::DensityAtPosition(0, p), the 256^3 mip level 0
// (core/volume.cu:1495-1497), with the density grid's max_density as majorant.
int orc_train_points(const float* density, int res, float max_density, float alpha, float g, uint32_t seed,
                     int n_rays, int cap, float* pos, float* dir) {
  Vol vol{density, res, max_density, nullptr, nullptr, nullptr};
  Scene sc{};
  sc.alpha = alpha; sc.g = g; sc.tr_scale = 1.0f;
  Tracker tk{vol, sc};
  int count = 0;
  for (int r = 0; r < n_rays; ++r) {
    Rng rng(seed, (uint32_t)r, 0u, TAG_GEN);
    float e0 = rng.next(), e1 = rng.next(), e2 = rng.next(), e3 = rng.next();
    V3 ori = uniform_sphere(e0, e1) * 0.5f;
    V3 d = normalize(uniform_sphere(e2, e3) + normalize(ori * -1.0f));
    float dis = ray_box_offset(ori, d);
    if (dis < 0) continue;
    V3 sp = ori + d * dis, rd = d;
    for (int i = 0; i < 4; ++i) {
      float dd = ray_box_distance(sp, rd);
      V3 np, nd;
      // dataGen.cu:148-172: one draw per tentative collision for both the
      // step and the acceptance test
      bool hit = false;
      {
        const float smax = max_density * alpha;
        float t = 0;
        int loop = 0;
        while (loop++ < 10000) {
          const float rk = rng.next();
          t -= std::log(1 - rk) / smax;
          if (t > dd) break;
          const float dv = tk.density(sp + rd * t);
          if (dv * alpha / smax > rk) { hit = true; break; }
          if (dv < 0) t -= dv;
        }
        if (!hit && loop > 10000) hit = true;  // the step cap accepts, as the reference's loop exit does
        if (hit) {
          const float e0 = rng.next(), e1 = rng.next();
          nd = hg_sample_dir(e0, e1, rd, g);
          np = rd * t + sp;
        }
      }
      if (!hit) break;
      float uk = rng.next(), uj = rng.next(), j0 = rng.next(), j1 = rng.next(), j2 = rng.next(), uv = rng.next();
      V3 dv = sp - np;
      if (i == 0 || dot(dv, dv) > 1.0f / 64.0f || uk > 0.9f) {
        V3 p = np;
        // hash3box (dataGen.cu:115-118): uniform in the ball of radius 1/128
        if (uj > 0.5f) p = p + uniform_sphere(j0, j1) * (std::cbrt(j2) * (1.0f / 128.0f));
        V3 v = uv > 0.25f ? d : rd;
        if (count < cap) {
          pos[3 * count] = p.x; pos[3 * count + 1] = p.y; pos[3 * count + 2] = p.z;
          dir[3 * count] = v.x; dir[3 * count + 1] = v.y; dir[3 * count + 2] = v.z;
        }
        ++count;
      }
      sp = np;
      rd = nd;
    }
  }
  return count;
}

// Frames of NNPredict for view directions (stream (seed; k, 1, ., TAG_MISC)).
void orc_train_frames(const float* dir, int n, const float* light, uint32_t seed, float* frame) {
  V3 L = normalize(v3(light[0], light[1], light[2]));
  for (int k = 0; k < n; ++k) {
    Rng rng(seed, (uint32_t)k, 1u, TAG_MISC);
    V3 X, Y, Z, LX, ly, lz;
    frame_from(rng, v3(dir[3 * k], dir[3 * k + 1], dir[3 * k + 2]), X, Y, Z);
    frame_from(rng, L, LX, ly, lz);
    float* f = frame + 12 * k;
    f[0] = X.x; f[1] = X.y; f[2] = X.z; f[3] = Y.x; f[4] = Y.y; f[5] = Y.z;
    f[6] = Z.x; f[7] = Z.y; f[8] = Z.z; f[9] = LX.x; f[10] = LX.y; f[11] = LX.z;
  }
}

// Training loss of the network on n rows: mean of (X - log(1 + label/srp.x))^2,
// X the head output (before exp) of the first albedo channel.
double orc_train_loss(const float* weights, const float* desc, const float* aux, const float* label, int n) {
  Net net(weights);
  double loss = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : loss)
  for (int k = 0; k < n; ++k) {
    NetState s;
    std::memcpy(s.xv, desc + 576 * k, 192 * sizeof(float));
    std::memcpy(s.xs, desc + 576 * k + 192, 192 * sizeof(float));
    std::memcpy(s.xh, desc + 576 * k + 384, 192 * sizeof(float));
    const float* ax = aux + 5 * k;
    trunks(s, net, ax[0], ax[1]);
    float X = head(s, net, ax[2]);
    float T = std::log1p(std::max(label[k], 0.0f) / ax[2]);
    double e = (double)X - (double)T;
    loss += e * e;
  }
  return loss / n;
}


// ---- interactive path: histograms, Denoise, tone mapping (core/volume.cu:101-124,
// 181-264; core/render.cuh:640-732) -------------------------------------------------
static inline float lerp_f(float a, float b, float t) { return a * (1.0f - t) + b * t; }

// One frame's histogram / running-mean update from this frame's radiance
// (RenderCamera<false>, core/volume.cu:101-124); hist is W*H x 33 floats.
void orc_histogram_frame(const float* rad, int n, int fnum, float* accum, float* hist) {
  const float rate = 1.0f / (float)(1 + fnum);
  for (int p = 0; p < n; ++p) {
    float* h = hist + 33 * p;
    if (fnum == 0)
      for (int i = 0; i < 33; ++i) h[i] = 0.0f;
    float r[3];
    for (int c = 0; c < 3; ++c) {
      const float L = std::max(rad[3 * p + c], 0.0f);
      accum[3 * p + c] = lerp_f(accum[3 * p + c], L, rate);
      r[c] = L / (L + 1.0f);
    }
    h[30] += 1.0f;
    for (int c = 0; c < 3; ++c) h[(int)std::floor(std::min(r[c], 0.999f) * 10) + 10 * c] += 1.0f;
    const float l = r[0] + r[1] + r[2];
    h[32] = lerp_f(h[32], l, rate);
    h[31] = lerp_f(h[31], l * l, rate);
  }
}

// The interactive neural mode's temporal reuse (RenderCamera<true>,
// core/volume.cu:126-143, with this project's camera inversion): the pixel's
// first-hit point (distance 10 for sky pixels, at least 0.001) is projected
// into the previous camera (prev_ori, prev_up, prev_right; forward =
// normalize(-prev_ori)); the history colour stored there (hist scalars
// total, x, x2) is blended with this frame's radiance at rate 1 / (1 + fnum),
// capped at 0.2 where the ray hit the medium and the checkerboard is off.
// Then ReprojectionDenoise (:266-287) keeps the result as the next history.
// p: this frame's camera and jitter stream (sample_offset = frame index).
void orc_reproject(const mr_render_params* p, const float* prev_ori, const float* prev_up, const float* prev_right,
                   int fnum, int checker, const float* rad, const float* dist, float* hist, float* accum) {
  const int W = p->width, H = p->height;
  const V3 lori = v3(prev_ori[0], prev_ori[1], prev_ori[2]);
  const V3 lup = v3(prev_up[0], prev_up[1], prev_up[2]);
  const V3 lright = v3(prev_right[0], prev_right[1], prev_right[2]);
  const V3 lf = normalize(lori * -1.0f);
  std::vector<float> his((size_t)W * H * 3);
  for (int pix = 0; pix < W * H; ++pix) {
    his[3 * pix] = hist[33 * pix + 30];
    his[3 * pix + 1] = hist[33 * pix + 32];
    his[3 * pix + 2] = hist[33 * pix + 31];
  }
  for (int pix = 0; pix < W * H; ++pix) {
    const int row = pix / W, col = pix - row * W;
    Rng rng(p->seed, (uint32_t)pix, p->sample_offset, TAG_NN);
    const float jx = rng.next(), jy = rng.next();
    const V3 dir = camera_dir(*p, row, col, jx, jy);
    const float d = dist[pix];
    const bool skyp = d < 0.0f;
    const float dis = std::max(0.001f, skyp ? 10.0f : d);
    const V3 mp = f3(p->ori) + dir * dis;
    V3 ld = mp - lori;
    ld = ld / dot(ld, lf);
    ld = ld - lf;
    const float lu = 0.5f - dot(ld, lright) / (2.0f * dot(lright, lright));
    const float lv = 0.5f - dot(ld, lup) / (2.0f * dot(lup, lup));
    const int lx = std::min(W - 1, std::max(0, (int)(lu * W))), ly = std::min(H - 1, std::max(0, (int)(lv * H)));
    const size_t q = (size_t)ly * W + lx;
    float rate = 1.0f / (float)(1 + fnum);
    if (!skyp && !checker) rate = std::min(0.2f, rate);
    for (int c = 0; c < 3; ++c) accum[3 * pix + c] = his[3 * q + c] * (1.0f - rate) + rad[3 * pix + c] * rate;
  }
  for (int pix = 0; pix < W * H; ++pix) {
    hist[33 * pix + 30] = accum[3 * pix];
    hist[33 * pix + 32] = accum[3 * pix + 1];
    hist[33 * pix + 31] = accum[3 * pix + 2];
  }
}

static float hist_compare(const float* x, const float* y) {
  const float nx = x[30], ny = y[30];
  const float syx = std::sqrt(ny / nx), sxy = std::sqrt(nx / ny);
  float p = 0.0f, res = 0.0f;
  for (int i = 0; i < 30; ++i) {
    const float hx = x[i], hy = y[i];
    if (hx != 0.0f || hy != 0.0f) {
      p += 1.0f;
      const float t = syx * hx - sxy * hy;
      res += t * t / (hx + hy);
    }
  }
  return p == 0.0f ? 0.0f : res / p;
}

static V3 mul3(const float* m, V3 x) {
  return v3(m[0] * x.x + m[1] * x.y + m[2] * x.z, m[3] * x.x + m[4] * x.y + m[5] * x.z,
            m[6] * x.x + m[7] * x.y + m[8] * x.z);
}
static V3 gamma22_h(V3 c) {
  return v3(std::pow(std::max(c.x, 0.0f), 1.0f / 2.2f), std::pow(std::max(c.y, 0.0f), 1.0f / 2.2f),
            std::pow(std::max(c.z, 0.0f), 1.0f / 2.2f));
}
static V3 aces_h(V3 c) {
  static const float srgb_ap0[9] = {0.4397010f, 0.3829780f, 0.1773350f, 0.0897923f, 0.8134230f,
                                    0.0967616f, 0.0175440f, 0.1115440f, 0.8707040f};
  static const float ap0_ap1[9] = {1.4514393161f, -0.2365107469f, -0.2149285693f, -0.0765537734f, 1.1762296998f,
                                   -0.0996759264f, 0.0083161484f, -0.0060324498f, 0.9977163014f};
  static const float ap1_xyz[9] = {0.6624541811f, 0.1340042065f, 0.1561876870f, 0.2722287168f, 0.6740817658f,
                                   0.0536895174f, -0.0055746495f, 0.0040607335f, 1.0103391003f};
  static const float xyz_ap1[9] = {1.6410233797f, -0.3248032942f, -0.2364246952f, -0.6636628587f, 1.6153315917f,
                                   0.0167563477f, 0.0117218943f, -0.0082844420f, 0.9883948585f};
  static const float d60_d65[9] = {0.98722400f, -0.00611327f, 0.0159533f, -0.00759836f, 1.00186000f,
                                   0.0053302f, 0.00307257f, -0.00509595f, 1.0816800f};
  static const float xyz_709[9] = {3.2409699419f, -1.5373831776f, -0.4986107603f, -0.9692436363f, 1.8759675015f,
                                   0.0415550574f, 0.0556300797f, -0.2039769589f, 1.0569715142f};
  const V3 ap1_y = v3(0.272229f, 0.674082f, 0.0536895f);
  V3 x = mul3(ap0_ap1, mul3(srgb_ap0, c));
  float y = dot(x, ap1_y);
  x = v3(y, y, y) * (1.0f - 0.96f) + x * 0.96f;
  auto ts = [](float t) { return (t * (t * 278.5085f + 10.7772f)) / (t * (t * 293.6045f + 88.7122f) + 80.6889f); };
  x = v3(ts(x.x), ts(x.y), ts(x.z));
  V3 XYZ = mul3(ap1_xyz, x);
  const float div = std::max(XYZ.x + XYZ.y + XYZ.z, 1e-4f);
  const float cx = XYZ.x / div, cy = XYZ.y / div;
  const float Y = std::pow(std::min(std::max(XYZ.y, 0.0f), 65504.0f), 0.9811f);
  const float m = Y / std::max(cy, 1e-4f);
  x = mul3(xyz_ap1, v3(cx * m, Y, (1.0f - cx - cy) * m));
  y = dot(x, ap1_y);
  x = v3(y, y, y) * (1.0f - 0.93f) + x * 0.93f;
  return gamma22_h(mul3(xyz_709, mul3(d60_d65, mul3(ap1_xyz, x))));
}
static uint32_t pack_h(V3 res, float exposure, int tone) {
  V3 v = res * exposure;
  if (tone == 1) v = gamma22_h(v);
  else if (tone == 2) v = aces_h(v);
  auto q = [](float t) { return (uint32_t)(255.0f * std::min(std::max(t, 0.0f), 1.0f)); };
  return 0xff000000u | (q(v.x) << 16) | (q(v.y) << 8) | q(v.z);
}

// Denoise<denoise> + tone map + pack (core/volume.cu:210-264), row-major.
void orc_denoise(const float* accum, const float* hist, int W, int H, int frame, int flip, int tone, int denoise,
                 float exposure, uint32_t* out) {
  auto at = [&](int r, int c) {
    r = std::min(std::max(r, 0), H - 1);
    c = std::min(std::max(c, 0), W - 1);
    return r * W + c;
  };
  auto col3 = [&](int q) { return v3(accum[3 * q], accum[3 * q + 1], accum[3 * q + 2]); };
  for (int r = 0; r < H; ++r)
    for (int c = 0; c < W; ++c) {
      const int id = r * W + c;
      V3 res;
      if (frame == 0) {
        if ((((r + flip) % 2) + c) % 2 == 0) res = col3(id);
        else res = (col3(at(r - 1, c)) + col3(at(r + 1, c)) + col3(at(r, c - 1)) + col3(at(r, c + 1))) / 4.0f;
      } else {
        const float* h = hist + 33 * id;
        const float variance = std::fabs(h[31] - h[32] * h[32]);
        if (denoise && variance > 0.01f) {
          res = v3(0, 0, 0);
          float ws = 0.0f;
          for (int i = -5; i <= 5; ++i)
            for (int j = -5; j <= 5; ++j) {
              const int t = at(r + i, c + j);
              const float w = std::max(0.0f, 1.0f - 1.2f * hist_compare(h, hist + 33 * t));
              res = res + col3(t) * w;
              ws += w;
            }
          res = res / ws;
        } else {
          res = col3(id);
        }
      }
      out[id] = pack_h(res, exposure, tone);
    }
}

}  // extern "C"
