// Woodcock delta tracking on a raw fp32 density grid: free flight, NEE
// transmittance and the path estimator (core/render.cuh:93-258).
#pragma once
#include "mr_device.cuh"

namespace mr {

struct Medium {
  const float* __restrict__ density;  // res^3, x-major
  int res;
  float max_density;  // global majorant (before alpha)
  float tr_scale;
  cudaTextureObject_t tex;  // layered copy of density read by texture gathers, or 0: texel loads
};

struct TrackStats {
  unsigned fetches;
  unsigned caps;
};

__device__ __forceinline__ float fetch_density(const Medium& m, F3 pos, TrackStats& st) {
  ++st.fetches;
  return m.tex ? tri_border_tex(m.tex, m.res, pos + 0.5f) : tri_border(m.density, m.res, pos + 0.5f);
}

// DeterminateNextVertex (core/render.cuh:138-172).
__device__ __forceinline__ bool next_vertex(const Medium& m, Rng& rng, float alpha, float g, F3 pos, F3 dir,
                                            float dis, F3& npos, F3& ndir, TrackStats& st) {
  float smax = m.max_density * alpha;
  float t = 0;
  int loop = 0;
  bool capped = true;
  while (loop++ < 10000) {
    float rk = rng.next();
    t -= logf(1 - rk) / smax;
    if (t > dis) { npos = f3(0, 0, 0); ndir = f3(0, 0, 0); return false; }
    rk = rng.next();
    float d = fetch_density(m, pos + (dir * t), st);
    float s = d * alpha;
    if (s / smax > rk) { capped = false; break; }
    if (d < 0) t -= d;
  }
  if (capped) ++st.caps;
  float e0 = rng.next();
  float e1 = rng.next();
  ndir = hg_sample_dir(e0, e1, dir, g);
  npos = (dir * t) + pos;
  return true;
}

// Tr (core/render.cuh:93-136): ratio tracking while tr > 0.5, then delta tracking.
__device__ __forceinline__ float transmittance(const Medium& m, Rng& rng, F3 pos, F3 dir, float dis, float alpha,
                                               TrackStats& st) {
  float smax = m.max_density * alpha;
  float tr = 1, t = 0;
  int loop = 0;
  while (loop++ < 10000 && tr > 0.5f) {
    float rk = rng.next();
    t -= logf(1 - rk) / smax * m.tr_scale;
    if (t > dis) break;
    float d = fetch_density(m, pos + (dir * t), st);
    float s = d * alpha;
    tr *= 1 - fmaxf(0.0f, s / smax);
    if (d < 0) t -= d;
  }
  while (loop++ < 10000 && tr > 0.001f) {
    float rk = rng.next();
    t -= logf(1 - rk) / smax * m.tr_scale;
    if (t > dis) break;
    float d = fetch_density(m, pos + (dir * t), st);
    float s = d * alpha;
    if (rng.next() < fmaxf(0.0f, s / smax)) { tr = 0; break; }
    if (d < 0) t -= d;
  }
  if (loop > 10000) ++st.caps;
  return tr;
}

// GetMatrixFromNormal (core/render.cuh:355-369), rejection capped at 64 tries.
__device__ __forceinline__ void frame_from(Rng& rng, F3 v1, F3& a, F3& b, F3& c) {
  v1 = normalize(v1);
  for (int tries = 0; tries < 64; ++tries) {
    float ex = rng.next();
    float ey = rng.next();
    F3 r = uniform_sphere(ex, ey);
    if (fabsf(dot(r, v1)) < 0.01f) continue;
    F3 v2 = normalize(cross(v1, r));
    a = v1; b = v2; c = cross(v2, v1);
    return;
  }
  F3 r = fabsf(v1.x) < 0.5f ? f3(1, 0, 0) : f3(0, 1, 0);
  F3 v2 = normalize(cross(v1, r));
  a = v1; b = v2; c = cross(v2, v1);
}

struct PathScene {
  F3 L;            // normalized light direction
  F3 light_color;
  F3 scatter;      // albedo per channel
  F3 env;          // radiance of escaped rays, or the scale of the environment map
  float alpha, g;
  int max_bounces;
  const float4* env_map;  // SetHDRI image (w x h, row 0 = straight up), or null
  int env_w, env_h;
};

// Environment radiance seen along dir: SkyBox (core/render.cuh:57-61), the
// environment map at u = atan2(-d.z, d.x) / 2 pi + 1/2, v = acos(d.y) / pi,
// bilinear with wrap addressing as the reference's texture filter reads it
// (here in fp32), times the env scale (SetEnvExp); without a map, the
// constant env colour.
__device__ __forceinline__ F3 env_lookup(const float4* __restrict__ map, int w, int h, F3 scale, F3 d) {
  const float u = atan2f(-d.z, d.x) * (float)(0.5 / 3.1415926) + 0.5f;
  const float v = acosf(fmaxf(fminf(d.y, 1.0f), -1.0f)) * (float)(1.0 / 3.1415926);
  const float x = u * (float)w - 0.5f, y = v * (float)h - 0.5f;
  const float x0 = floorf(x), y0 = floorf(y);
  const float fx = x - x0, fy = y - y0;
  int i0 = (int)x0 % w, j0 = (int)y0 % h;
  if (i0 < 0) i0 += w;
  if (j0 < 0) j0 += h;
  const int i1 = i0 + 1 == w ? 0 : i0 + 1, j1 = j0 + 1 == h ? 0 : j0 + 1;
  const float4 a = __ldg(map + (size_t)j0 * w + i0), b = __ldg(map + (size_t)j0 * w + i1);
  const float4 c = __ldg(map + (size_t)j1 * w + i0), e = __ldg(map + (size_t)j1 * w + i1);
  const float r = lerpf(lerpf(a.x, b.x, fx), lerpf(c.x, e.x, fx), fy);
  const float g = lerpf(lerpf(a.y, b.y, fx), lerpf(c.y, e.y, fx), fy);
  const float bl = lerpf(lerpf(a.z, b.z, fx), lerpf(c.z, e.z, fx), fy);
  return f3(r * scale.x, g * scale.y, bl * scale.z);
}
__device__ __forceinline__ F3 sky(const PathScene& sc, F3 d) {
  return sc.env_map ? env_lookup(sc.env_map, sc.env_w, sc.env_h, sc.env, d) : sc.env;
}

// CalculateRadiance (core/render.cuh:200-258), one sample.
__device__ __forceinline__ F3 path_radiance(const Medium& m, const PathScene& sc, Rng& rng, F3 ori, F3 dir,
                                            float* first_t, TrackStats& st) {
  dir = normalize(dir);
  float t = -1;
  float dis = ray_box_offset(ori, dir);
  if (dis < 0) { *first_t = t; return sky(sc, dir); }
  F3 res = f3(0, 0, 0);
  F3 pos = ori + dir * dis;
  F3 rd = dir;
  F3 rate = f3(1, 1, 1);
  for (int s = 0; s < sc.max_bounces; ++s) {
    F3 np, nd;
    float maxd = ray_box_distance(pos, rd);
    bool hit = next_vertex(m, rng, sc.alpha, sc.g, pos, rd, maxd, np, nd, st);
    if (!hit) { res = res + sky(sc, rd) * rate; break; }
    if (s == 0) t = length(ori - np);
    pos = np;
    rate = rate * sc.scatter;
    maxd = ray_box_distance(pos, sc.L);
    float ph = hg_phase(dot(rd, sc.L), sc.g);
    res = res + (sc.light_color * rate) * (transmittance(m, rng, pos, sc.L, maxd, sc.alpha, st) * ph);
    rd = nd;
  }
  *first_t = t;
  return res;
}

struct CameraModel {
  F3 ori, fwd, up, right;
  int width, height;
};

// Camera ray of pixel (row, col) (core/volume.cu:155-163, row-major W x H).
__device__ __forceinline__ F3 camera_dir(const CameraModel& c, int row, int col, float jx, float jy) {
  float u = 1.0f - ((float)col + jx) / (float)c.width;
  float v = 1.0f - ((float)row + jy) / (float)c.height;
  F3 d = c.fwd + (c.right * (u * 2 - 1)) + (c.up * (v * 2 - 1));
  return normalize(d);
}

// Warp-aggregated claim of one work item per calling lane.
__device__ __forceinline__ unsigned long long claim_work(unsigned long long* counter) {
  unsigned mask = __activemask();
  int lane = threadIdx.x & 31;
  int leader = __ffs(mask) - 1;
  unsigned lt = mask & ((1u << lane) - 1u);
  unsigned long long base = 0;
  if (lane == leader) base = atomicAdd(counter, (unsigned long long)__popc(mask));
  base = __shfl_sync(mask, base, leader);
  return base + __popc(lt);
}

}  // namespace mr
