// Neural render (render type MRPNN): NNPredict<MRPNN> of
// core/render.cuh:469-523 split into three stream-ordered kernels.
//  1. k_nn_trace: per pixel, camera ray + first Woodcock collision
//     (GetSamplePoint), the two random frames (GetMatrixFromNormal) and the
//     single-scatter NEE term Tr*HG; active pixels are compacted into a record
//     list with warp-aggregated atomics, inactive ones get the environment.
//  2. k_gather_fm: per active record, the 192-point multi-scale descriptor
//     gather (core/radiancePredict.cu:319-368) into feature-major columns.
//  3. the network body: k_simt_trunk, k_light_trunk, k_tc32_head and
//     k_tc32_tail (fp32, mr_mlp_simt.cu) or k_mlp_tc (BF16 / E4M3 tcgen05,
//     mr_mlp_tc.cu); the last kernel also writes the pixel.
// The gather's per-point table (k_sphere_h0) runs on a side stream beside
// the trace.
#include <algorithm>
#include <mutex>
#include <vector>

#include "mr_internal.h"
#include "mr_net_layout.cuh"
#include "mr_track.cuh"

namespace mr {

struct Tables {
  const float* __restrict__ mips;
  const float* __restrict__ tr;
  const float* __restrict__ lut;
  // texture-unit copies (MR_SAMPLER_TEXTURE only)
  cudaTextureObject_t mip_tex[9], tr_tex[8], lut_tex;
  // layered copies read by texture gathers (exact sampler, kSampGather)
  cudaTextureObject_t mip_g[9], tr_g[8], lut_g;
};

// Sampler forms of the descriptor gather: the fp32 software filter over
// texel loads; the texture units' trilinear filter for the 3-D tables
// (MR_SAMPLER_TEXTURE); and the fp32 software filter over texture gathers for
// the 3-D tables (same values as the loads: the default form of
// MR_SAMPLER_EXACT). Both texture forms keep the texture data path busy (78 %
// of its peak while active in the exact form), so both read the 2-D HG table
// with texel loads and the fp32 bilinear filter, off that path: 15 % less
// gather time for the exact form, 13 % for the texture form.
enum { kSampLoad = 0, kSampTex = 1, kSampGather = 2 };

__constant__ unsigned c_mip_off[9] = {0u, 16777216u, 18874368u, 19136512u, 19169280u, 19173376u, 19173888u,
                                      19173952u, 19173960u};
__constant__ unsigned c_tr_off[8] = {0u, 2097152u, 2359296u, 2392064u, 2396160u, 2396672u, 2396736u, 2396744u};

__device__ __forceinline__ float mip_density(const Tables& t, int mip, F3 p) {
  return tri_border(t.mips + c_mip_off[mip], 256 >> mip, p + 0.5f);
}
__device__ __forceinline__ float mip_tr(const Tables& t, int mip, F3 p) {
  return tri_clamp(t.tr + c_tr_off[mip], 128 >> mip, p + 0.5f);
}
// ShadowTerm_TRTex (core/renderResources.cu:121-139), light colour 1.
__device__ __forceinline__ float shadow_tr(const Tables& t, F3 p, F3 L, int mip) {
  if (p.x < -0.5f || p.y < -0.5f || p.z < -0.5f || p.x > 0.5f || p.y > 0.5f || p.z > 0.5f) {
    float off = ray_box_offset(p, L);
    if (off >= 0) return mip_tr(t, mip, p + L * off);
    return 1.0f;
  }
  return mip_tr(t, mip, p);
}

struct Frame { F3 X, Y, Z, LX; };

// Active-pixel record written by the trace kernel (SoA for coalescing).
struct Records {
  int* pix;        // n
  float* pos;      // 3n
  float* frame;    // 12n: X, Y, Z, LX
  float* trph;     // n
  unsigned* count; // 1
  int* job;        // n, batched renders only (null otherwise)
};

struct NNTraceArgs {
  Medium m;
  PathScene sc;
  CameraModel cam;
  uint32_t seed, frame_index;
  float* out;
  float* dist;  // optional first-hit distance per pixel (< 0: escaped), interactive reprojection
  Records rec;
  unsigned long long* counters;
};

// Warp-aggregated slot allocation in a 32-bit counter.
__device__ __forceinline__ unsigned claim_slot(unsigned* counter) {
  unsigned mask = __activemask();
  int lane = threadIdx.x & 31;
  int leader = __ffs(mask) - 1;
  unsigned base = 0;
  if (lane == leader) base = atomicAdd(counter, (unsigned)__popc(mask));
  base = __shfl_sync(mask, base, leader);
  return base + __popc(mask & ((1u << lane) - 1u));
}

// One pixel of NNPredict's first half: returns 1 when the pixel became an
// active record (job = its batch job, -1 for a single render).
__device__ __forceinline__ unsigned trace_pixel(const Medium& m, const PathScene& sc, const CameraModel& cam,
                                                uint32_t seed, uint32_t frame_index, int pix, float* out,
                                                float* dist, const Records& rec, int job, TrackStats& st) {
  int row = pix / cam.width, col = pix - row * cam.width;
  Rng rng;
  rng.init(seed, (uint32_t)pix, frame_index, TAG_NN);
  float jx = rng.next(), jy = rng.next();
  F3 dir = camera_dir(cam, row, col, jx, jy);
  // GetSamplePoint (core/render.cuh:174-198)
  bool active = false;
  F3 pos = f3(0, 0, 0);
  float dis = ray_box_offset(cam.ori, dir);
  if (dis >= 0) {
    F3 sp = cam.ori + dir * dis;
    float maxd = ray_box_distance(sp, dir);
    F3 p0, p1;
    active = next_vertex(m, rng, sc.alpha, 0.0f, sp, dir, maxd, p0, p1, st);
    if (active) pos = p0;
  }
  Frame f;
  F3 ly, lz;
  frame_from(rng, dir, f.X, f.Y, f.Z);
  frame_from(rng, sc.L, f.LX, ly, lz);
  if (dist) dist[pix] = active ? length(cam.ori - pos) : -1.0f;
  if (!active) {
    const F3 e = sky(sc, dir);  // SkyBox(dir) for pixels that see no medium
    out[3 * (size_t)pix + 0] = fmaxf(e.x, 0.0f);
    out[3 * (size_t)pix + 1] = fmaxf(e.y, 0.0f);
    out[3 * (size_t)pix + 2] = fmaxf(e.z, 0.0f);
    return 0;
  }
  float d2 = ray_box_distance(pos, f.LX);
  float ph = hg_phase(dot(f.X, f.LX), sc.g);
  float tr = transmittance(m, rng, pos, f.LX, d2, sc.alpha, st) * ph;
  unsigned k = claim_slot(rec.count);
  rec.pix[k] = pix;
  if (rec.job) rec.job[k] = job;
  rec.pos[3 * (size_t)k + 0] = pos.x;
  rec.pos[3 * (size_t)k + 1] = pos.y;
  rec.pos[3 * (size_t)k + 2] = pos.z;
  float* fr = rec.frame + 12 * (size_t)k;
  fr[0] = f.X.x; fr[1] = f.X.y; fr[2] = f.X.z;
  fr[3] = f.Y.x; fr[4] = f.Y.y; fr[5] = f.Y.z;
  fr[6] = f.Z.x; fr[7] = f.Z.y; fr[8] = f.Z.z;
  fr[9] = f.LX.x; fr[10] = f.LX.y; fr[11] = f.LX.z;
  rec.trph[k] = tr;
  return 1;
}

__device__ __forceinline__ void trace_counters(unsigned long long* counters, const TrackStats& st, unsigned act) {
  unsigned fsum = st.fetches, csum = st.caps;
  for (int o = 16; o; o >>= 1) {
    fsum += __shfl_xor_sync(0xffffffffu, fsum, o);
    csum += __shfl_xor_sync(0xffffffffu, csum, o);
    act += __shfl_xor_sync(0xffffffffu, act, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(counters + 0, (unsigned long long)fsum);
    if (csum) atomicAdd(counters + 2, (unsigned long long)csum);
    atomicAdd(counters + 3, (unsigned long long)act);
  }
}

// Bound by the latency of dependent density fetches: registers capped for
// twelve 128-thread blocks per SM.
__global__ void __launch_bounds__(128, 12) k_nn_trace(NNTraceArgs a) {
  int pix = blockIdx.x * blockDim.x + threadIdx.x;
  int npx = a.cam.width * a.cam.height;
  TrackStats st{0, 0};
  unsigned act = 0;
  if (pix < npx) act = trace_pixel(a.m, a.sc, a.cam, a.seed, a.frame_index, pix, a.out, a.dist, a.rec, -1, st);
  trace_counters(a.counters, st, act);
}

// ---- marching variant (NNPredict<Type::marching_MRPNN>, core/render.cuh:524-633) ----
// The camera ray is marched in fixed steps (1/1023 of the ray's box length,
// longer where a negative density gives a distance to skip); the network's
// point is drawn among the marched samples with weight T (1 - exp(-sigma dt))
// by reservoir sampling. With a surface IOR > 0 the first positive sample is
// a dielectric surface (normal from the negative-density field): its GGX
// specular term lit through Tr is kept, and the ray continues reflected or
// refracted with the Fresnel probability. The pixel is
// ref + lerp((network + Tr * phase) * light, sky(dir), T_end).

// Normal (core/render.cuh:371-387): central differences of max(0, -density),
// the step widened by 0.01 (up to 10 times) while the gradient is zero.
__device__ __forceinline__ F3 surface_normal(const Medium& m, F3 p, TrackStats& st) {
  float dl = 0.02f;
  F3 n;
  int left = 10;
  do {
    auto neg = [&](F3 q) { return fmaxf(0.0f, -fetch_density(m, q, st)); };
    n = f3(neg(p + f3(dl, 0, 0)) - neg(p - f3(dl, 0, 0)), neg(p + f3(0, dl, 0)) - neg(p - f3(0, dl, 0)),
           neg(p + f3(0, 0, dl)) - neg(p - f3(0, 0, dl)));
    dl += 0.01f;
  } while (n.x == 0.0f && n.y == 0.0f && n.z == 0.0f && left-- > 0);
  return normalize(n);
}
__device__ __forceinline__ float sat(float x) { return fminf(fmaxf(x, 0.0f), 1.0f); }
// GGX distribution (GGXTerm, :389-395).
__device__ __forceinline__ float ggx_d(float nh, float rough) {
  const float a2 = rough * rough;
  const float d = (nh * a2 - nh) * nh + 1.0f;
  return 0.318309886183790671538f * a2 / (d * d + 1e-7f);
}
// Smith joint visibility (SmithJointGGXVisibilityTerm, :400-404).
__device__ __forceinline__ float smith_v(float nl, float nv, float rough) {
  const float k = (rough + 0.01f) * (rough + 0.01f) / 1.01f / 1.01f / 2.0f;
  return (1e-5f + nl * nv) / (1e-5f + lerpf(nl, 1.0f, k) * lerpf(nv, 1.0f, k));
}
// Unpolarised dielectric Fresnel reflectance (PhysicsFresnel, :410-419).
__device__ __forceinline__ float fresnel_dielectric(float ior, F3 i, F3 n) {
  const float ci = fabsf(dot(i, n));
  const float si = sqrtf(fmaxf(0.0f, 1.0f - ci * ci));
  const float st = si / ior;
  const float ct = sqrtf(fmaxf(0.0f, 1.0f - st * st));
  const float r1 = (ior * ci - ct) / (ior * ci + ct);
  const float r2 = (ci - ior * ct) / (ci + ior * ct);
  return (r1 * r1 + r2 * r2) / 2.0f;
}
// Specular BRDF * n.l (Schlick Fresnel from F0 = 0.04, GGX, Smith; roughness
// 0.008) and, in .w, the dielectric reflectance (BRDF, :428-461).
__device__ __forceinline__ float4 surface_brdf(F3 n, F3 v, F3 l, float ior) {
  const F3 h = normalize(l + v);
  const float shift = dot(n, v);
  if (shift < 0.0f) n = n + v * (-shift + 1e-5f);
  const float nv = sat(dot(n, v)), nl = sat(dot(n, l)), nh = sat(dot(n, h)), lh = sat(dot(l, h));
  const float rough = 0.008f;
  const float D = ggx_d(nh, rough);
  const float G = smith_v(nl, nv, rough) * 3.1415926f;
  const float t = 1.0f - lh;
  const float F = 0.04f + (1.0f - 0.04f) * (t * t * t * t * t);
  const float dfg = F * G * D * nl;
  return make_float4(dfg, dfg, dfg, fresnel_dielectric(ior, v, n));
}
__device__ __forceinline__ F3 refract_dir(F3 i, F3 n, float eta) {
  const float ci = dot(i * -1.0f, n);
  const float c2 = 1.0f - eta * eta * (1.0f - ci * ci);
  const F3 t = i * eta + n * (eta * ci - sqrtf(fabsf(c2)));
  return t * (c2 > 0.0f ? 1.0f : 0.0f);
}
__device__ __forceinline__ F3 reflect_dir(F3 i, F3 n) { return i - n * (dot(i, n) * 2.0f); }

struct MarchArgs {
  Medium m;
  PathScene sc;
  CameraModel cam;
  uint32_t seed, frame_index;
  float ior;
  float* out;
  Records rec;
  float4* madd;  // per record: xyz = ref + sky * T_end, w = 1 - T_end
  unsigned long long* counters;
};

constexpr int kMarchSteps = 1024;

__global__ void __launch_bounds__(128) k_march_trace(MarchArgs a) {
  const int pix = blockIdx.x * blockDim.x + threadIdx.x;
  const int npx = a.cam.width * a.cam.height;
  TrackStats st{0, 0};
  unsigned act = 0;
  if (pix < npx) {
    const PathScene& sc = a.sc;
    const int row = pix / a.cam.width, col = pix - row * a.cam.width;
    Rng rng;
    rng.init(a.seed, (uint32_t)pix, a.frame_index, TAG_NN);
    const float jx = rng.next(), jy = rng.next();
    F3 dir = camera_dir(a.cam, row, col, jx, jy);
    Frame f;
    F3 ly, lz;
    frame_from(rng, dir, f.X, f.Y, f.Z);
    frame_from(rng, sc.L, f.LX, ly, lz);
    const float offset = ray_box_offset(a.cam.ori, dir);
    bool go = offset >= 0.0f;
    F3 ori = a.cam.ori + dir * offset;
    float dis = ray_box_distance(ori, dir);
    float inv = dis / (float)(kMarchSteps - 1);
    float trans = 1.0f, t = 0.0f, hit_dis = -1.0f, total_w = 0.0f;
    bool surfaced = !(a.ior > 0.0f);
    F3 ref = f3(0, 0, 0), pos = f3(0, 0, 0);
    for (int step = 0; go; ++step) {
      if (trans < 0.005f || t >= dis || step > kMarchSteps * 2) break;
      const F3 sp = ori + dir * t;
      const float vd = fetch_density(a.m, sp, st);
      if (vd > 0.0f && hit_dis == -1.0f) hit_dis = offset + t;
      t += fmaxf(inv, -vd);
      if (vd <= 0.0f) continue;
      if (!surfaced) {
        F3 n = surface_normal(a.m, sp, st);
        n = n - dir * fmaxf(0.0f, dot(n, dir) + 0.01f);
        const float4 b = surface_brdf(n, dir * -1.0f, sc.L, a.ior);
        const float ldis = ray_box_distance(sp, sc.L);
        const float tr = transmittance(a.m, rng, sp, sc.L, ldis, sc.alpha, st);
        ref = f3(b.x, b.y, b.z) * tr * sc.light_color;
        dir = rng.next() < b.w ? reflect_dir(dir, n) : refract_dir(dir, n, 1.0f / a.ior);
        ori = sp;
        t = 0.0f;
        dis = ray_box_distance(ori, dir);
        inv = dis / (float)(kMarchSteps - 1);
        frame_from(rng, dir, f.X, f.Y, f.Z);
        frame_from(rng, sc.L, f.LX, ly, lz);
        surfaced = true;
      }
      const float tr_step = expf(-vd * sc.alpha * inv);
      const float w = trans * (1.0f - tr_step);
      total_w += w;
      if (rng.next() < w / total_w) pos = sp;
      trans *= tr_step;
    }
    const F3 skyc = sky(sc, dir);
    if (hit_dis < 0.0f) {
      const F3 o = ref + skyc;
      a.out[3 * (size_t)pix] = fmaxf(o.x, 0.0f);
      a.out[3 * (size_t)pix + 1] = fmaxf(o.y, 0.0f);
      a.out[3 * (size_t)pix + 2] = fmaxf(o.z, 0.0f);
    } else {
      const float d2 = ray_box_distance(pos, f.LX);
      const float ph = hg_phase(dot(f.X, f.LX), sc.g);
      const float tr = transmittance(a.m, rng, pos, f.LX, d2, sc.alpha, st) * ph;
      const unsigned k = claim_slot(a.rec.count);
      a.rec.pix[k] = pix;
      a.rec.pos[3 * (size_t)k + 0] = pos.x;
      a.rec.pos[3 * (size_t)k + 1] = pos.y;
      a.rec.pos[3 * (size_t)k + 2] = pos.z;
      float* fr = a.rec.frame + 12 * (size_t)k;
      fr[0] = f.X.x; fr[1] = f.X.y; fr[2] = f.X.z;
      fr[3] = f.Y.x; fr[4] = f.Y.y; fr[5] = f.Y.z;
      fr[6] = f.Z.x; fr[7] = f.Z.y; fr[8] = f.Z.z;
      fr[9] = f.LX.x; fr[10] = f.LX.y; fr[11] = f.LX.z;
      a.rec.trph[k] = tr;
      const F3 add = ref + skyc * trans;
      a.madd[k] = make_float4(add.x, add.y, add.z, 1.0f - trans);
      act = 1;
    }
  }
  trace_counters(a.counters, st, act);
}

// out = ref + sky * T + (network + Tr * phase) * light * (1 - T) for the
// marching records (the network wrote (network + Tr * phase) * light).
__global__ void k_march_compose(const unsigned* __restrict__ count, const int* __restrict__ pix,
                                const float4* __restrict__ madd, float* __restrict__ out) {
  const unsigned k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= *count) return;
  const float4 m = madd[k];
  float* o = out + 3 * (size_t)pix[k];
  o[0] = fmaxf(m.x + o[0] * m.w, 0.0f);
  o[1] = fmaxf(m.y + o[1] * m.w, 0.0f);
  o[2] = fmaxf(m.z + o[2] * m.w, 0.0f);
}

inline __device__ Frame load_frame(const float* fr) {
  Frame f;
  f.X = f3(fr[0], fr[1], fr[2]);
  f.Y = f3(fr[3], fr[4], fr[5]);
  f.Z = f3(fr[6], fr[7], fr[8]);
  f.LX = f3(fr[9], fr[10], fr[11]);
  return f;
}


// ---- specialised gather ---------------------------------------------------------
// The 192 stencil points fall into 12 segments of constant mip level and
// offset (core/vector.cu:299-400). Per segment, the level's resolution and
// table base are compile-time constants and the HG-table row v (from the cone
// angle) is computed once. For a sphere point p - pos = off * (X s.x + Y s.y
// + Z s.z) with an orthonormal frame, so the cone cosines are
// dot(X, md) = s.x/|s| and dot(LX, md) = (LX.X s.x + LX.Y s.y + LX.Z s.z)/|s|;
// for a light-direction point md = L. Same arithmetic as gather_sink up to
// rounding.
template <int RES>
__device__ __forceinline__ float tri_border_c(const float* __restrict__ d, F3 uv) {
  float px = uv.x * RES - 0.5f, py = uv.y * RES - 0.5f, pz = uv.z * RES - 0.5f;
  float fx = floorf(px), fy = floorf(py), fz = floorf(pz);
  int x = (int)fx, y = (int)fy, z = (int)fz;
  float wx = px - fx, wy = py - fy, wz = pz - fz;
  bool x0 = (unsigned)x < (unsigned)RES, x1 = (unsigned)(x + 1) < (unsigned)RES;
  bool y0 = (unsigned)y < (unsigned)RES, y1 = (unsigned)(y + 1) < (unsigned)RES;
  bool z0 = (unsigned)z < (unsigned)RES, z1 = (unsigned)(z + 1) < (unsigned)RES;
  const float* b = d + (x * RES + y) * RES + z;  // 32-bit index: RES^3 < 2^31
  float c000 = (x0 && y0 && z0) ? __ldg(b) : 0.0f;
  float c001 = (x0 && y0 && z1) ? __ldg(b + 1) : 0.0f;
  float c010 = (x0 && y1 && z0) ? __ldg(b + RES) : 0.0f;
  float c011 = (x0 && y1 && z1) ? __ldg(b + RES + 1) : 0.0f;
  float c100 = (x1 && y0 && z0) ? __ldg(b + RES * RES) : 0.0f;
  float c101 = (x1 && y0 && z1) ? __ldg(b + RES * RES + 1) : 0.0f;
  float c110 = (x1 && y1 && z0) ? __ldg(b + RES * RES + RES) : 0.0f;
  float c111 = (x1 && y1 && z1) ? __ldg(b + RES * RES + RES + 1) : 0.0f;
  return lerpf(lerpf(lerpf(c000, c001, wz), lerpf(c010, c011, wz), wy),
               lerpf(lerpf(c100, c101, wz), lerpf(c110, c111, wz), wy), wx);
}
template <int RES>
__device__ __forceinline__ float tri_clamp_c(const float* __restrict__ d, F3 uv) {
  float px = uv.x * RES - 0.5f, py = uv.y * RES - 0.5f, pz = uv.z * RES - 0.5f;
  float fx = floorf(px), fy = floorf(py), fz = floorf(pz);
  int x = (int)fx, y = (int)fy, z = (int)fz;
  float wx = px - fx, wy = py - fy, wz = pz - fz;
  int xa = min(max(x, 0), RES - 1), xb = min(max(x + 1, 0), RES - 1);
  int ya = min(max(y, 0), RES - 1), yb = min(max(y + 1, 0), RES - 1);
  int za = min(max(z, 0), RES - 1), zb = min(max(z + 1, 0), RES - 1);
  const int ra = xa * RES * RES, rb = xb * RES * RES, sa = ya * RES, sb = yb * RES;
  float c000 = __ldg(d + ra + sa + za), c001 = __ldg(d + ra + sa + zb);
  float c010 = __ldg(d + ra + sb + za), c011 = __ldg(d + ra + sb + zb);
  float c100 = __ldg(d + rb + sa + za), c101 = __ldg(d + rb + sa + zb);
  float c110 = __ldg(d + rb + sb + za), c111 = __ldg(d + rb + sb + zb);
  return lerpf(lerpf(lerpf(c000, c001, wz), lerpf(c010, c011, wz), wy),
               lerpf(lerpf(c100, c101, wz), lerpf(c110, c111, wz), wy), wx);
}

// tri_border_c / tri_clamp_c / bilinear_clamp over texture gathers: two
// footprints (layers x and x+1) per trilinear sample, one per bilinear.
// Same corner values and the same fp32 arithmetic.
template <int RES>
__device__ __forceinline__ float tri_border_g(cudaTextureObject_t t, F3 uv) {
  float px = uv.x * RES - 0.5f, py = uv.y * RES - 0.5f, pz = uv.z * RES - 0.5f;
  float fx = floorf(px), fy = floorf(py), fz = floorf(pz);
  int x = (int)fx;
  float wx = px - fx, wy = py - fy, wz = pz - fz;
  const float4 z4 = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  const float4 a = (unsigned)x < (unsigned)RES ? gather_a2d(t, x, fz, fy) : z4;
  const float4 b = (unsigned)(x + 1) < (unsigned)RES ? gather_a2d(t, x + 1, fz, fy) : z4;
  return lerpf(lerpf(lerpf(a.x, a.y, wz), lerpf(a.z, a.w, wz), wy),
               lerpf(lerpf(b.x, b.y, wz), lerpf(b.z, b.w, wz), wy), wx);
}
template <int RES>
__device__ __forceinline__ float tri_clamp_g(cudaTextureObject_t t, F3 uv) {
  float px = uv.x * RES - 0.5f, py = uv.y * RES - 0.5f, pz = uv.z * RES - 0.5f;
  float fx = floorf(px), fy = floorf(py), fz = floorf(pz);
  int x = (int)fx;
  float wx = px - fx, wy = py - fy, wz = pz - fz;
  const float4 a = gather_a2d(t, min(max(x, 0), RES - 1), fz, fy);
  const float4 b = gather_a2d(t, min(max(x + 1, 0), RES - 1), fz, fy);
  return lerpf(lerpf(lerpf(a.x, a.y, wz), lerpf(a.z, a.w, wz), wy),
               lerpf(lerpf(b.x, b.y, wz), lerpf(b.z, b.w, wz), wy), wx);
}
__device__ __forceinline__ float bilinear_clamp_g(cudaTextureObject_t t, int w, int h, float u, float v) {
  float px = u * w - 0.5f, py = v * h - 0.5f;
  float fx = floorf(px), fy = floorf(py);
  float wx = px - fx, wy = py - fy;
  const float4 c = gather_2d(t, fx, fy);
  float a = lerpf(c.x, c.y, wx);
  float b = lerpf(c.z, c.w, wx);
  return lerpf(a, b, wy);
}

struct PixelGather {
  F3 pos, L, X, Y, Z, LX;
  float lx, ly, lz;   // LX in the (X, Y, Z) frame
  float cXL, cLXL;    // cone cosines of the light-direction points
  float alpha, hg0;
};

constexpr unsigned kMipOff[9] = {0u, 16777216u, 18874368u, 19136512u, 19169280u, 19173376u, 19173888u, 19173952u,
                                 19173960u};
constexpr unsigned kTrOff[8] = {0u, 2097152u, 2359296u, 2392064u, 2396160u, 2396672u, 2396736u, 2396744u};

// Stencil points [I0, I1) at mip level MIP, offset `off` (sphere points), or
// the light-direction points with per-point offsets (SPHERE = false). HW
// samples through the texture units instead of the fp32 software filter.
// Bilinear HG-table sample in sampler form SAMP.
template <int SAMP>
__device__ __forceinline__ float lut_sample(const Tables& t, float u, float v) {
  if (SAMP == kSampTex) return bilinear_clamp(t.lut, kLut, kLut, u, v);  // texel loads, see kSampGather
  if (SAMP == kSampGather) return bilinear_clamp(t.lut, kLut, kLut, u, v);  // texel loads, see kSampGather
  return bilinear_clamp(t.lut, kLut, kLut, u, v);
}

// Per-point constants of the gather, the same for every pixel (kPtTable
// floats): [0, 192) the first HG-table factor of each sphere point (it
// depends only on the stencil point - the cone cosine dot(X, md) = s.x / |s|
// in an orthonormal frame - and the segment's table row), [192, 384) the
// table row v of every point (atan(radius / 2 off) / 60 degrees). Segment
// [I0, I1) by the block's threads; SPHERE = false: light-direction points
// with per-point offsets (1..8, 9.5.., 26.5.., 60.5..)/256
// (core/vector.cu:367-398).
constexpr int kPtTable = 384;
template <int MIP, bool SPHERE, int SAMP, int I0, int I1>
__device__ __forceinline__ void point_table_seg(const Tables& t, const float* __restrict__ stencil, float off,
                                                float* tab) {
  const float radius = (float)(1 << MIP) / 256.0f;
  const float kAng = 3.1415926535f * 60.0f / 180.0f;
  for (int i = I0 + (int)threadIdx.x; i < I1; i += (int)blockDim.x) {
    if (SPHERE) {
      const float vrow = atanf(0.5f * radius / off) / kAng;
      const float sx = __ldg(stencil + 3 * i), sy = __ldg(stencil + 3 * i + 1), sz = __ldg(stencil + 3 * i + 2);
      const float inv = rsqrtf(sx * sx + sy * sy + sz * sz);
      const float c1 = sx * inv;
      tab[i] = lut_sample<SAMP>(t, c1 * 0.5f + 0.5f, vrow);
      tab[192 + i] = vrow;
    } else {
      const int j = i - I0;
      const float o = (MIP == 0 ? (float)(j + 1) : MIP == 1 ? 8.5f + 1.0f + 2.0f * (float)j
                                 : MIP == 2 ? 26.5f + 4.0f * (float)j : 60.5f + 8.0f * (float)j) / 256.0f;
      tab[i] = 0.0f;
      tab[192 + i] = atanf(0.5f * radius / o) / kAng;
    }
  }
}

template <int MIP, bool SPHERE, int SAMP, int I0, int I1, class Sink>
__device__ __forceinline__ void gather_seg(const Tables& t, const float* __restrict__ stencil, const PixelGather& q,
                                           float off, const float* h0s, Sink& sink) {
  constexpr int R = 256 >> MIP;
  constexpr int TL = MIP > 0 ? MIP - 1 : 0;
  constexpr int RT = 128 >> TL;
  const float* mb = t.mips + kMipOff[MIP];
  const float* tb = t.tr + kTrOff[TL];
  const float radius = (float)(1 << MIP) / 256.0f;
  const float kAng = 3.1415926535f * 60.0f / 180.0f;
  float vrow = h0s ? h0s[192 + I0] : atanf(0.5f * radius / off) / kAng;
  static_assert(I0 % 4 == 0 && I1 % 4 == 0, "segments are whole 4-feature chunks");
#pragma unroll 1
  for (int i0 = I0; i0 < I1; i0 += 4)
#pragma unroll
  for (int u = 0; u < 4; ++u) {
    const int i = i0 + u;
    F3 p;
    float c1, c2;
    if (SPHERE) {
      const float sx = __ldg(stencil + 3 * i), sy = __ldg(stencil + 3 * i + 1), sz = __ldg(stencil + 3 * i + 2);
      p = q.pos + ((q.X * sx + q.Y * sy + q.Z * sz) * off);
      const float inv = rsqrtf(sx * sx + sy * sy + sz * sz);
      c1 = sx * inv;
      c2 = (q.lx * sx + q.ly * sy + q.lz * sz) * inv;
    } else {
      // light-direction points: offsets (1..8, 9.5.., 26.5.., 60.5..)/256 per
      // point (core/vector.cu:367-398)
      const int j = i - I0;
      off = (MIP == 0 ? (float)(j + 1) : MIP == 1 ? 8.5f + 1.0f + 2.0f * (float)j
                                       : MIP == 2 ? 26.5f + 4.0f * (float)j : 60.5f + 8.0f * (float)j) / 256.0f;
      vrow = h0s ? h0s[192 + i] : atanf(0.5f * radius / off) / kAng;
      p = q.pos + q.L * off;
      c1 = q.cXL;
      c2 = q.cLXL;
    }
    const float dens = SAMP == kSampTex      ? tex3D<float>(t.mip_tex[MIP], p.z + 0.5f, p.y + 0.5f, p.x + 0.5f)
                       : SAMP == kSampGather ? tri_border_g<R>(t.mip_g[MIP], p + 0.5f)
                                             : tri_border_c<R>(mb, p + 0.5f);
    const float xv = __logf(1.0f + q.alpha * dens / 64.0f);
    float xh;
    if (SPHERE && MIP == 0 && I0 == 0 && i == 0) {
      xh = q.hg0;
    } else {
      const float u1 = c1 * 0.5f + 0.5f, u2 = c2 * 0.5f + 0.5f;
      const float h0 = SPHERE && h0s ? h0s[i] : lut_sample<SAMP>(t, u1, vrow);
      const float h1 = lut_sample<SAMP>(t, u2, vrow);
      xh = __logf(h0 * h1 + 1.0f);
    }
    F3 pt = p;
    float xs = 1.0f;
    bool fetch = true;
    if (p.x < -0.5f || p.y < -0.5f || p.z < -0.5f || p.x > 0.5f || p.y > 0.5f || p.z > 0.5f) {
      const float o2 = ray_box_offset(p, q.LX);  // ShadowTerm_TRTex (core/renderResources.cu:121-139)
      fetch = o2 >= 0;
      pt = p + q.LX * o2;
    }
    if (fetch)
      xs = SAMP == kSampTex      ? tex3D<float>(t.tr_tex[TL], pt.z + 0.5f, pt.y + 0.5f, pt.x + 0.5f)
           : SAMP == kSampGather ? tri_clamp_g<RT>(t.tr_g[TL], pt + 0.5f)
                                 : tri_clamp_c<RT>(tb, pt + 0.5f);
    sink(i, u, xv, xs, xh);
  }
}

// The per-point table (see point_table_seg), with the segment offsets of
// gather_fast.
template <int SAMP>
__device__ __forceinline__ void point_table(const Tables& t, const float* __restrict__ stencil, float* tab) {
  const float ms = 0.6f;
  point_table_seg<0, true, SAMP, 0, 8>(t, stencil, 1.0f / 256.0f * lerpf(ms, 1.0f, 1.0f), tab);
  point_table_seg<1, true, SAMP, 8, 16>(t, stencil, 2.5f / 256.0f * lerpf(ms, 1.0f, 0.8f), tab);
  point_table_seg<2, true, SAMP, 16, 32>(t, stencil, 5.5f / 256.0f * lerpf(ms, 1.0f, 0.6f), tab);
  point_table_seg<3, true, SAMP, 32, 48>(t, stencil, 11.5f / 256.0f * lerpf(ms, 1.0f, 0.4f), tab);
  point_table_seg<4, true, SAMP, 48, 64>(t, stencil, 23.5f / 256.0f * lerpf(ms, 1.0f, 0.2f), tab);
  point_table_seg<5, true, SAMP, 64, 96>(t, stencil, 47.5f / 256.0f * ms, tab);
  point_table_seg<6, true, SAMP, 96, 128>(t, stencil, 95.5f / 256.0f * ms, tab);
  point_table_seg<7, true, SAMP, 128, 160>(t, stencil, 191.5f / 256.0f * ms, tab);
  point_table_seg<0, false, SAMP, 160, 168>(t, stencil, 1.0f, tab);
  point_table_seg<1, false, SAMP, 168, 176>(t, stencil, 1.0f, tab);
  point_table_seg<2, false, SAMP, 176, 184>(t, stencil, 1.0f, tab);
  point_table_seg<3, false, SAMP, 184, 192>(t, stencil, 1.0f, tab);
}

// The table, once per render (one block), into h0s[kPtTable].
template <int SAMP>
__global__ void k_sphere_h0(Tables t, const float* __restrict__ stencil, float* __restrict__ h0s) {
  point_table<SAMP>(t, stencil, h0s);
}

// h0s: the per-point table (k_sphere_h0), or null to compute its entries per
// point.
template <int SAMP, class Sink>
__device__ __forceinline__ void gather_fast(const Tables& t, const float* __restrict__ stencil, F3 pos, F3 L,
                                            const Frame& f, float alpha, float g, const float* h0s, Sink sink) {
  PixelGather q;
  q.pos = pos; q.L = L; q.X = f.X; q.Y = f.Y; q.Z = f.Z; q.LX = f.LX;
  q.lx = dot(f.LX, f.X); q.ly = dot(f.LX, f.Y); q.lz = dot(f.LX, f.Z);
  q.cXL = dot(f.X, L);
  q.cLXL = dot(f.LX, L);
  q.alpha = alpha;
  q.hg0 = __logf(hg_phase(dot(f.X, L), g) + 1.0f);
  const float ms = 0.6f;
  gather_seg<0, true, SAMP, 0, 8>(t, stencil, q, 1.0f / 256.0f * lerpf(ms, 1.0f, 1.0f), h0s, sink);
  gather_seg<1, true, SAMP, 8, 16>(t, stencil, q, 2.5f / 256.0f * lerpf(ms, 1.0f, 0.8f), h0s, sink);
  gather_seg<2, true, SAMP, 16, 32>(t, stencil, q, 5.5f / 256.0f * lerpf(ms, 1.0f, 0.6f), h0s, sink);
  gather_seg<3, true, SAMP, 32, 48>(t, stencil, q, 11.5f / 256.0f * lerpf(ms, 1.0f, 0.4f), h0s, sink);
  gather_seg<4, true, SAMP, 48, 64>(t, stencil, q, 23.5f / 256.0f * lerpf(ms, 1.0f, 0.2f), h0s, sink);
  gather_seg<5, true, SAMP, 64, 96>(t, stencil, q, 47.5f / 256.0f * ms, h0s, sink);
  gather_seg<6, true, SAMP, 96, 128>(t, stencil, q, 95.5f / 256.0f * ms, h0s, sink);
  gather_seg<7, true, SAMP, 128, 160>(t, stencil, q, 191.5f / 256.0f * ms, h0s, sink);
  gather_seg<0, false, SAMP, 160, 168>(t, stencil, q, 1.0f, h0s, sink);
  gather_seg<1, false, SAMP, 168, 176>(t, stencil, q, 1.0f, h0s, sink);
  gather_seg<2, false, SAMP, 176, 184>(t, stencil, q, 1.0f, h0s, sink);
  gather_seg<3, false, SAMP, 184, 192>(t, stencil, q, 1.0f, h0s, sink);
}

// Gather only, for explicit points and frames (test / training entry).
__global__ void k_gather(Tables t, const float* __restrict__ stencil, const float* __restrict__ pos,
                         const float* __restrict__ frame, int n, F3 L, float alpha, float g, F3 srp,
                         float* __restrict__ desc, float* __restrict__ aux) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  Frame f = load_frame(frame + 12 * (size_t)k);
  float* d = desc + 576 * (size_t)k;
  auto sink = [&](int i, int, float xv, float xs, float xh) {
    d[i] = xv;
    d[192 + i] = xs;
    d[384 + i] = xh;
  };
  gather_fast<kSampLoad>(t, stencil, f3(pos[3 * k], pos[3 * k + 1], pos[3 * k + 2]), L, f, alpha, g, nullptr, sink);
  float* ax = aux + 5 * (size_t)k;
  ax[0] = g;
  ax[1] = acosf(dot(f.X, f.LX));
  ax[2] = srp.x; ax[3] = srp.y; ax[4] = srp.z;
}

// Gather for the compacted records in chunk-of-4 feature-major order:
// features 4j..4j+3 of record k at desc[(j*cap + k)*4 .. +3] (aux: feature i at
// aux[i*cap + k]). A warp's 16-byte stores and the network's 16-byte loads of
// one chunk are contiguous 512-byte transactions.
// The texture forms are bound by fetch latency: registers capped for six
// 128-thread blocks per SM.
template <int SAMP>
__global__ void __launch_bounds__(128, SAMP == kSampLoad ? 1 : 6)
    k_gather_fm(Tables t, const float* __restrict__ stencil, const float* __restrict__ h0s, Records rec, int cap, F3 L,
                float alpha, float g, F3 srp, float* __restrict__ desc, float* __restrict__ aux) {
  const unsigned n = min(*rec.count, (unsigned)cap);
  // a resident grid strides over the records (the record count is known on
  // the device only)
  for (unsigned k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    F3 pos = f3(rec.pos[3 * (size_t)k], rec.pos[3 * (size_t)k + 1], rec.pos[3 * (size_t)k + 2]);
    Frame f = load_frame(rec.frame + 12 * (size_t)k);
    // chunk-of-4 feature-major: features 4j..4j+3 of record k are the float4
    // at desc[(j*cap + k)*4]; a warp's store of one chunk is 512 contiguous bytes
    float4* d = reinterpret_cast<float4*>(desc) + k;
    const size_t c = (size_t)cap;
    float4 bv, bs, bh;
    auto sink = [&](int i, int u, float xv, float xs, float xh) {
      (&bv.x)[u] = xv;
      (&bs.x)[u] = xs;
      (&bh.x)[u] = xh;
      if (u == 3) {
        d[(i >> 2) * c] = bv;
        d[(48 + (i >> 2)) * c] = bs;
        d[(96 + (i >> 2)) * c] = bh;
      }
    };
    gather_fast<SAMP>(t, stencil, pos, L, f, alpha, g, h0s, sink);
    aux[k] = g;
    aux[c + k] = acosf(dot(f.X, f.LX));
    aux[2 * c + k] = srp.x;
    aux[3 * c + k] = srp.y;
    aux[4 * c + k] = srp.z;
  }
}

int launch_mlp_tc(const Network* net, const float* desc, const float* aux, long long rs, long long cs,
                  long long ars, long long afs, int n, float* out, const int* pix, const float* trph,
                  const unsigned* count, F3 light_color, F3 scatter, float* spill, bool f8, cudaStream_t s,
                  const int* job = nullptr, const BatchOut* bout = nullptr);
int launch_mlp_simt(const Network* net, const float* desc, const float* aux, long long rs, long long cs,
                    long long ars, long long afs, int n, const unsigned* count, float* out, const int* pix,
                    const float* trph, F3 light_color, F3 scatter, cudaStream_t s, const int* job, const BatchOut* bout,
                    float* tout, long long trs, long long tcs, float* stg, long long srs, long long scs,
                    StageTimer* timer = nullptr);
int mlp_tc_error(const Network* net, bool reset);

extern int check_params(const mr_render_params* p);
extern CameraModel make_camera(const mr_render_params* p);
extern PathScene make_path_scene(const mr_render_params* p);

constexpr size_t records_bytes(size_t n) { return n * (sizeof(int) + 16 * sizeof(float)) + 256; }
constexpr size_t records_round(size_t n) { return (records_bytes(n) + 255) / 256 * 256; }
// Scratch of one neural render of n pixels: records, then 576 feature-major
// descriptor columns and 5 aux columns, then (when the albedo channels
// differ) 120 spill columns of the tensor-core network's head input, then the
// per-point table (k_sphere_h0, kPtTable floats).
constexpr size_t h0_offset(size_t n, bool spill) {
  return (records_round(n) + n * (576 + 5 + (spill ? 120 : 0)) * sizeof(float) + 255) / 256 * 256;
}
constexpr size_t neural_scratch_bytes(size_t n, bool spill) { return h0_offset(n, spill) + 2048; }
static bool distinct_channels(const mr_render_params* p) {
  return p->scatter_rate.x != p->scatter_rate.y || p->scatter_rate.x != p->scatter_rate.z;
}

static int neural_passes(Volume* v, const Network* net, const mr_render_params* p, float* dev_rgb, cudaStream_t s,
                         void* base, bool timed, float* dev_dist = nullptr, bool no_alloc = false,
                         bool marching = false);

// Linear tables of a volume plus the texture objects sampler form `samp`
// reads, whose copies are brought up to date on stream s.
static int fill_tables(Volume* v, int samp, Tables* t, cudaStream_t s) {
  *t = Tables{};
  t->mips = v->mips;
  t->tr = v->tr;
  t->lut = v->lut;
  if (samp == kSampTex) {
    int rc = refresh_textures(v, s);
    if (rc) return rc;
    for (int k = 0; k < 9; ++k) t->mip_tex[k] = v->mip_tex[k];
    for (int k = 0; k < 8; ++k) t->tr_tex[k] = v->tr_tex[k];
    t->lut_tex = v->lut_tex;
  } else if (samp == kSampGather) {
    int rc = refresh_gather_textures(v, s);
    if (rc) return rc;
    for (int k = 0; k < 9; ++k) t->mip_g[k] = v->gth_mip_tex[k];
    for (int k = 0; k < 8; ++k) t->tr_g[k] = v->gth_tr_tex[k];
    t->lut_g = v->gth_lut_tex;
  }
  return MR_OK;
}

static Records carve_records(void* base, size_t n) {
  char* p = (char*)base;
  Records r;
  r.job = nullptr;
  r.count = (unsigned*)p; p += 256;
  r.pix = (int*)p; p += n * sizeof(int);
  r.pos = (float*)p; p += 3 * n * sizeof(float);
  r.frame = (float*)p; p += 12 * n * sizeof(float);
  r.trph = (float*)p;
  return r;
}

static int render_neural_impl(Volume* v, const Network* net, const mr_render_params* p, float* dev_rgb,
                              float* dev_dist, cudaStream_t s, bool marching = false);
int render_neural(Volume* v, const Network* net, const mr_render_params* p, float* dev_rgb, cudaStream_t s) {
  return render_neural_impl(v, net, p, dev_rgb, nullptr, s);
}
// NNPredict<Type::marching_MRPNN> (ray marching, optional dielectric surface).
int render_marching(Volume* v, const Network* net, const mr_render_params* p, float* dev_rgb, cudaStream_t s) {
  return render_neural_impl(v, net, p, dev_rgb, nullptr, s, true);
}
static size_t march_extra_bytes(size_t n) { return (n * sizeof(float4) + 255) / 256 * 256; }
// Same, also writing the first-hit distance of every pixel (interactive mode).
int render_neural_dist(Volume* v, const Network* net, const mr_render_params* p, float* dev_rgb, float* dev_dist,
                       cudaStream_t s) {
  return render_neural_impl(v, net, p, dev_rgb, dev_dist, s);
}

static int render_neural_impl(Volume* v, const Network* net, const mr_render_params* p, float* dev_rgb,
                              float* dev_dist, cudaStream_t s, bool marching) {
  if (!net) return set_error(MR_ERR_ARG, "MRPNN render needs a network (mr_network_create)");
  if (!v->data_set) return set_error(MR_ERR_STATE, "render before mr_volume_set_data");
  if (!v->mips_valid) return set_error(MR_ERR_STATE, "render before mr_volume_update");
  if (p->precision != MR_PREC_FP32 && p->precision != MR_PREC_BF16 && p->precision != MR_PREC_FP8)
    return set_error(MR_ERR_ARG, "unknown precision %d", p->precision);
  // with an environment map, this pass's light is drawn from it or from the
  // directional light (the transmittance pyramid follows the chosen light)
  mr_render_params q = *p;
  select_env_light(v, &q);
  p = &q;
  F3 L = normalize(to_f3(p->light_dir));
  // UpdateHGLut / Update_TR on demand (core/volume.cu:434-437).
  if (!v->lut_valid || v->lut_g != p->g || v->lut_seed != p->seed) {
    int rc = launch_update_lut(v, p->g, p->seed, s);
    if (rc) return rc;
  }
  if (!v->tr_valid || L.x != v->tr_light.x || L.y != v->tr_light.y || L.z != v->tr_light.z || p->alpha != v->tr_alpha) {
    int rc = launch_update_tr(v, L, p->alpha, s);
    if (rc) return rc;
  }
  size_t npx = (size_t)p->width * p->height;
  int rc = ensure_scratch(v, neural_scratch_bytes(npx, distinct_channels(p)) + (marching ? march_extra_bytes(npx) : 0),
                          s);
  if (rc) return rc;
  return neural_passes(v, net, p, dev_rgb, s, v->scratch, true, dev_dist, false, marching);
}

// Trace, gather and network over scratch at `base` (neural_scratch_bytes of
// width*height); `timed` = record stage events when the volume's timer is on.
static int neural_passes(Volume* v, const Network* net, const mr_render_params* p, float* dev_rgb, cudaStream_t s,
                         void* base, bool timed, float* dev_dist, bool no_alloc, bool marching) {
  auto mark = [&](int st) { if (timed) v->timer.mark(st, s); };
  int rc = MR_OK;
  const F3 L = normalize(to_f3(p->light_dir));
  const size_t npx = (size_t)p->width * p->height;
  const bool tc = p->precision != MR_PREC_FP32;
  // records, then the feature-major descriptor and aux columns
  const size_t rbytes = records_round(npx);
  Records rec = carve_records(base, npx);
  float* desc = (float*)((char*)base + rbytes);
  float* aux = desc + npx * 576;
  float* spill = distinct_channels(p) ? aux + npx * 5 : nullptr;
  MR_CUDA(cudaMemsetAsync(v->d_counters, 0, kCounters * sizeof(unsigned long long), s));
  MR_CUDA(cudaMemsetAsync(rec.count, 0, sizeof(unsigned), s));
  NNTraceArgs ta;
  ta.m = Medium{v->density, v->res, v->max_density, p->tr_scale, 0};
  if (!no_alloc) {
    rc = density_gather_texture(v, s, &ta.m.tex);
    if (rc) return rc;
  }
  ta.sc = make_path_scene(p);
  attach_env(ta.sc, v);
  ta.cam = make_camera(p);
  ta.seed = p->seed;
  ta.frame_index = p->sample_offset;
  ta.out = dev_rgb;
  ta.dist = dev_dist;
  ta.rec = rec;
  ta.counters = v->d_counters;
  // the exact sampler reads texture gathers, or texel loads where nothing
  // may be allocated (the layered copies are created on first use)
  const int samp = p->sampler == MR_SAMPLER_TEXTURE ? kSampTex : no_alloc ? kSampLoad : kSampGather;
  Tables tabs;
  rc = fill_tables(v, samp, &tabs, s);
  if (rc) return rc;
  // The per-point table (one block) runs on the volume's side stream beside
  // the trace, which does not read it; the gather waits for it. Where nothing
  // may be created it runs in line.
  float* h0s = (float*)((char*)base + h0_offset(npx, distinct_channels(p)));
  cudaStream_t hs = s;
  if (!no_alloc) {
    if (!v->side_stream) {
      MR_CUDA(cudaStreamCreateWithFlags(&v->side_stream, cudaStreamNonBlocking));
      MR_CUDA(cudaEventCreateWithFlags(&v->side_fork, cudaEventDisableTiming));
      MR_CUDA(cudaEventCreateWithFlags(&v->side_join, cudaEventDisableTiming));
    }
    hs = v->side_stream;
    MR_CUDA(cudaEventRecord(v->side_fork, s));
    MR_CUDA(cudaStreamWaitEvent(hs, v->side_fork, 0));
  }
  if (samp == kSampTex)
    k_sphere_h0<kSampTex><<<1, 192, 0, hs>>>(tabs, net->stencil, h0s);
  else if (samp == kSampGather)
    k_sphere_h0<kSampGather><<<1, 192, 0, hs>>>(tabs, net->stencil, h0s);
  else
    k_sphere_h0<kSampLoad><<<1, 192, 0, hs>>>(tabs, net->stencil, h0s);
  MR_CUDA(cudaGetLastError());
  if (hs != s) MR_CUDA(cudaEventRecord(v->side_join, hs));
  float4* madd = marching ? (float4*)((char*)base + neural_scratch_bytes(npx, distinct_channels(p))) : nullptr;
  mark(ST_NN_TRACE);
  if (marching) {
    MarchArgs ma;
    ma.m = ta.m;
    ma.sc = ta.sc;
    ma.cam = ta.cam;
    ma.seed = ta.seed;
    ma.frame_index = ta.frame_index;
    ma.ior = v->surface_ior;
    ma.out = dev_rgb;
    ma.rec = rec;
    ma.madd = madd;
    ma.counters = v->d_counters;
    k_march_trace<<<(unsigned)((npx + 127) / 128), 128, 0, s>>>(ma);
  } else {
    k_nn_trace<<<(unsigned)((npx + 127) / 128), 128, 0, s>>>(ta);
  }
  mark(ST_NN_TRACE);
  MR_CUDA(cudaGetLastError());
  if (hs != s) MR_CUDA(cudaStreamWaitEvent(s, v->side_join, 0));
  F3 sr = to_f3(p->scatter_rate) / 1.001f;
  mark(ST_NN_PREDICT);
  // resident grids: as many 128-thread blocks as fit on the GPU at once
  static DeviceCache gather_occ[3];  // per sampler, per device
  const int per_sm = gather_occ[samp].get([samp] {
    int n = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &n,
        samp == kSampTex ? (const void*)k_gather_fm<kSampTex>
                         : samp == kSampGather ? (const void*)k_gather_fm<kSampGather> : (const void*)k_gather_fm<kSampLoad>,
        128, 0);
    return std::max(1, n);
  });
  const unsigned ggrid = (unsigned)std::min<size_t>((npx + 127) / 128, (size_t)per_sm * sm_count());
  if (samp == kSampTex)
    k_gather_fm<kSampTex><<<ggrid, 128, 0, s>>>(tabs, net->stencil, h0s, rec, (int)npx, L, p->alpha, p->g,
                                               srp_of(sr), desc, aux);
  else if (samp == kSampGather)
    k_gather_fm<kSampGather><<<ggrid, 128, 0, s>>>(tabs, net->stencil, h0s, rec, (int)npx, L, p->alpha, p->g,
                                                  srp_of(sr), desc, aux);
  else
    k_gather_fm<kSampLoad><<<ggrid, 128, 0, s>>>(tabs, net->stencil, h0s, rec, (int)npx, L, p->alpha, p->g,
                                                srp_of(sr), desc, aux);
  mark(ST_NN_PREDICT);
  MR_CUDA(cudaGetLastError());
  const long long cap = (long long)npx;
  // the marching form weights the network's light by 1 - T afterwards and
  // does not multiply it by the albedo (core/render.cuh:631)
  const F3 out_scale = marching ? f3(1, 1, 1) : to_f3(p->scatter_rate);
  mark(ST_NN_MLP);
  if (tc)
    rc = launch_mlp_tc(net, desc, aux, 4, 4 * cap, 1, cap, (int)npx, dev_rgb, rec.pix, rec.trph, rec.count,
                       to_f3(p->light_color), out_scale, spill, p->precision == MR_PREC_FP8, s);
  else
    // trunk outputs over the row's first 38 descriptor chunks, the head's LC2
    // outputs over chunks 48..71 (all consumed by the trunk)
    rc = launch_mlp_simt(net, desc, aux, 4, 4 * cap, 1, cap, (int)npx, rec.count, dev_rgb, rec.pix, rec.trph,
                         to_f3(p->light_color), out_scale, s, nullptr, nullptr, desc, 4, 4 * cap,
                         desc + 48 * 4 * cap, 4, 4 * cap, timed ? &v->timer : nullptr);
  mark(ST_NN_MLP);
  if (rc == MR_OK && marching) {
    k_march_compose<<<(unsigned)((npx + 127) / 128), 128, 0, s>>>(rec.count, rec.pix, madd, dev_rgb);
    MR_CUDA(cudaGetLastError());
  }
  return rc;
}

}  // namespace mr

using namespace mr;

extern "C" int mr_gather_descriptors(const mr_volume* h, const mr_network* nh, const float* dev_pos,
                                     const float* dev_frame, int32_t n, float alpha, float g,
                                     mr_float3 scatter_rate, float* dev_desc, float* dev_aux, void* stream) {
  clear_error();
  if (!h || !nh || !dev_pos || !dev_frame || !dev_desc || !dev_aux)
    return set_error(MR_ERR_ARG, "mr_gather_descriptors: NULL argument");
  if (n < 0) return set_error(MR_ERR_ARG, "n < 0");
  if (n == 0) return MR_OK;
  const Volume* v = &h->v;
  if (!v->mips_valid || !v->tr_valid || !v->lut_valid)
    return set_error(MR_ERR_STATE, "gather needs mr_volume_update, _update_tr and _update_hglut first");
  F3 sr = to_f3(scatter_rate) / 1.001f;
  k_gather<<<(n + 127) / 128, 128, 0, (cudaStream_t)stream>>>(Tables{v->mips, v->tr, v->lut, {}, {}, 0}, nh->n.stencil,
                                                            dev_pos, dev_frame, n, v->tr_light, alpha, g,
                                                            srp_of(sr), dev_desc, dev_aux);
  MR_CUDA(cudaGetLastError());
  return MR_OK;
}

namespace mr {
// Both exact sampler forms on the same points: texel loads and texture
// gathers, for the trilinear border / clamp filters and the bilinear clamp.
__global__ void k_sampler_selftest(cudaTextureObject_t tb, cudaTextureObject_t tc, cudaTextureObject_t t2,
                                   const float* __restrict__ d, const float* __restrict__ uv, int n, float* out) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const F3 p = f3(uv[3 * k], uv[3 * k + 1], uv[3 * k + 2]);
  float* o = out + 6 * (size_t)k;
  o[0] = tri_border_c<MR_SAMPLER_SELFTEST_RES>(d, p);
  o[1] = tri_border_g<MR_SAMPLER_SELFTEST_RES>(tb, p);
  o[2] = tri_clamp_c<MR_SAMPLER_SELFTEST_RES>(d, p);
  o[3] = tri_clamp_g<MR_SAMPLER_SELFTEST_RES>(tc, p);
  o[4] = bilinear_clamp(d, MR_SAMPLER_SELFTEST_RES, MR_SAMPLER_SELFTEST_RES, p.x, p.y);
  o[5] = bilinear_clamp_g(t2, MR_SAMPLER_SELFTEST_RES, MR_SAMPLER_SELFTEST_RES, p.x, p.y);
}
}  // namespace mr

extern "C" int mr_sampler_selftest(int32_t n, const float* host_table, const float* host_uv, float* host_out) {
  clear_error();
  if (n <= 0 || !host_table || !host_uv || !host_out) return set_error(MR_ERR_ARG, "mr_sampler_selftest: bad argument");
  constexpr int R = MR_SAMPLER_SELFTEST_RES;
  float *d = nullptr, *uv = nullptr, *out = nullptr;
  cudaArray_t ab = nullptr, ac = nullptr, a2 = nullptr;
  cudaTextureObject_t tb = 0, tc = 0, t2 = 0;
  int rc = MR_OK;
  auto run = [&]() -> int {
    MR_CUDA(cudaMalloc(&d, (size_t)R * R * R * sizeof(float)));
    MR_CUDA(cudaMalloc(&uv, 3 * (size_t)n * sizeof(float)));
    MR_CUDA(cudaMalloc(&out, 6 * (size_t)n * sizeof(float)));
    MR_CUDA(cudaMemcpy(d, host_table, (size_t)R * R * R * sizeof(float), cudaMemcpyHostToDevice));
    MR_CUDA(cudaMemcpy(uv, host_uv, 3 * (size_t)n * sizeof(float), cudaMemcpyHostToDevice));
    int r = make_gather_tex(&ab, &tb, R, cudaAddressModeBorder);
    if (!r) r = make_gather_tex(&ac, &tc, R, cudaAddressModeClamp);
    if (!r) r = copy_to_array(ab, d, R, 0);
    if (!r) r = copy_to_array(ac, d, R, 0);
    if (r) return r;
    cudaChannelFormatDesc ch = cudaCreateChannelDesc<float>();
    MR_CUDA(cudaMallocArray(&a2, &ch, R, R));
    MR_CUDA(cudaMemcpy2DToArray(a2, 0, 0, d, R * sizeof(float), R * sizeof(float), R, cudaMemcpyDeviceToDevice));
    cudaResourceDesc rd = {};
    rd.resType = cudaResourceTypeArray;
    rd.res.array.array = a2;
    cudaTextureDesc td = {};
    td.addressMode[0] = td.addressMode[1] = cudaAddressModeClamp;
    td.filterMode = cudaFilterModePoint;
    td.readMode = cudaReadModeElementType;
    td.normalizedCoords = 0;
    MR_CUDA(cudaCreateTextureObject(&t2, &rd, &td, nullptr));
    k_sampler_selftest<<<(n + 127) / 128, 128>>>(tb, tc, t2, d, uv, n, out);
    MR_CUDA(cudaGetLastError());
    MR_CUDA(cudaMemcpy(host_out, out, 6 * (size_t)n * sizeof(float), cudaMemcpyDeviceToHost));
    return MR_OK;
  };
  rc = run();
  if (tb) cudaDestroyTextureObject(tb);
  if (tc) cudaDestroyTextureObject(tc);
  if (t2) cudaDestroyTextureObject(t2);
  if (ab) cudaFreeArray(ab);
  if (ac) cudaFreeArray(ac);
  if (a2) cudaFreeArray(a2);
  cudaFree(d);
  cudaFree(uv);
  cudaFree(out);
  return rc;
}

extern "C" int mr_radiance_predict(const mr_network* nh, int32_t precision, const float* dev_desc,
                                   const float* dev_aux, int32_t n, float* dev_out, void* stream) {
  clear_error();
  if (!nh || !dev_desc || !dev_aux || !dev_out) return set_error(MR_ERR_ARG, "mr_radiance_predict: NULL argument");
  if (n < 0) return set_error(MR_ERR_ARG, "n < 0");
  if (n == 0) return MR_OK;
  if (reinterpret_cast<uintptr_t>(dev_desc) & 15)
    return set_error(MR_ERR_ARG, "mr_radiance_predict: dev_desc must be 16-byte aligned");
  if (precision == MR_PREC_BF16 || precision == MR_PREC_FP8) {
    // rows may carry distinct albedo channels: spill space for further heads
    cudaStream_t s = (cudaStream_t)stream;
    float* spill = nullptr;
    cudaError_t e = cudaMallocAsync(&spill, (size_t)n * 120 * sizeof(float), s);
    if (e != cudaSuccess) return set_error(MR_ERR_NOMEM, "spill allocation failed: %s", cudaGetErrorString(e));
    int rc = launch_mlp_tc(&nh->n, dev_desc, dev_aux, 576, 4, 5, 1, n, dev_out, nullptr, nullptr, nullptr,
                           f3(1, 1, 1), f3(1, 1, 1), spill, precision == MR_PREC_FP8, s);
    MR_CUDA(cudaFreeAsync(spill, s));
    return rc;
  }
  if (precision != MR_PREC_FP32) return set_error(MR_ERR_ARG, "unknown precision %d", precision);
  // the caller's descriptors stay untouched: trunk outputs (152) and the
  // head's LC2 outputs (96) of a row go to a temporary
  cudaStream_t s = (cudaStream_t)stream;
  float* tout = nullptr;
  cudaError_t e = cudaMallocAsync(&tout, (size_t)n * 248 * sizeof(float), s);
  if (e != cudaSuccess) return set_error(MR_ERR_NOMEM, "trunk buffer: %s", cudaGetErrorString(e));
  int rc = launch_mlp_simt(&nh->n, dev_desc, dev_aux, 576, 4, 5, 1, n, nullptr, dev_out, nullptr, nullptr,
                           f3(1, 1, 1), f3(1, 1, 1), s, nullptr, nullptr, tout, 248, 4, tout + 152, 248, 4);
  MR_CUDA(cudaFreeAsync(tout, s));
  return rc;
}

// ---- fixed-scratch neural render (mr_render_neural_noalloc) -------------------

namespace mr {
// Module-resident scratch for mr_render_neural_noalloc: records plus
// descriptor columns of up to MR_NOALLOC_MAX_PIXELS pixels.
constexpr size_t kNoallocBytes = (size_t)MR_NOALLOC_SCRATCH_MIB << 20;
static_assert(neural_scratch_bytes(MR_NOALLOC_MAX_PIXELS, true) <= kNoallocBytes, "no-alloc scratch too small");
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocBytes];

constexpr int kNoallocDevices = 64;
static std::mutex g_noalloc_mu;
static void* g_noalloc_ptr[kNoallocDevices];

// Address of g_noalloc_scratch on the current device, looked up once per
// device (cudaGetSymbolAddress also loads the module there on first use).
static int noalloc_scratch(void** out) {
  int dev = 0;
  MR_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kNoallocDevices) return set_error(MR_ERR_ARG, "device ordinal %d out of range", dev);
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    void* ptr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_error(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
    g_noalloc_ptr[dev] = ptr;
  }
  *out = g_noalloc_ptr[dev];
  return MR_OK;
}
}  // namespace mr

extern "C" int mr_render_neural_noalloc(mr_volume* h, const mr_network* nh, const mr_render_params* p,
                                        float* dev_rgb, void* stream) {
  clear_error();
  if (!h || !nh || !p || !dev_rgb) return set_error(MR_ERR_ARG, "mr_render_neural_noalloc: NULL argument");
  int rc = check_params(p);
  if (rc) return rc;
  if (p->render_type != MR_RT_MRPNN)
    return set_error(MR_ERR_ARG, "mr_render_neural_noalloc renders MR_RT_MRPNN only (got %d)", p->render_type);
  if (p->precision != MR_PREC_FP32 && p->precision != MR_PREC_BF16)
    return set_error(MR_ERR_UNSUPPORTED, "mr_render_neural_noalloc supports MR_PREC_FP32 and MR_PREC_BF16 (got %d)",
                     p->precision);
  if (p->sampler != MR_SAMPLER_EXACT)
    return set_error(MR_ERR_ARG, "mr_render_neural_noalloc supports MR_SAMPLER_EXACT only "
                                 "(texture tables are allocated on first use)");
  const size_t npx = (size_t)p->width * p->height;
  if (npx > MR_NOALLOC_MAX_PIXELS)
    return set_error(MR_ERR_ARG, "mr_render_neural_noalloc: %d x %d = %zu pixels exceeds MR_NOALLOC_MAX_PIXELS (%d)",
                     p->width, p->height, npx, MR_NOALLOC_MAX_PIXELS);
  Volume* v = &h->v;
  if (!v->data_set || !v->mips_valid) return set_error(MR_ERR_STATE, "render before mr_volume_set_data / _update");
  const F3 L = normalize(to_f3(p->light_dir));
  if (!v->lut_valid || v->lut_g != p->g || v->lut_seed != p->seed)
    return set_error(MR_ERR_STATE, "HG table not built for g=%g seed=%u: call mr_volume_update_hglut first", p->g,
                     p->seed);
  if (!v->tr_valid || L.x != v->tr_light.x || L.y != v->tr_light.y || L.z != v->tr_light.z || p->alpha != v->tr_alpha)
    return set_error(MR_ERR_STATE, "transmittance pyramid not built for this light/alpha: call mr_volume_update_tr first");
  void* base = nullptr;
  rc = noalloc_scratch(&base);
  if (rc) return rc;
  return neural_passes(v, &nh->n, p, dev_rgb, (cudaStream_t)stream, base, false, nullptr, true);
}

// ---- batched neural render ------------------------------------------------------------
// Many (volume, view) jobs rendered together: the jobs' pixels form one
// flattened space, processed in waves of `wave` pixels; each wave is one
// batched trace, one batched gather and one network launch over the records
// of all jobs in it. Every launch of a batch frame can be captured into one
// CUDA graph; the graph ends with a kernel that advances the jobs' sample
// indices, so each replay renders the next frame.

namespace mr {

struct BatchJob {
  Medium m;
  PathScene sc;
  CameraModel cam;
  uint32_t seed, frame;
  Tables tabs;      // the job's volume tables (and texture objects for the texture sampler)
  F3 srp;           // (albedo / 1.001)^4
  long long pix0;   // first pixel of the job in the flattened pixel space
  int npx;
};

__global__ void __launch_bounds__(256) k_trace_batch(const BatchJob* __restrict__ jobs, int njobs, long long w0,
                                                     long long w1, const BatchOut* __restrict__ bout, Records rec,
                                                     unsigned long long* counters) {
  const long long p = w0 + (long long)blockIdx.x * blockDim.x + threadIdx.x;
  TrackStats st{0, 0};
  unsigned act = 0;
  int lo = -1;
  if (p < w1) {
    int hi = njobs - 1;  // last job with pix0 <= p
    lo = 0;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (jobs[mid].pix0 <= p) lo = mid;
      else hi = mid - 1;
    }
  }
  // one job at a time per warp: the density texture handle must be uniform
  // across the lanes of a texture fetch (see k_gather_batch)
  unsigned todo = __ballot_sync(0xffffffffu, p < w1);
  while (todo) {
    const int jj = __shfl_sync(0xffffffffu, lo, __ffs(todo) - 1);
    const bool mine = p < w1 && lo == jj;
    if (mine) {
      const BatchJob& j = jobs[jj];
      act = trace_pixel(j.m, j.sc, j.cam, j.seed, j.frame, (int)(p - j.pix0), bout[jj].out, nullptr, rec, jj, st);
    }
    todo &= ~__ballot_sync(0xffffffffu, mine);
  }
  trace_counters(counters, st, act);
}

// The per-point table of every job (point_table over the job's tables), one
// block per job, into h0[job * kPtTable].
template <int SAMP>
__global__ void k_sphere_h0_batch(const BatchJob* __restrict__ jobs, const float* __restrict__ stencil,
                                  float* __restrict__ h0) {
  point_table<SAMP>(jobs[blockIdx.x].tabs, stencil, h0 + (size_t)blockIdx.x * kPtTable);
}

template <int SAMP>
__global__ void __launch_bounds__(256, 3) k_gather_batch(const BatchJob* __restrict__ jobs,
                                                      const float* __restrict__ stencil,
                                                      const float* __restrict__ h0, Records rec, int cap,
                                                      float* __restrict__ desc, float* __restrict__ aux) {
  const unsigned k = blockIdx.x * blockDim.x + threadIdx.x;
  const unsigned n = min(*rec.count, (unsigned)cap);
  const bool valid = k < n;
  const int job = valid ? rec.job[k] : -1;
  // One job at a time per warp. The texture handles of a fetch must be the
  // same in all its lanes: with records of two volumes in one warp, fetches
  // returned wrong texels (measured: batches mixing two volumes in one wave
  // differed from single renders by up to 48 % in 4 % of the values; with
  // warp-uniform jobs they agree to 3e-6).
  unsigned todo = __ballot_sync(0xffffffffu, valid);
  while (todo) {
    const int jj = __shfl_sync(0xffffffffu, job, __ffs(todo) - 1);
    const bool mine = valid && job == jj;
    if (mine) {
      const BatchJob& j = jobs[jj];
      const F3 pos = f3(rec.pos[3 * (size_t)k], rec.pos[3 * (size_t)k + 1], rec.pos[3 * (size_t)k + 2]);
      const Frame f = load_frame(rec.frame + 12 * (size_t)k);
      float4* d = reinterpret_cast<float4*>(desc) + k;
      const size_t c = (size_t)cap;
      float4 bv, bs, bh;
      auto sink = [&](int i, int u, float xv, float xs, float xh) {
        (&bv.x)[u] = xv;
        (&bs.x)[u] = xs;
        (&bh.x)[u] = xh;
        if (u == 3) {
          d[(i >> 2) * c] = bv;
          d[(48 + (i >> 2)) * c] = bs;
          d[(96 + (i >> 2)) * c] = bh;
        }
      };
      gather_fast<SAMP>(j.tabs, stencil, pos, j.sc.L, f, j.sc.alpha, j.sc.g, h0 + (size_t)jj * kPtTable, sink);
      aux[k] = j.sc.g;
      aux[c + k] = acosf(dot(f.X, f.LX));
      aux[2 * c + k] = j.srp.x;
      aux[3 * c + k] = j.srp.y;
      aux[4 * c + k] = j.srp.z;
    }
    todo &= ~__ballot_sync(0xffffffffu, mine);
  }
}

__global__ void k_batch_advance(BatchJob* jobs, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) jobs[i].frame += 1u;
}

// The device's global nanosecond timer, by one thread, when the stream
// reaches this launch.
__global__ void k_stamp(unsigned long long* out) {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  *out = t;
}

struct Batch {
  struct HostJob {
    Volume* v;
    mr_render_params p;
    float* out;
  };
  std::vector<HostJob> jobs;
  BatchJob* d_jobs = nullptr;
  float* d_h0 = nullptr;  // per-job point tables (k_sphere_h0_batch), kPtTable floats each
  BatchOut* d_out = nullptr;
  unsigned long long* counters = nullptr;
  void* scratch = nullptr;
  size_t scratch_bytes = 0;
  long long total = 0, wave = 0;
  int trace_block = 128, gather_block = 128;
  int precision = MR_PREC_BF16, sampler = MR_SAMPLER_EXACT;
  bool spill = false, prepared = false;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  // Per-frame completion times (mr_batch_set_timing): one-thread kernels
  // write the device's global nanosecond timer before the first launch
  // (slot 0) and after each wave's network (slot 1 + wave). Kernel nodes
  // behave the same in a captured graph as on a stream.
  bool timing = false;
  unsigned long long* d_stamps = nullptr;
  size_t n_stamps = 0;

  void drop_events() {
    if (d_stamps) cudaFree(d_stamps);
    d_stamps = nullptr;
    n_stamps = 0;
  }
  void drop_graph() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    exec = nullptr;
    graph = nullptr;
  }
  void release() {
    drop_graph();
    drop_events();
    if (d_jobs) cudaFree(d_jobs);
    if (d_h0) cudaFree(d_h0);
    if (d_out) cudaFree(d_out);
    if (counters) cudaFree(counters);
    if (scratch) cudaFree(scratch);
    d_jobs = nullptr;
    d_h0 = nullptr;
    d_out = nullptr;
    counters = nullptr;
    scratch = nullptr;
    scratch_bytes = 0;
    prepared = false;
  }
};

static size_t batch_scratch_bytes(long long wave, bool spill) {
  return neural_scratch_bytes((size_t)wave, spill) + ((size_t)wave * sizeof(int) + 255) / 256 * 256;
}

// Stream-ordered launches of one batch frame (eager or under capture).
static int batch_launches(Batch& b, const Network* net, cudaStream_t s) {
  const size_t cap = (size_t)b.wave;
  const size_t rbytes = records_round(cap);
  Records rec = carve_records(b.scratch, cap);
  float* desc = (float*)((char*)b.scratch + rbytes);
  float* aux = desc + cap * 576;
  float* spill = b.spill ? aux + cap * 5 : nullptr;
  rec.job = (int*)((char*)b.scratch + neural_scratch_bytes(cap, b.spill));
  const bool tc = b.precision != MR_PREC_FP32;
  const bool hw = b.sampler == MR_SAMPLER_TEXTURE;
  const int nj = (int)b.jobs.size();
  const bool timed = b.timing && b.d_stamps && (long long)(b.n_stamps - 1) * b.wave >= b.total;
  if (timed) {
    k_stamp<<<1, 1, 0, s>>>(b.d_stamps);
    MR_CUDA(cudaGetLastError());
  }
  MR_CUDA(cudaMemsetAsync(b.counters, 0, kCounters * sizeof(unsigned long long), s));
  // the jobs' per-point tables, for the network given to this call
  if (hw)
    k_sphere_h0_batch<kSampTex><<<nj, 192, 0, s>>>(b.d_jobs, net->stencil, b.d_h0);
  else
    k_sphere_h0_batch<kSampGather><<<nj, 192, 0, s>>>(b.d_jobs, net->stencil, b.d_h0);
  MR_CUDA(cudaGetLastError());
  for (long long w0 = 0; w0 < b.total; w0 += b.wave) {
    const long long w1 = std::min(b.total, w0 + b.wave);
    MR_CUDA(cudaMemsetAsync(rec.count, 0, sizeof(unsigned), s));
    const unsigned tgrid = (unsigned)((w1 - w0 + b.trace_block - 1) / b.trace_block);
    k_trace_batch<<<tgrid, b.trace_block, 0, s>>>(b.d_jobs, nj, w0, w1, b.d_out, rec, b.counters);
    MR_CUDA(cudaGetLastError());
    const unsigned ggrid = (unsigned)((w1 - w0 + b.gather_block - 1) / b.gather_block);
    if (hw)
      k_gather_batch<kSampTex><<<ggrid, b.gather_block, 0, s>>>(b.d_jobs, net->stencil, b.d_h0, rec, (int)cap, desc,
                                                                aux);
    else
      k_gather_batch<kSampGather><<<ggrid, b.gather_block, 0, s>>>(b.d_jobs, net->stencil, b.d_h0, rec, (int)cap,
                                                                   desc, aux);
    MR_CUDA(cudaGetLastError());
    const long long ccap = (long long)cap;
    int rc;
    if (tc)
      rc = launch_mlp_tc(net, desc, aux, 4, 4 * ccap, 1, ccap, (int)cap, nullptr, rec.pix, rec.trph, rec.count,
                         f3(1, 1, 1), f3(1, 1, 1), spill, b.precision == MR_PREC_FP8, s, rec.job, b.d_out);
    else
      rc = launch_mlp_simt(net, desc, aux, 4, 4 * ccap, 1, ccap, (int)cap, rec.count, nullptr, rec.pix, rec.trph,
                           f3(1, 1, 1), f3(1, 1, 1), s, rec.job, b.d_out, desc, 4, 4 * ccap, desc + 48 * 4 * ccap, 4,
                           4 * ccap);
    if (rc) return rc;
    if (timed) {
      k_stamp<<<1, 1, 0, s>>>(b.d_stamps + 1 + w0 / b.wave);
      MR_CUDA(cudaGetLastError());
    }
  }
  k_batch_advance<<<(nj + 127) / 128, 128, 0, s>>>(b.d_jobs, nj);
  MR_CUDA(cudaGetLastError());
  return MR_OK;
}

static int batch_alloc_scratch(Batch& b, long long wave) {
  const size_t need = batch_scratch_bytes(wave, b.spill);
  if (b.scratch_bytes >= need) return MR_OK;
  if (b.scratch) MR_CUDA(cudaFree(b.scratch));
  b.scratch = nullptr;
  b.scratch_bytes = 0;
  cudaError_t e = cudaMalloc(&b.scratch, need);
  if (e != cudaSuccess) return set_error(MR_ERR_NOMEM, "batch scratch of %zu bytes: %s", need, cudaGetErrorString(e));
  b.scratch_bytes = need;
  return MR_OK;
}

}  // namespace mr

struct mr_batch { mr::Batch b; };

extern "C" int mr_batch_create(mr_batch** out) {
  clear_error();
  if (!out) return set_error(MR_ERR_ARG, "mr_batch_create: NULL argument");
  *out = new mr_batch();
  return MR_OK;
}

extern "C" int mr_batch_destroy(mr_batch* h) {
  if (!h) return MR_OK;
  h->b.release();
  delete h;
  return MR_OK;
}

extern "C" int mr_batch_add(mr_batch* h, mr_volume* v, const mr_render_params* p, float* dev_rgb) {
  clear_error();
  if (!h || !v || !p || !dev_rgb) return set_error(MR_ERR_ARG, "mr_batch_add: NULL argument");
  int rc = check_params(p);
  if (rc) return rc;
  if (p->render_type != MR_RT_MRPNN) return set_error(MR_ERR_ARG, "batched renders are neural (MR_RT_MRPNN)");
  if (!v->v.data_set || !v->v.mips_valid) return set_error(MR_ERR_STATE, "volume needs mr_volume_set_data / _update");
  Batch& b = h->b;
  if (!b.jobs.empty() && (p->precision != b.jobs[0].p.precision || p->sampler != b.jobs[0].p.sampler))
    return set_error(MR_ERR_ARG, "all jobs of a batch share one precision and sampler");
  b.jobs.push_back({&v->v, *p, dev_rgb});
  b.prepared = false;
  b.drop_graph();
  return MR_OK;
}

extern "C" int mr_batch_prepare(mr_batch* h, const mr_network* nh, int64_t wave_pixels, void* stream) {
  clear_error();
  if (!h || !nh) return set_error(MR_ERR_ARG, "mr_batch_prepare: NULL argument");
  Batch& b = h->b;
  if (b.jobs.empty()) return set_error(MR_ERR_STATE, "empty batch");
  if (wave_pixels < 0) return set_error(MR_ERR_ARG, "wave_pixels < 0");
  cudaStream_t s = (cudaStream_t)stream;
  b.drop_graph();
  b.precision = b.jobs[0].p.precision;
  b.sampler = b.jobs[0].p.sampler;
  if (b.precision != MR_PREC_FP32 && b.precision != MR_PREC_BF16 && b.precision != MR_PREC_FP8)
    return set_error(MR_ERR_ARG, "unknown precision %d", b.precision);
  std::vector<BatchJob> hj(b.jobs.size());
  std::vector<BatchOut> ho(b.jobs.size());
  long long off = 0;
  b.spill = false;
  for (size_t i = 0; i < b.jobs.size(); ++i) {
    Batch::HostJob& J = b.jobs[i];
    Volume* v = J.v;
    const mr_render_params* p = &J.p;
    const F3 L = normalize(to_f3(p->light_dir));
    // a volume's tables serve one (g, seed) and one (light, alpha): the first
    // job on a volume builds them, later jobs must agree
    bool first = true;
    for (size_t k = 0; k < i; ++k) first = first && b.jobs[k].v != v;
    const bool lut_ok = v->lut_valid && v->lut_g == p->g && v->lut_seed == p->seed;
    const bool tr_ok = v->tr_valid && L.x == v->tr_light.x && L.y == v->tr_light.y && L.z == v->tr_light.z &&
                       p->alpha == v->tr_alpha;
    if (!first && (!lut_ok || !tr_ok))
      return set_error(MR_ERR_ARG, "job %zu: shares a volume with an earlier job but needs other light/alpha/g "
                                   "tables; give it its own volume", i);
    if (!lut_ok) {
      int rc = launch_update_lut(v, p->g, p->seed, s);
      if (rc) return rc;
    }
    if (!tr_ok) {
      int rc = launch_update_tr(v, L, p->alpha, s);
      if (rc) return rc;
    }
    BatchJob& j = hj[i];
    j.m = Medium{v->density, v->res, v->max_density, p->tr_scale, 0};
    {
      int rc = density_gather_texture(v, s, &j.m.tex);
      if (rc) return rc;
    }
    j.sc = make_path_scene(p);
    attach_env(j.sc, v);  // escaped rays see the map; the light stays the job's directional light
    j.cam = make_camera(p);
    j.seed = p->seed;
    j.frame = p->sample_offset;
    {
      int rc = fill_tables(v, b.sampler == MR_SAMPLER_TEXTURE ? kSampTex : kSampGather, &j.tabs, s);
      if (rc) return rc;
    }
    j.srp = srp_of(to_f3(p->scatter_rate) / 1.001f);
    j.pix0 = off;
    j.npx = p->width * p->height;
    off += j.npx;
    ho[i] = BatchOut{J.out, to_f3(p->light_color), to_f3(p->scatter_rate)};
    if (distinct_channels(p)) b.spill = true;
  }
  b.total = off;
  b.wave = wave_pixels > 0 ? std::min<long long>(wave_pixels, b.total) : std::min<long long>(b.total, 4ll << 20);
  if (b.wave > (1ll << 28)) return set_error(MR_ERR_ARG, "wave of %lld pixels too large", b.wave);
  if (b.d_jobs) cudaFree(b.d_jobs);
  if (b.d_h0) cudaFree(b.d_h0);
  if (b.d_out) cudaFree(b.d_out);
  b.d_jobs = nullptr;
  b.d_h0 = nullptr;
  b.d_out = nullptr;
  MR_CUDA(cudaMalloc(&b.d_jobs, hj.size() * sizeof(BatchJob)));
  MR_CUDA(cudaMalloc(&b.d_h0, hj.size() * kPtTable * sizeof(float)));
  MR_CUDA(cudaMalloc(&b.d_out, ho.size() * sizeof(BatchOut)));
  if (!b.counters) MR_CUDA(cudaMalloc(&b.counters, kCounters * sizeof(unsigned long long)));
  MR_CUDA(cudaMemcpyAsync(b.d_jobs, hj.data(), hj.size() * sizeof(BatchJob), cudaMemcpyHostToDevice, s));
  MR_CUDA(cudaMemcpyAsync(b.d_out, ho.data(), ho.size() * sizeof(BatchOut), cudaMemcpyHostToDevice, s));
  int rc = batch_alloc_scratch(b, b.wave);
  if (rc) return rc;
  MR_CUDA(cudaStreamSynchronize(s));
  b.prepared = true;
  return MR_OK;
}

extern "C" int mr_batch_render(mr_batch* h, const mr_network* nh, void* stream) {
  clear_error();
  if (!h || !nh) return set_error(MR_ERR_ARG, "mr_batch_render: NULL argument");
  if (!h->b.prepared) return set_error(MR_ERR_STATE, "mr_batch_prepare first");
  return batch_launches(h->b, &nh->n, (cudaStream_t)stream);
}

extern "C" int mr_batch_autotune(mr_batch* h, const mr_network* nh, int64_t* host_wave, int32_t* host_trace_block,
                                 int32_t* host_gather_block, void* stream) {
  clear_error();
  if (!h || !nh) return set_error(MR_ERR_ARG, "mr_batch_autotune: NULL argument");
  Batch& b = h->b;
  if (!b.prepared) return set_error(MR_ERR_STATE, "mr_batch_prepare first");
  cudaStream_t s = (cudaStream_t)stream;
  b.drop_graph();
  cudaEvent_t e0, e1;
  MR_CUDA(cudaEventCreate(&e0));
  MR_CUDA(cudaEventCreate(&e1));
  auto timed = [&](float* ms) -> int {
    MR_CUDA(cudaEventRecord(e0, s));
    int rc = batch_launches(b, &nh->n, s);
    if (rc) return rc;
    MR_CUDA(cudaEventRecord(e1, s));
    MR_CUDA(cudaEventSynchronize(e1));
    MR_CUDA(cudaEventElapsedTime(ms, e0, e1));
    return MR_OK;
  };
  int rc = MR_OK;
  float best = 1e30f, ms = 0;
  // wave size first (default blocks), then the trace and gather block sizes
  const long long waves[] = {1ll << 20, 2ll << 20, 4ll << 20};
  long long best_wave = b.wave;
  for (long long w : waves) {
    const long long ww = std::min(w, b.total);
    if ((rc = batch_alloc_scratch(b, ww))) break;
    b.wave = ww;
    if ((rc = timed(&ms)) || (rc = timed(&ms))) break;
    if (ms < best) { best = ms; best_wave = ww; }
    if (ww == b.total) break;
  }
  b.wave = best_wave;
  const int blocks[] = {64, 128, 256};
  for (int pass = 0; pass < 2 && !rc; ++pass) {
    int* knob = pass == 0 ? &b.trace_block : &b.gather_block;
    int best_blk = *knob;
    best = 1e30f;
    for (int blk : blocks) {
      *knob = blk;
      if ((rc = timed(&ms)) || (rc = timed(&ms))) break;
      if (ms < best) { best = ms; best_blk = blk; }
    }
    *knob = best_blk;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc) return rc;
  if (host_wave) *host_wave = b.wave;
  if (host_trace_block) *host_trace_block = b.trace_block;
  if (host_gather_block) *host_gather_block = b.gather_block;
  return MR_OK;
}

extern "C" int mr_batch_capture(mr_batch* h, const mr_network* nh, void* stream) {
  clear_error();
  if (!h || !nh) return set_error(MR_ERR_ARG, "mr_batch_capture: NULL argument");
  Batch& b = h->b;
  if (!b.prepared) return set_error(MR_ERR_STATE, "mr_batch_prepare first");
  cudaStream_t s = (cudaStream_t)stream;
  if (s == nullptr) return set_error(MR_ERR_ARG, "graph capture needs a non-default stream");
  b.drop_graph();
  // one eager frame first: loads the modules and sets kernel attributes
  // outside the capture
  int rc = batch_launches(b, &nh->n, s);
  if (rc) return rc;
  MR_CUDA(cudaStreamSynchronize(s));
  MR_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  rc = batch_launches(b, &nh->n, s);
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaStreamEndCapture(s, &g);
  if (rc) {
    if (g) cudaGraphDestroy(g);
    return rc;
  }
  if (e != cudaSuccess) return cuda_error(e, "cudaStreamEndCapture");
  b.graph = g;
  e = cudaGraphInstantiate(&b.exec, g, 0);
  if (e != cudaSuccess) {
    b.drop_graph();
    return cuda_error(e, "cudaGraphInstantiate");
  }
  return MR_OK;
}

extern "C" int mr_batch_launch(mr_batch* h, void* stream) {
  clear_error();
  if (!h) return set_error(MR_ERR_ARG, "mr_batch_launch: NULL argument");
  if (!h->b.exec) return set_error(MR_ERR_STATE, "mr_batch_capture first");
  MR_CUDA(cudaGraphLaunch(h->b.exec, (cudaStream_t)stream));
  return MR_OK;
}

extern "C" int mr_batch_set_timing(mr_batch* h, int32_t enable) {
  clear_error();
  if (!h) return set_error(MR_ERR_ARG, "mr_batch_set_timing: NULL argument");
  Batch& b = h->b;
  if (!b.prepared) return set_error(MR_ERR_STATE, "mr_batch_prepare first");
  b.drop_graph();  // a captured graph holds the old event set
  b.drop_events();
  b.timing = enable != 0;
  if (!b.timing) return MR_OK;
  const size_t waves = (size_t)((b.total + b.wave - 1) / b.wave);
  MR_CUDA(cudaMalloc(&b.d_stamps, (waves + 1) * sizeof(unsigned long long)));
  MR_CUDA(cudaMemset(b.d_stamps, 0, (waves + 1) * sizeof(unsigned long long)));
  b.n_stamps = waves + 1;
  return MR_OK;
}

extern "C" int mr_batch_frame_times(mr_batch* h, float* host_ms, int32_t n) {
  clear_error();
  if (!h || !host_ms) return set_error(MR_ERR_ARG, "mr_batch_frame_times: NULL argument");
  Batch& b = h->b;
  if (!b.timing || !b.d_stamps) return set_error(MR_ERR_STATE, "mr_batch_set_timing(1) first");
  if (n != (int32_t)b.jobs.size()) return set_error(MR_ERR_ARG, "%d jobs, %d slots", (int)b.jobs.size(), n);
  MR_CUDA(cudaDeviceSynchronize());
  std::vector<unsigned long long> st(b.n_stamps);
  MR_CUDA(cudaMemcpy(st.data(), b.d_stamps, st.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost));
  if (st[0] == 0) return set_error(MR_ERR_STATE, "no batch frame has run since mr_batch_set_timing");
  long long pix = 0;
  for (int j = 0; j < n; ++j) {
    pix += (long long)b.jobs[j].p.width * b.jobs[j].p.height;
    const size_t w = (size_t)((pix - 1) / b.wave);  // the wave holding the job's last pixel
    host_ms[j] = (float)((double)(long long)(st[1 + w] - st[0]) * 1e-6);
  }
  return MR_OK;
}

extern "C" int mr_batch_counters(const mr_batch* h, uint64_t* host_out4) {
  clear_error();
  if (!h || !host_out4) return set_error(MR_ERR_ARG, "mr_batch_counters: NULL argument");
  if (!h->b.counters) return set_error(MR_ERR_STATE, "mr_batch_prepare first");
  unsigned long long c[kCounters];
  MR_CUDA(cudaMemcpy(c, h->b.counters, sizeof(c), cudaMemcpyDeviceToHost));
  for (int i = 0; i < 4; ++i) host_out4[i] = c[i];
  return MR_OK;
}
