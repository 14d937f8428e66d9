// Interactive rendering: VolumeRender::Render(float3*, Histogram*, unsigned*, ...)
// (core/volume.cu:57-145,181-295,469-547) as stream-ordered kernels.
//
//  * k_interactive_pt: one delta-tracking sample per pixel and frame (half the
//    pixels with the checkerboard option), running mean of the radiance and the
//    per-pixel histogram of x / (1 + x) (10 bins per channel) with running
//    means of the luminance l = sum(x / (1 + x)) and of l^2. The means are
//    kept as FP64 sums (the volume's moment buffer) and written to the fp32
//    accumulation and Histogram fields as sum / n, so that no rounding builds
//    up over the frames; the denoiser's variance E[l^2] - E[l]^2 is taken
//    from the same FP64 sums.
//  * k_denoise: the histogram-weighted 11 x 11 filter of Denoise<true>
//    (weights max(0, 1 - 1.2 Compare(h_center, h_neighbour)) where the
//    luminance variance exceeds 0.01), the frame-0 checkerboard fill, exposure,
//    Gamma / ACES tone mapping and the 0xAARRGGBB pack. A 16 x 16 tile of
//    output pixels stages its 26 x 26 halo of histograms and colours in shared
//    memory, so each histogram is read from memory once per tile instead of
//    121 times.
//  * k_reproject / k_reproject_pack: the neural mode's temporal reuse
//    (RenderCamera<true> + ReprojectionDenoise): this frame's radiance blended
//    with the previous frame's colour at the reprojected pixel, the result
//    kept in the histogram's three scalar fields as the next frame's history.
#include <algorithm>
#include <cfloat>

#include "mr_internal.h"
#include "mr_track.cuh"

namespace mr {

constexpr int kBins = 10;  // HISTO_SIZE (core/volume.hpp:12)

// ---- tone mapping (core/render.cuh:640-732) --------------------------------------
// ACES: sRGB -> AP0 -> AP1 (ACEScg), desaturation, the fitted RRT + ODT
// rational tonescale, dim-surround gamma on Y, desaturation, AP1 -> XYZ,
// D60 -> D65 and XYZ -> Rec.709 (the ACES colour-space matrices), then gamma 2.2.
struct M3 { float m[9]; };
__device__ __forceinline__ F3 mul(const M3& a, F3 x) {
  return f3(a.m[0] * x.x + a.m[1] * x.y + a.m[2] * x.z, a.m[3] * x.x + a.m[4] * x.y + a.m[5] * x.z,
            a.m[6] * x.x + a.m[7] * x.y + a.m[8] * x.z);
}
__device__ __forceinline__ F3 gamma22(F3 c) {
  return f3(powf(fmaxf(c.x, 0.0f), 1.0f / 2.2f), powf(fmaxf(c.y, 0.0f), 1.0f / 2.2f),
            powf(fmaxf(c.z, 0.0f), 1.0f / 2.2f));
}
__device__ F3 aces(F3 c) {
  const M3 srgb_ap0{{0.4397010f, 0.3829780f, 0.1773350f, 0.0897923f, 0.8134230f, 0.0967616f, 0.0175440f, 0.1115440f,
                     0.8707040f}};
  const M3 ap0_ap1{{1.4514393161f, -0.2365107469f, -0.2149285693f, -0.0765537734f, 1.1762296998f, -0.0996759264f,
                    0.0083161484f, -0.0060324498f, 0.9977163014f}};
  const M3 ap1_xyz{{0.6624541811f, 0.1340042065f, 0.1561876870f, 0.2722287168f, 0.6740817658f, 0.0536895174f,
                    -0.0055746495f, 0.0040607335f, 1.0103391003f}};
  const M3 xyz_ap1{{1.6410233797f, -0.3248032942f, -0.2364246952f, -0.6636628587f, 1.6153315917f, 0.0167563477f,
                    0.0117218943f, -0.0082844420f, 0.9883948585f}};
  const M3 d60_d65{{0.98722400f, -0.00611327f, 0.0159533f, -0.00759836f, 1.00186000f, 0.0053302f, 0.00307257f,
                    -0.00509595f, 1.0816800f}};
  const M3 xyz_709{{3.2409699419f, -1.5373831776f, -0.4986107603f, -0.9692436363f, 1.8759675015f, 0.0415550574f,
                    0.0556300797f, -0.2039769589f, 1.0569715142f}};
  const F3 ap1_y = f3(0.272229f, 0.674082f, 0.0536895f);
  F3 x = mul(ap0_ap1, mul(srgb_ap0, c));
  float y = dot(x, ap1_y);
  x = f3(y, y, y) * (1.0f - 0.96f) + x * 0.96f;
  x = f3((x.x * (x.x * 278.5085f + 10.7772f)) / (x.x * (x.x * 293.6045f + 88.7122f) + 80.6889f),
         (x.y * (x.y * 278.5085f + 10.7772f)) / (x.y * (x.y * 293.6045f + 88.7122f) + 80.6889f),
         (x.z * (x.z * 278.5085f + 10.7772f)) / (x.z * (x.z * 293.6045f + 88.7122f) + 80.6889f));
  // dark -> dim surround on xyY
  F3 XYZ = mul(ap1_xyz, x);
  const float div = fmaxf(XYZ.x + XYZ.y + XYZ.z, 1e-4f);
  const float cx = XYZ.x / div, cy = XYZ.y / div;
  const float Y = powf(fminf(fmaxf(XYZ.y, 0.0f), 65504.0f), 0.9811f);
  const float m = Y / fmaxf(cy, 1e-4f);
  x = mul(xyz_ap1, f3(cx * m, Y, (1.0f - cx - cy) * m));
  y = dot(x, ap1_y);
  x = f3(y, y, y) * (1.0f - 0.93f) + x * 0.93f;
  return gamma22(mul(xyz_709, mul(d60_d65, mul(ap1_xyz, x))));
}

__device__ __forceinline__ uint32_t pack_bgra(F3 res, float exposure, int tone) {
  F3 v = res * exposure;
  if (tone == 1) v = gamma22(v);
  else if (tone == 2) v = aces(v);
  const uint32_t r = (uint32_t)(255.0f * fminf(fmaxf(v.x, 0.0f), 1.0f));
  const uint32_t g = (uint32_t)(255.0f * fminf(fmaxf(v.y, 0.0f), 1.0f));
  const uint32_t b = (uint32_t)(255.0f * fminf(fmaxf(v.z, 0.0f), 1.0f));
  return 0xff000000u | (r << 16) | (g << 8) | b;
}

// ---- per-frame delta tracking with histograms -------------------------------------

struct InterArgs {
  Medium m;
  PathScene sc;
  CameraModel cam;
  uint32_t seed;
  int frame, fnum, checker, flip;
  float* accum;
  mr_histogram* hist;
  double* mom;  // 5 x npx FP64 sums: r, g, b, l, l^2
  size_t npx;
};

// Rebuilds the FP64 sums from the fp32 state (accum and the Histogram's count
// and means) when the moment buffer is new for this histogram buffer while an
// accumulation is under way (frame_index > 0).
__global__ void k_seed_moments(const float* __restrict__ accum, const mr_histogram* __restrict__ hist,
                               double* __restrict__ mom, size_t npx) {
  const size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (p >= npx) return;
  const double n = (double)hist[p].total_samples;
  for (int c = 0; c < 3; ++c) mom[c * npx + p] = (double)accum[3 * p + c] * n;
  mom[3 * npx + p] = (double)hist[p].x * n;
  mom[4 * npx + p] = (double)hist[p].x2 * n;
}

__global__ void __launch_bounds__(128) k_interactive_pt(InterArgs a) {
  const int W = a.cam.width, H = a.cam.height;
  const int per_row = a.checker ? (W + 1) / 2 : W;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= per_row * H) return;
  const int row = t / per_row, c = t - row * per_row;
  const int col = a.checker ? 2 * c + ((row + a.flip) & 1) : c;
  if (col >= W) return;
  const int pix = row * W + col;
  TrackStats st{0, 0};
  Rng rng;
  rng.init(a.seed, (uint32_t)pix, (uint32_t)a.frame, TAG_PT);
  const float jx = rng.next(), jy = rng.next();
  float tt;
  F3 L = path_radiance(a.m, a.sc, rng, a.cam.ori, camera_dir(a.cam, row, col, jx, jy), &tt, st);
  L = vmax(L, f3(0, 0, 0));
  mr_histogram& h = a.hist[pix];
  double* m = a.mom + pix;
  const size_t N = a.npx;
  if (a.fnum == 0) {
    for (int i = 0; i < 3 * kBins; ++i) h.bin[i] = 0.0f;
    h.total_samples = 0.0f;
    h.x2 = 0.0f;
    h.x = 0.0f;
    for (int k = 0; k < 5; ++k) m[k * N] = 0.0;
  }
  const F3 r = f3(L.x / (L.x + 1.0f), L.y / (L.y + 1.0f), L.z / (L.z + 1.0f));
  h.total_samples += 1.0f;
  h.bin[(int)floorf(fminf(r.x, 0.999f) * kBins)] += 1.0f;
  h.bin[(int)floorf(fminf(r.y, 0.999f) * kBins) + kBins] += 1.0f;
  h.bin[(int)floorf(fminf(r.z, 0.999f) * kBins) + 2 * kBins] += 1.0f;
  const float l = r.x + r.y + r.z;
  // FP64 sums; the fp32 fields hold sum / n, n = fnum + 1 (the reference's
  // running means with rate 1 / (1 + fnum))
  const double s0 = m[0] + (double)L.x, s1 = m[N] + (double)L.y, s2 = m[2 * N] + (double)L.z;
  const double s3 = m[3 * N] + (double)l, s4 = m[4 * N] + (double)l * (double)l;
  m[0] = s0;
  m[N] = s1;
  m[2 * N] = s2;
  m[3 * N] = s3;
  m[4 * N] = s4;
  const double inv = 1.0 / (double)(1 + a.fnum);
  float* acc = a.accum + 3 * (size_t)pix;
  acc[0] = (float)(s0 * inv);
  acc[1] = (float)(s1 * inv);
  acc[2] = (float)(s2 * inv);
  h.x = (float)(s3 * inv);
  h.x2 = (float)(s4 * inv);
}

// ---- denoise + tone map + pack ----------------------------------------------------

constexpr int kTile = 16, kHalo = 5, kSpan = kTile + 2 * kHalo;  // 26
constexpr int kHistFloats = 3 * kBins + 3;                       // 33
// One staged halo pixel: its histogram (bins, total, x2, x) then its colour,
// 36 floats (144 bytes), so every record starts on a 16-byte boundary.
constexpr int kRec = kHistFloats + 3;
// records, nonzero-bin masks, (sqrt n, 1 / sqrt n) of each record's count
constexpr int kDenoiseSmem = kSpan * kSpan * (kRec + 3) * (int)sizeof(float);

__device__ __forceinline__ void cp_async4(float* dst, const float* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"((unsigned)__cvta_generic_to_shared(dst)), "l"(src)
               : "memory");
}

// Packed fp32 pairs (the sm_100 .f32x2 forms of add, mul and fma: two
// independent fp32 operations, each rounded as its scalar form).
struct P2 { float x, y; };
__device__ __forceinline__ P2 add2(P2 a, P2 b) {
  P2 d;
  asm("{\n\t.reg .b64 a, b, d;\n\tmov.b64 a, {%2, %3};\n\tmov.b64 b, {%4, %5};\n\t"
      "add.rn.f32x2 d, a, b;\n\tmov.b64 {%0, %1}, d;\n\t}"
      : "=f"(d.x), "=f"(d.y) : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  return d;
}
__device__ __forceinline__ P2 mul2(P2 a, P2 b) {
  P2 d;
  asm("{\n\t.reg .b64 a, b, d;\n\tmov.b64 a, {%2, %3};\n\tmov.b64 b, {%4, %5};\n\t"
      "mul.rn.f32x2 d, a, b;\n\tmov.b64 {%0, %1}, d;\n\t}"
      : "=f"(d.x), "=f"(d.y) : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  return d;
}
__device__ __forceinline__ P2 fma2(P2 a, P2 b, P2 c) {
  P2 d;
  asm("{\n\t.reg .b64 a, b, c, d;\n\tmov.b64 a, {%2, %3};\n\tmov.b64 b, {%4, %5};\n\tmov.b64 c, {%6, %7};\n\t"
      "fma.rn.f32x2 d, a, b, c;\n\tmov.b64 {%0, %1}, d;\n\t}"
      : "=f"(d.x), "=f"(d.y) : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y), "f"(c.x), "f"(c.y));
  return d;
}
// 1 / y by the PTX approximate reciprocal, subnormals flushed to zero. A
// quotient x / y is taken as x * (1 / y), the form the PTX ISA gives for its
// approximate division (at most 2 ulp for y in [2^-126, 2^126]); a subnormal
// bin term is far below any weight's resolution.
__device__ __forceinline__ float rcp_approx_ftz(float y) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(y));
  return r;
}

// Compare (core/volume.cu:187-207): chi-square-like distance of two
// histograms normalised by their sample counts, averaged over the bins that
// are nonzero in either. cb / cn / cm: the centre's bins, count and
// nonzero-bin mask; nr / nm: a staged neighbour record and its mask. Bins are
// sample counts (>= 0), so a bin that is zero in both histograms adds
// t^2 / FLT_MIN with t = 0, exactly 0: the loop runs without a branch and adds
// a term for the same bins, in the same order, as the guarded loop of the
// reference, and p is the popcount of the joint mask. Bins go in pairs through the packed
// fp32 forms; the terms are still summed one by one in bin order. The count
// ratios sqrt(nn / cn) and sqrt(cn / nn) are taken as products of each
// count's staged sqrt(n) and 1 / sqrt(n) (cs: the centre's, ns: the
// neighbour's), and the mean over the p bins by an approximate division:
// each within a few ulp of the reference's divisions and roots.
__device__ __forceinline__ float compare(const float (&cb)[3 * kBins], float2 cs, uint32_t cm, const float* nr,
                                         float2 ns, uint32_t nm) {
  float hy[32];
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const float4 v = reinterpret_cast<const float4*>(nr)[k];
    hy[4 * k] = v.x; hy[4 * k + 1] = v.y; hy[4 * k + 2] = v.z; hy[4 * k + 3] = v.w;
  }
  const float syx = ns.x * cs.y, sxy = cs.x * ns.y;
  const P2 a2{syx, syx}, b2{-sxy, -sxy};
  float res = 0.0f;
#pragma unroll
  for (int i = 0; i < 3 * kBins; i += 2) {
    const P2 hx{cb[i], cb[i + 1]}, h{hy[i], hy[i + 1]};
    const P2 s = add2(hx, h);
    const P2 t = fma2(a2, hx, mul2(b2, h));  // syx hx - sxy h
    const P2 q = mul2(mul2(t, t), P2{rcp_approx_ftz(fmaxf(s.x, FLT_MIN)), rcp_approx_ftz(fmaxf(s.y, FLT_MIN))});
    res += q.x;
    res += q.y;
  }
  const float p = (float)__popc(cm | nm);
  return p == 0.0f ? 0.0f : res * rcp_approx_ftz(p);
}

struct DenoiseArgs {
  const float* accum;
  const mr_histogram* hist;
  uint32_t* out;
  int W, H, frame, flip, tone, denoise;
  float exposure;
  const double* mom;  // FP64 sums of l and l^2 (interactive path), or null: the Histogram's fp32 means
  size_t npx;
};

__global__ void __launch_bounds__(256, 2) k_denoise(DenoiseArgs a) {
  extern __shared__ __align__(16) float sm[];
  float* rec = sm;                                                           // kSpan^2 records
  uint32_t* msk = reinterpret_cast<uint32_t*>(sm + kSpan * kSpan * kRec);  // nonzero bins of each record
  float2* rsq = reinterpret_cast<float2*>(sm + kSpan * kSpan * (kRec + 1));  // (sqrt n, 1 / sqrt n) per record
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const int c0 = blockIdx.x * kTile - kHalo, r0 = blockIdx.y * kTile - kHalo;
  const bool filter = a.denoise && a.frame != 0;
  // stage the clamped halo (UnRoll, core/volume.cu:181-185) by asynchronous
  // 4-byte copies: every load is in flight at once
  for (int i = threadIdx.x; i < kSpan * kSpan * 3; i += blockDim.x) {
    const int q = i / 3, c = i - 3 * q;
    const int rr = min(max(r0 + q / kSpan, 0), a.H - 1), cc = min(max(c0 + q % kSpan, 0), a.W - 1);
    cp_async4(rec + q * kRec + kHistFloats + c, a.accum + 3 * ((size_t)rr * a.W + cc) + c);
  }
  if (filter) {
    for (int i = threadIdx.x; i < kSpan * kSpan * kHistFloats; i += blockDim.x) {
      const int q = i / kHistFloats, f = i - q * kHistFloats;
      const int rr = min(max(r0 + q / kSpan, 0), a.H - 1), cc = min(max(c0 + q % kSpan, 0), a.W - 1);
      cp_async4(rec + q * kRec + f, reinterpret_cast<const float*>(a.hist + (size_t)rr * a.W + cc) + f);
    }
  }
  asm volatile("cp.async.wait_all;\n" ::: "memory");
  __syncthreads();
  if (filter) {
    for (int q = threadIdx.x; q < kSpan * kSpan; q += blockDim.x) {
      const float4* r = reinterpret_cast<const float4*>(rec + q * kRec);
      uint32_t m = 0;
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const float4 v = r[k];
        const float e[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
        for (int j = 0; j < 4; ++j)
          if (4 * k + j < 3 * kBins) m |= (e[j] != 0.0f ? 1u : 0u) << (4 * k + j);
      }
      msk[q] = m;
      const float rn = sqrtf(rec[q * kRec + 3 * kBins]);
      rsq[q] = make_float2(rn, 1.0f / rn);
    }
    __syncthreads();
  }
  const int row = blockIdx.y * kTile + ty, col = blockIdx.x * kTile + tx;
  if (row >= a.H || col >= a.W) return;
  const int li = (ty + kHalo) * kSpan + (tx + kHalo);
  auto C = [&](int q) {
    const float* r = rec + q * kRec + kHistFloats;
    return f3(r[0], r[1], r[2]);
  };
  F3 res = C(li);
  if (a.frame == 0) {
    // checkerboard fill of the first frame (core/volume.cu:218-228)
    if ((((row + a.flip) & 1) + col) % 2 != 0) {
      // neighbours clamped at the image border
      const int up = row > 0 ? -kSpan : 0, dn = row < a.H - 1 ? kSpan : 0, lf = col > 0 ? -1 : 0,
                rt = col < a.W - 1 ? 1 : 0;
      res = (C(li + up) + C(li + dn) + C(li + lf) + C(li + rt)) / 4.0f;
    }
  } else if (filter) {
    const float* ch = rec + li * kRec;
    float variance;
    if (a.mom) {
      // |E[l^2] - E[l]^2| from the FP64 sums over the pixel's samples
      const size_t p = (size_t)row * a.W + col;
      const double n = (double)ch[3 * kBins];
      const double el = a.mom[3 * a.npx + p] / n, el2 = a.mom[4 * a.npx + p] / n;
      variance = (float)fabs(el2 - el * el);
    } else {
      variance = fabsf(ch[3 * kBins + 1] - ch[3 * kBins + 2] * ch[3 * kBins + 2]);
    }
    if (variance > 0.01f) {
      float cb[3 * kBins];
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const float4 v = reinterpret_cast<const float4*>(ch)[k];
        const float e[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
        for (int j = 0; j < 4; ++j)
          if (4 * k + j < 3 * kBins) cb[4 * k + j] = e[j];
      }
      const uint32_t cm = msk[li];
      const float2 cs = rsq[li];
      res = f3(0, 0, 0);
      float ws = 0.0f;
      for (int dr = -kHalo; dr <= kHalo; ++dr)
#pragma unroll
        for (int dc = -kHalo; dc <= kHalo; ++dc) {
          // the staged halo is already clamped, as UnRoll clamps
          const int q = li + dr * kSpan + dc;
          const float* nr = rec + q * kRec;
          const float w = fmaxf(0.0f, 1.0f - 1.2f * compare(cb, cs, cm, nr, rsq[q], msk[q]));
          const float4 cv = *reinterpret_cast<const float4*>(nr + 32);  // x, then the colour
          res = res + f3(cv.y, cv.z, cv.w) * w;
          ws += w;
        }
      res = res / ws;
    }
  }
  a.out[(size_t)row * a.W + col] = pack_bgra(res, a.exposure, a.tone);
}

// ---- neural mode: reprojection ------------------------------------------------------

struct ReprojArgs {
  CameraModel cam;
  F3 lori, lup, lright;  // previous camera
  uint32_t seed, frame;
  int fnum, checker;
  const float* rad;   // this frame's radiance W x H x 3
  const float* dist;  // first-hit distance, < 0 for escaped rays
  const mr_histogram* hist;
  float* accum;
};

// RenderCamera<true> (core/volume.cu:126-143): the pixel's first-hit point is
// projected into the previous camera; that pixel's stored colour is blended
// with this frame's radiance.
__global__ void k_reproject(ReprojArgs a) {
  const int W = a.cam.width, H = a.cam.height;
  const int pix = blockIdx.x * blockDim.x + threadIdx.x;
  if (pix >= W * H) return;
  const int row = pix / W, col = pix - row * W;
  Rng rng;
  rng.init(a.seed, (uint32_t)pix, a.frame, TAG_NN);
  const float jx = rng.next(), jy = rng.next();
  const F3 dir = camera_dir(a.cam, row, col, jx, jy);
  const float d = a.dist[pix];
  const bool sky = d < 0.0f;
  const float dis = fmaxf(0.001f, sky ? 10.0f : d);
  const F3 mp = a.cam.ori + dir * dis;
  F3 ld = mp - a.lori;
  const F3 lf = normalize(a.lori * -1.0f);
  ld = ld / dot(ld, lf);
  ld = ld - lf;
  // previous frame's pixel, in the same row-major convention as camera_dir
  const float lu = 0.5f - dot(ld, a.lright) / (2.0f * dot(a.lright, a.lright));
  const float lv = 0.5f - dot(ld, a.lup) / (2.0f * dot(a.lup, a.lup));
  const int lx = min(W - 1, max(0, (int)(lu * W))), ly = min(H - 1, max(0, (int)(lv * H)));
  const mr_histogram& h = a.hist[(size_t)ly * W + lx];
  const F3 his = f3(h.total_samples, h.x, h.x2);
  float rate = 1.0f / (float)(1 + a.fnum);
  if (!sky && !a.checker) rate = fminf(0.2f, rate);
  const F3 r = f3(a.rad[3 * (size_t)pix], a.rad[3 * (size_t)pix + 1], a.rad[3 * (size_t)pix + 2]);
  const F3 out = his * (1.0f - rate) + r * rate;
  a.accum[3 * (size_t)pix] = out.x;
  a.accum[3 * (size_t)pix + 1] = out.y;
  a.accum[3 * (size_t)pix + 2] = out.z;
}

// ReprojectionDenoise (core/volume.cu:266-287): keep the colour as history,
// tone map and pack.
__global__ void k_reproject_pack(const float* accum, mr_histogram* hist, uint32_t* out, int n, float exposure,
                                 int tone) {
  const int pix = blockIdx.x * blockDim.x + threadIdx.x;
  if (pix >= n) return;
  const F3 c = f3(accum[3 * (size_t)pix], accum[3 * (size_t)pix + 1], accum[3 * (size_t)pix + 2]);
  hist[pix].total_samples = c.x;
  hist[pix].x = c.y;
  hist[pix].x2 = c.z;
  out[pix] = pack_bgra(c, exposure, tone);
}

extern int check_params(const mr_render_params* p);
extern CameraModel make_camera(const mr_render_params* p);
extern PathScene make_path_scene(const mr_render_params* p);
int render_neural_dist(Volume* v, const Network* net, const mr_render_params* p, float* dev_rgb, float* dev_dist,
                       cudaStream_t s);

static int launch_denoise(const float* accum, const mr_histogram* hist, uint32_t* bgra, int W, int H,
                          const mr_interactive* it, cudaStream_t s, const double* mom = nullptr) {
  static DeviceCache attr;  // the attribute belongs to each device's context
  int rc = attr.once([] {
    MR_CUDA(cudaFuncSetAttribute(k_denoise, cudaFuncAttributeMaxDynamicSharedMemorySize, kDenoiseSmem));
    return (int)MR_OK;
  });
  if (rc) return rc;
  DenoiseArgs a{accum, hist, bgra, W, H, it->frame_index, it->frame_index & 1, it->tone, it->denoise, it->exposure,
                mom, (size_t)W * H};
  dim3 grid((W + kTile - 1) / kTile, (H + kTile - 1) / kTile);
  k_denoise<<<grid, 256, kDenoiseSmem, s>>>(a);
  MR_CUDA(cudaGetLastError());
  return MR_OK;
}

}  // namespace mr

using namespace mr;

static int check_interactive(const mr_interactive* it) {
  if (!it) return set_error(MR_ERR_ARG, "NULL interactive state");
  if (it->frame_index < 0) return set_error(MR_ERR_ARG, "frame_index < 0");
  if (it->tone < 0 || it->tone > 2) return set_error(MR_ERR_ARG, "tone must be 0 (none), 1 (gamma) or 2 (ACES)");
  if (!std::isfinite(it->exposure)) return set_error(MR_ERR_ARG, "exposure is not finite");
  return MR_OK;
}

extern "C" int mr_denoise(const float* dev_accum, const mr_histogram* dev_hist, uint32_t* dev_bgra, int32_t width,
                          int32_t height, const mr_interactive* it, void* stream) {
  clear_error();
  if (!dev_accum || !dev_bgra || (!dev_hist && it && it->denoise)) return set_error(MR_ERR_ARG, "mr_denoise: NULL argument");
  int rc = check_interactive(it);
  if (rc) return rc;
  if (width <= 0 || height <= 0) return set_error(MR_ERR_ARG, "bad size %d x %d", width, height);
  return launch_denoise(dev_accum, dev_hist, dev_bgra, width, height, it, (cudaStream_t)stream);
}

extern "C" int mr_render_interactive(mr_volume* h, const mr_network* net, const mr_render_params* p,
                                     const mr_interactive* it, float* dev_accum, mr_histogram* dev_hist,
                                     uint32_t* dev_bgra, void* stream) {
  clear_error();
  if (!h || !dev_accum || !dev_hist || !dev_bgra) return set_error(MR_ERR_ARG, "mr_render_interactive: NULL argument");
  int rc = check_params(p);
  if (rc) return rc;
  rc = check_interactive(it);
  if (rc) return rc;
  Volume* v = &h->v;
  if (!v->data_set || !v->mips_valid) return set_error(MR_ERR_STATE, "render before mr_volume_set_data / _update");
  cudaStream_t s = (cudaStream_t)stream;
  const int W = p->width, H = p->height;
  const int fnum = it->checkerboard ? it->frame_index / 2 : it->frame_index;
  if (p->render_type == MR_RT_PT) {
    InterArgs a;
    a.m = Medium{v->density, v->res, v->max_density, p->tr_scale, 0};
    rc = density_gather_texture(v, s, &a.m.tex);
    if (rc) return rc;
    a.sc = make_path_scene(p);
    attach_env(a.sc, v);
    a.cam = make_camera(p);
    a.seed = p->seed;
    a.frame = it->frame_index;
    a.fnum = fnum;
    a.checker = it->checkerboard ? 1 : 0;
    a.flip = it->frame_index & 1;
    a.accum = dev_accum;
    a.hist = dev_hist;
    // FP64 moment buffer of this histogram buffer (grown on demand; rebuilt
    // from the fp32 state when it is new mid-accumulation)
    const size_t npx = (size_t)W * H;
    const size_t need = 5 * npx * sizeof(double);
    bool fresh = v->mom_hist != (const void*)dev_hist || v->mom_npx != npx;
    if (v->mom_bytes < need) {
      if (v->mom) MR_CUDA(cudaFreeAsync(v->mom, s));
      v->mom = nullptr;
      v->mom_bytes = 0;
      cudaError_t e = cudaMallocAsync(&v->mom, need, s);
      if (e != cudaSuccess) return set_error(MR_ERR_NOMEM, "interactive moment buffer: %s", cudaGetErrorString(e));
      v->mom_bytes = need;
      fresh = true;
    }
    v->mom_hist = dev_hist;
    v->mom_npx = npx;
    if (fresh && it->frame_index > 0) {
      k_seed_moments<<<(unsigned)((npx + 127) / 128), 128, 0, s>>>(dev_accum, dev_hist, v->mom, npx);
      MR_CUDA(cudaGetLastError());
    }
    a.mom = v->mom;
    a.npx = npx;
    const int per_row = a.checker ? (W + 1) / 2 : W;
    const long long n = (long long)per_row * H;
    k_interactive_pt<<<(unsigned)((n + 127) / 128), 128, 0, s>>>(a);
    MR_CUDA(cudaGetLastError());
    return launch_denoise(dev_accum, dev_hist, dev_bgra, W, H, it, s, v->mom);
  }
  if (p->render_type != MR_RT_MRPNN) return set_error(MR_ERR_UNSUPPORTED, "render type %d", p->render_type);
  if (!net) return set_error(MR_ERR_ARG, "neural interactive render needs a network");
  // this frame's radiance and first-hit distances, then the reprojection
  const size_t npx = (size_t)W * H;
  const size_t need = npx * 4 * sizeof(float);
  if (v->inter_bytes < need) {
    if (v->inter) MR_CUDA(cudaFreeAsync(v->inter, s));
    v->inter = nullptr;
    v->inter_bytes = 0;
    cudaError_t e = cudaMallocAsync(&v->inter, need, s);
    if (e != cudaSuccess) return set_error(MR_ERR_NOMEM, "interactive buffer: %s", cudaGetErrorString(e));
    v->inter_bytes = need;
  }
  float* rad = (float*)v->inter;
  float* dist = rad + 3 * npx;
  mr_render_params q = *p;
  q.sample_offset = (uint32_t)it->frame_index;
  rc = render_neural_dist(v, &net->n, &q, rad, dist, s);
  if (rc) return rc;
  ReprojArgs a;
  a.cam = make_camera(p);
  a.lori = to_f3(it->prev_ori);
  a.lup = to_f3(it->prev_up);
  a.lright = to_f3(it->prev_right);
  a.seed = p->seed;
  a.frame = (uint32_t)it->frame_index;
  a.fnum = fnum;
  a.checker = it->checkerboard ? 1 : 0;
  a.rad = rad;
  a.dist = dist;
  a.hist = dev_hist;
  a.accum = dev_accum;
  k_reproject<<<(unsigned)((npx + 127) / 128), 128, 0, s>>>(a);
  MR_CUDA(cudaGetLastError());
  k_reproject_pack<<<(unsigned)((npx + 127) / 128), 128, 0, s>>>(dev_accum, dev_hist, dev_bgra, (int)npx,
                                                                it->exposure, it->tone);
  MR_CUDA(cudaGetLastError());
  return MR_OK;
}
