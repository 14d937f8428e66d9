// FP32 radiance-predictor network, one thread per pixel, activations in
// registers (core/radiancePredict.cu:370-485 in fp32).
//
// Descriptors are read in chunks of 4 features: (row k, features 4j..4j+3) is
// the float4 at desc[k*rs + j*cs]; the render path passes chunk-of-4
// feature-major columns (rs = 4, cs = 4*capacity) so that a warp's
// 32 loads of one feature are one coalesced transaction. Every layer up to
// 32 wide is fully unrolled with compile-time register indices; the three
// branches of a block are evaluated together (three independent FMA chains),
// and blocks of equal width share one code instance through a runtime loop
// over their weight offsets. Weights are read as warp-uniform float4 loads.
// The 128-wide head vectors live in per-thread shared-memory columns.
#include "mr_internal.h"
#include "mr_net_layout.cuh"

namespace mr {

constexpr int kSimtThreads = 128;

struct SimtArgs {
  const float* __restrict__ w;
  const float* __restrict__ desc;
  const float* __restrict__ aux;
  long long rs, cs;      // desc strides (row, 4-feature chunk)
  long long ars, afs;    // aux strides
  int n;
  const unsigned* __restrict__ count;  // device row count (render path) or null
  float* out;                          // n x 3, or image (compose mode)
  const int* __restrict__ pix;
  const float* __restrict__ trph;
  F3 light_color, scatter;
  const int* job;        // batched compose: job of each record (null: single image)
  const BatchOut* bout;  // batched compose: per-job outputs
};

__device__ __forceinline__ float4 ldg4(const float* p) { return __ldg(reinterpret_cast<const float4*>(p)); }
__device__ __forceinline__ float relu0(float x) { return x >= 0.0f ? x : 0.0f; }

// y_b = ReLU(B_b + W_b x_b) for three branches b, S x S, bias first then
// ascending inputs (LinearReLU<S> / LinearReLU_SFL order).
template <int S>
__device__ __forceinline__ void dense3(const float (&x)[3][32], float (&y)[3][32], const float* __restrict__ w,
                                       int w0, int w1, int w2) {
  const float* W[3] = {w + w0, w + w1, w + w2};
#pragma unroll
  for (int i = 0; i < S; ++i) {
    float acc[3];
#pragma unroll
    for (int b = 0; b < 3; ++b) acc[b] = __ldg(W[b] + S * S + i);
#pragma unroll
    for (int j = 0; j < S; j += 4) {
#pragma unroll
      for (int b = 0; b < 3; ++b) {
        float4 q = ldg4(W[b] + i * S + j);
        acc[b] += x[b][j] * q.x;
        acc[b] += x[b][j + 1] * q.y;
        acc[b] += x[b][j + 2] * q.z;
        acc[b] += x[b][j + 3] * q.w;
      }
    }
#pragma unroll
    for (int b = 0; b < 3; ++b) y[b][i] = relu0(acc[b]);
  }
}

struct RowIO {
  const float* __restrict__ d;
  long long cs;
  // features i..i+3, i a multiple of 4
  __device__ __forceinline__ float4 ld4(int i) const {
    return __ldg(reinterpret_cast<const float4*>(d + (i >> 2) * cs));
  }
};

// SE / SERES block of width S (radiancePredict.cu:240-294). MODE 0: SE +
// ADD3, 1: SERES + ADD3, 2: SERES + REP3. Weight offsets are runtime values
// so that blocks of equal width and mode share this code.
template <int S, int MODE>
__device__ __forceinline__ void simt_block(const RowIO& in, const float* __restrict__ w, int from, int pid, int sew0,
                                           int sew1, int wa, int wb, int wc, float g, float gamma,
                                           float (&y)[3][32], float (&pool)[75]) {
  float mean[3], mx[3];
#pragma unroll
  for (int b = 0; b < 3; ++b) {
    float s = 0.0f, m = -10000.0f;
#pragma unroll
    for (int i = 0; i < S; i += 4) {
      const float4 q = in.ld4(b * 192 + from + i);
      s += q.x; s += q.y; s += q.z; s += q.w;
      m = fmaxf(m, q.x); m = fmaxf(m, q.y); m = fmaxf(m, q.z); m = fmaxf(m, q.w);
    }
    mean[b] = s / (float)S;
    mx[b] = m;
  }
  // pool[pid + b] and pool[36 + pid + b]: written through a small switch-free
  // store into the register array (pid is one of 12 known values).
#pragma unroll
  for (int q = 0; q < 36; q += 3)
    if (q == pid) {
#pragma unroll
      for (int b = 0; b < 3; ++b) { pool[q + b] = mean[b]; pool[36 + q + b] = mx[b]; }
    }
  float tmp[8] = {mean[0], mean[1], mean[2], mx[0], mx[1], mx[2], g, gamma};
  float h[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    float a = 0.0f;
#pragma unroll
    for (int j = 0; j < 8; ++j) a += tmp[j] * __ldg(w + sew0 + j + i * 8);
    h[i] = relu0(a);
  }
  float gate[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    float a = 0.0f;
#pragma unroll
    for (int j = 0; j < 8; ++j) a += h[j] * __ldg(w + sew1 + j + i * 8);
    gate[i] = 1.0f / (1.0f + expf(-a));
  }
  float x[3][32];
#pragma unroll
  for (int b = 0; b < 3; ++b)
#pragma unroll
    for (int i = 0; i < S; i += 4) {
      const float4 q = in.ld4(b * 192 + from + i);
      const float qv[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        float v = qv[u] * gate[b];
        x[b][i + u] = MODE == 0 ? v : v + y[b][i + u];
      }
    }
  float yn[3][32];
  dense3<S>(x, yn, w, wa, wb, wc);
#pragma unroll
  for (int b = 0; b < 3; ++b)
#pragma unroll
    for (int i = 0; i < S; i += 4) {
      const float4 q = in.ld4(b * 192 + from + i);
      const float qv[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        if (MODE == 2) {
          y[b][i + u] = yn[b][i + u];
          y[b][S + i + u] = qv[u];
        } else {
          y[b][i + u] = yn[b][i + u] + qv[u];
        }
      }
    }
}

// out[i] = ReLU(B[i] + sum_j in[j] W[i*FROM + j]): the FROM inputs are
// loaded into registers once (compile-time indices), the TO outputs are
// produced 8 per loop trip and stored with a runtime index.
template <int FROM, int TO>
__device__ __forceinline__ void dense_loc(const float* in, float* out, const float* __restrict__ W,
                                          const float* __restrict__ B) {
  float x[FROM];
#pragma unroll
  for (int j = 0; j < FROM; ++j) x[j] = in[j];
#pragma unroll 1
  for (int i0 = 0; i0 < TO; i0 += 8) {
    float acc[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) acc[q] = __ldg(B + i0 + q);
#pragma unroll
    for (int j = 0; j < FROM; j += 4) {
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        float4 wv = ldg4(W + (i0 + q) * FROM + j);
        acc[q] += x[j] * wv.x;
        acc[q] += x[j + 1] * wv.y;
        acc[q] += x[j + 2] * wv.z;
        acc[q] += x[j + 3] * wv.w;
      }
    }
#pragma unroll
    for (int q = 0; q < 8; ++q) out[i0 + q] = relu0(acc[q]);
  }
}

// 16 -> 16 layer in registers.
__device__ __forceinline__ void dense16(const float (&x)[16], float (&y)[16], const float* __restrict__ W,
                                        const float* __restrict__ B) {
#pragma unroll
  for (int i = 0; i < 16; ++i) {
    float acc = __ldg(B + i);
#pragma unroll
    for (int j = 0; j < 16; j += 4) {
      float4 q = ldg4(W + i * 16 + j);
      acc += x[j] * q.x;
      acc += x[j + 1] * q.y;
      acc += x[j + 2] * q.z;
      acc += x[j + 3] * q.w;
    }
    y[i] = relu0(acc);
  }
}

// Head SC(p) for one albedo channel (radiancePredict.cu:439-473) from the raw
// comb[0..120) and the pooled statistics; returns the pre-exponential X.
__device__ __noinline__ float simt_head(const float* comb, const float (&pool)[75], float srpc,
                                        const float* __restrict__ w) {
  float hA[128], hB[128];
#pragma unroll
  for (int i = 0; i < 120; ++i) hA[i] = comb[i];
#pragma unroll
  for (int i = 0; i < 8; ++i) {  // LGGS 3 -> 8, bias after the sum
    float acc = pool[72] * __ldg(w + WOFF(LGGSW) + 3 * i) + pool[73] * __ldg(w + WOFF(LGGSW) + 3 * i + 1) +
                srpc * __ldg(w + WOFF(LGGSW) + 3 * i + 2);
    acc += __ldg(w + WOFF(LGGSB) + i);
    hA[120 + i] = relu0(acc);
  }
  float sew[16];
#pragma unroll
  for (int j = 0; j < 16; ++j) {  // LSEFin1 75 -> 16 (pool[74] = srp)
    float acc = 0.0f;
#pragma unroll
    for (int i = 0; i < 74; ++i) acc += pool[i] * __ldg(w + WOFF(LSEFin1W) + j * 75 + i);
    acc += srpc * __ldg(w + WOFF(LSEFin1W) + j * 75 + 74);
    sew[j] = relu0(acc);
  }
  float sep[6];
#pragma unroll
  for (int i = 0; i < 6; ++i) {  // LSEFin2 16 -> 6
    float acc = 0.0f;
#pragma unroll
    for (int j = 0; j < 16; ++j) acc += sew[j] * __ldg(w + WOFF(LSEFin2W) + j + i * 16);
    sep[i] = 1.0f / (1.0f + expf(-acc));
  }
#pragma unroll
  for (int i = 0; i < 32; ++i) { hA[i] *= sep[0]; hA[32 + i] *= sep[1]; hA[64 + i] *= sep[2]; }
#pragma unroll
  for (int i = 0; i < 8; ++i) { hA[96 + i] *= sep[3]; hA[104 + i] *= sep[4]; hA[112 + i] *= sep[5]; }
  dense_loc<128, 128>(hA, hB, w + WOFF(LC0W), w + WOFF(LC0B));
  dense_loc<128, 64>(hB, hA, w + WOFF(LC1W), w + WOFF(LC1B));
  dense_loc<64, 32>(hA, hB, w + WOFF(LC2W), w + WOFF(LC2B));
  float x32[32];
#pragma unroll
  for (int i = 0; i < 32; ++i) x32[i] = hB[i];
  float a16[16];
#pragma unroll
  for (int i = 0; i < 16; ++i) {  // LX 32 -> 16
    float acc = __ldg(w + WOFF(LXB) + i);
#pragma unroll
    for (int j = 0; j < 32; j += 4) {
      float4 q = ldg4(w + WOFF(LXW) + i * 32 + j);
      acc += x32[j] * q.x;
      acc += x32[j + 1] * q.y;
      acc += x32[j + 2] * q.z;
      acc += x32[j + 3] * q.w;
    }
    a16[i] = relu0(acc);
  }
  const int lx[12] = {WOFF(LX0W), WOFF(LX1W), WOFF(LX2W), WOFF(LX3W), WOFF(LX4W), WOFF(LX5W),
                      WOFF(LX6W), WOFF(LX7W), WOFF(LX8W), WOFF(LX9W), WOFF(LX10W), WOFF(LX11W)};
#pragma unroll 1
  for (int r = 0; r < 6; ++r) {  // residual pairs (:454-471)
    float b16[16], c16[16];
    dense16(a16, b16, w + lx[2 * r], w + lx[2 * r] + 256);
    dense16(b16, c16, w + lx[2 * r + 1], w + lx[2 * r + 1] + 256);
#pragma unroll
    for (int i = 0; i < 16; ++i) a16[i] = a16[i] + c16[i];
  }
  float o = 0.0f;  // LX12 16 -> 1, bias after the sum
#pragma unroll
  for (int i = 0; i < 16; ++i) o += a16[i] * __ldg(w + WOFF(LX12W) + i);
  o += __ldg(w + WOFF(LX12B));
  return relu0(o);
}

__global__ void __launch_bounds__(kSimtThreads) k_mlp_simt(SimtArgs a) {
  const int n = a.count ? (int)min(*a.count, (unsigned)a.n) : a.n;
  const int k = blockIdx.x * kSimtThreads + threadIdx.x;
  if (k >= n) return;
  const float* __restrict__ w = a.w;
  RowIO in{a.desc + (long long)k * a.rs, a.cs};
  const float* ax = a.aux + (long long)k * a.ars;
  const float g = __ldg(ax), gamma = __ldg(ax + a.afs);
  const float srp[3] = {__ldg(ax + 2 * a.afs), __ldg(ax + 3 * a.afs), __ldg(ax + 4 * a.afs)};
  float pool[75];
  float y[3][32];
#pragma unroll
  for (int b = 0; b < 3; ++b)
#pragma unroll
    for (int i = 0; i < 32; ++i) y[b][i] = 0.0f;
  pool[72] = g;
  pool[73] = gamma;
  pool[74] = 0.0f;
  // main trunk (radiancePredict.cu:396-421)
  simt_block<8, 0>(in, w, 0, 0, WOFF(LSE01W), WOFF(LSE02W), WOFF(L01W), WOFF(L_Tr01W), WOFF(L_Hg01W), g, gamma, y, pool);
  simt_block<8, 2>(in, w, 8, 3, WOFF(LSE11W), WOFF(LSE12W), WOFF(L11W), WOFF(L_Tr11W), WOFF(L_Hg11W), g, gamma, y, pool);
  {
    const int p16[2][5] = {{WOFF(LSE21W), WOFF(LSE22W), WOFF(L21W), WOFF(L_Tr21W), WOFF(L_Hg21W)},
                           {WOFF(LSE31W), WOFF(LSE32W), WOFF(L31W), WOFF(L_Tr31W), WOFF(L_Hg31W)}};
#pragma unroll 1
    for (int b = 0; b < 2; ++b)
      simt_block<16, 1>(in, w, 16 + 16 * b, 6 + 3 * b, p16[b][0], p16[b][1], p16[b][2], p16[b][3], p16[b][4], g,
                        gamma, y, pool);
  }
  simt_block<16, 2>(in, w, 48, 12, WOFF(LSE41W), WOFF(LSE42W), WOFF(L41W), WOFF(L_Tr41W), WOFF(L_Hg41W), g, gamma, y,
                    pool);
  {
    const int p32[3][5] = {{WOFF(LSE51W), WOFF(LSE52W), WOFF(L51W), WOFF(L_Tr51W), WOFF(L_Hg51W)},
                           {WOFF(LSE61W), WOFF(LSE62W), WOFF(L61W), WOFF(L_Tr61W), WOFF(L_Hg61W)},
                           {WOFF(LSE71W), WOFF(LSE72W), WOFF(L71W), WOFF(L_Tr71W), WOFF(L_Hg71W)}};
#pragma unroll 1
    for (int b = 0; b < 3; ++b)
      simt_block<32, 1>(in, w, 64 + 32 * b, 15 + 3 * b, p32[b][0], p32[b][1], p32[b][2], p32[b][3], p32[b][4], g,
                        gamma, y, pool);
  }
  float comb[120];
  {  // L81: comb[0..96)
    float c3[3][32];
    dense3<32>(y, c3, w, WOFF(L81W), WOFF(L_Tr81W), WOFF(L_Hg81W));
#pragma unroll
    for (int b = 0; b < 3; ++b)
#pragma unroll
      for (int i = 0; i < 32; ++i) comb[32 * b + i] = c3[b][i];
  }
  // light-direction trunk (:424-437)
  simt_block<8, 0>(in, w, 160, 24, WOFF(LDSE01W), WOFF(LDSE02W), WOFF(LD01W), WOFF(LD_Tr01W), WOFF(LD_Hg01W), g, gamma,
                   y, pool);
  {
    const int pd[3][5] = {{WOFF(LDSE11W), WOFF(LDSE12W), WOFF(LD11W), WOFF(LD_Tr11W), WOFF(LD_Hg11W)},
                          {WOFF(LDSE21W), WOFF(LDSE22W), WOFF(LD21W), WOFF(LD_Tr21W), WOFF(LD_Hg21W)},
                          {WOFF(LDSE31W), WOFF(LDSE32W), WOFF(LD31W), WOFF(LD_Tr31W), WOFF(LD_Hg31W)}};
#pragma unroll 1
    for (int b = 0; b < 3; ++b)
      simt_block<8, 1>(in, w, 168 + 8 * b, 27 + 3 * b, pd[b][0], pd[b][1], pd[b][2], pd[b][3], pd[b][4], g, gamma, y,
                       pool);
  }
  {  // LD41: comb[96..120)
    float c3[3][32];
    dense3<8>(y, c3, w, WOFF(LD41W), WOFF(LD_Tr41W), WOFF(LD_Hg41W));
#pragma unroll
    for (int b = 0; b < 3; ++b)
#pragma unroll
      for (int i = 0; i < 8; ++i) comb[96 + 8 * b + i] = c3[b][i];
  }
  // heads per distinct albedo channel (:475-483)
  float X = simt_head(comb, pool, srp[0], w), Y, Z;
  if (srp[1] == srp[0]) Y = X; else Y = simt_head(comb, pool, srp[1], w);
  if (srp[2] == srp[0]) Z = X;
  else if (srp[2] == srp[1]) Z = Y;
  else Z = simt_head(comb, pool, srp[2], w);
  float o[3] = {fmaxf(expf(X) - 1.0f, 0.0f) * srp[0], fmaxf(expf(Y) - 1.0f, 0.0f) * srp[1],
                fmaxf(expf(Z) - 1.0f, 0.0f) * srp[2]};
  if (a.pix) {
    const int px = a.pix[k];
    const float tr = a.trph[k];
    F3 lc = a.light_color, sc = a.scatter;
    float* dst = a.out;
    if (a.job) {
      const BatchOut& bo = a.bout[a.job[k]];
      lc = bo.light_color;
      sc = bo.scatter;
      dst = bo.out;
    }
    dst[3 * (size_t)px + 0] = fmaxf(((o[0] + tr) * lc.x) * sc.x, 0.0f);
    dst[3 * (size_t)px + 1] = fmaxf(((o[1] + tr) * lc.y) * sc.y, 0.0f);
    dst[3 * (size_t)px + 2] = fmaxf(((o[2] + tr) * lc.z) * sc.z, 0.0f);
  } else {
#pragma unroll
    for (int c = 0; c < 3; ++c) a.out[3 * (size_t)k + c] = o[c];
  }
}

int launch_mlp_simt(const Network* net, const float* desc, const float* aux, long long rs, long long cs,
                    long long ars, long long afs, int n, const unsigned* count, float* out, const int* pix,
                    const float* trph, F3 light_color, F3 scatter, cudaStream_t s, const int* job,
                    const BatchOut* bout) {
  SimtArgs a;
  a.w = net->w;
  a.desc = desc;
  a.aux = aux;
  a.rs = rs;
  a.cs = cs;
  a.ars = ars;
  a.afs = afs;
  a.n = n;
  a.count = count;
  a.out = out;
  a.pix = pix;
  a.trph = trph;
  a.light_color = light_color;
  a.scatter = scatter;
  a.job = job;
  a.bout = bout;
  k_mlp_simt<<<(unsigned)((n + kSimtThreads - 1) / kSimtThreads), kSimtThreads, 0, s>>>(a);
  MR_CUDA(cudaGetLastError());
  return MR_OK;
}

}  // namespace mr
