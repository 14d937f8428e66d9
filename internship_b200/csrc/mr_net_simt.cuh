// Per-thread fp32 evaluation of the radiance-predictor network
// (core/radiancePredict.cu:11-294, 370-485): one thread per pixel, the
// reference's arithmetic order (bias first, ascending inputs; LinearReLU with
// the bias last where the reference uses it). Weight reads are warp-uniform
// and served as broadcasts. This is the fp32 parity path.
#pragma once
#include "mr_device.cuh"
#include "mr_net_layout.cuh"

namespace mr {

struct NetSIMT {
  float xv[192], xs[192], xh[192];
  float a[160], b[160], c[160], a2[160], b2[160], c2[160];
  float pool[75], sew[16], sep[6], tmp[8], comb[128];
};

__device__ __forceinline__ float relu_(float x) { return x >= 0.0f ? x : 0.0f; }

__device__ __forceinline__ void n_avgmax(const float* in, float* out, int len, int at, int wa, int wm) {
  float s = 0.0f, m = -10000.0f;
  for (int i = 0; i < len; ++i) { s += in[at + i]; m = fmaxf(m, in[at + i]); }
  out[wa] = s / (float)len;
  out[wm] = m;
}
__device__ __forceinline__ void n_lin_relu_nobias(const float* in, float* out, int from, int to, int ra, int wa,
                                                  const float* __restrict__ W) {
  for (int i = 0; i < to; ++i) {
    float acc = 0.0f;
    for (int j = 0; j < from; ++j) acc += in[j + ra] * __ldg(W + j + i * from);
    out[i + wa] = relu_(acc);
  }
}
__device__ __forceinline__ void n_lin_sigmoid_nobias(const float* in, float* out, int from, int to, int ra, int wa,
                                                     const float* __restrict__ W) {
  for (int i = 0; i < to; ++i) {
    float acc = 0.0f;
    for (int j = 0; j < from; ++j) acc += in[j + ra] * __ldg(W + j + i * from);
    out[i + wa] = 1.0f / (1.0f + expf(-acc));
  }
}
__device__ __forceinline__ void n_lin_relu_bias_last(const float* in, float* out, int from, int to, int ra, int wa,
                                                     const float* __restrict__ W, const float* __restrict__ B) {
  for (int i = 0; i < to; ++i) {
    float acc = 0.0f;
    for (int j = 0; j < from; ++j) acc += in[j + ra] * __ldg(W + j + i * from);
    acc += __ldg(B + i);
    out[i + wa] = relu_(acc);
  }
}
template <int FROM, int TO>
__device__ __forceinline__ void n_lin_relu(const float* in, float* out, int ra, int wa, const float* __restrict__ W,
                                           const float* __restrict__ B) {
#pragma unroll 1
  for (int i = 0; i < TO; ++i) {
    float acc = __ldg(B + i);
#pragma unroll
    for (int j = 0; j < FROM; ++j) acc += in[j + ra] * __ldg(W + j + i * FROM);
    out[i + wa] = relu_(acc);
  }
}

constexpr int kPOOL = 36, kP_DI = 24, kDI = 160;

template <int SIZE>
__device__ __forceinline__ void n_se(NetSIMT& s, const float* __restrict__ w, int last, int from, int to, int pid,
                                     int sew0, int sew1, int ww, int trw, int hgw) {
  n_avgmax(s.xv, s.pool, SIZE, from, pid + 0, kPOOL + pid + 0);
  n_avgmax(s.xs, s.pool, SIZE, from, pid + 1, kPOOL + pid + 1);
  n_avgmax(s.xh, s.pool, SIZE, from, pid + 2, kPOOL + pid + 2);
  for (int i = 0; i < 3; ++i) { s.tmp[i] = s.pool[pid + i]; s.tmp[3 + i] = s.pool[kPOOL + pid + i]; }
  n_lin_relu_nobias(s.tmp, s.sew, 8, 8, 0, 0, w + sew0);
  n_lin_sigmoid_nobias(s.sew, s.sep, 8, 3, 0, 0, w + sew1);
  const float* srcs[3] = {s.xv, s.xs, s.xh};
  float* xs[3] = {s.a, s.b, s.c};
  float* ys[3] = {s.a2, s.b2, s.c2};
  const int wid[3] = {ww, trw, hgw};
#pragma unroll
  for (int br = 0; br < 3; ++br) {
    for (int i = 0; i < SIZE; ++i) xs[br][to + i] = srcs[br][from + i] * s.sep[br];
    if (last >= 0)
      for (int i = 0; i < SIZE; ++i) xs[br][to + i] = xs[br][to + i] + ys[br][last + i];
    n_lin_relu<SIZE, SIZE>(xs[br], ys[br], to, to, w + wid[br], w + wid[br] + SIZE * SIZE);
  }
}
__device__ __forceinline__ void n_add3(NetSIMT& s, int from, int to, int size) {
  for (int i = 0; i < size; ++i) {
    s.a2[to + i] = s.a2[to + i] + s.xv[from + i];
    s.b2[to + i] = s.b2[to + i] + s.xs[from + i];
    s.c2[to + i] = s.c2[to + i] + s.xh[from + i];
  }
}
__device__ __forceinline__ void n_rep3(NetSIMT& s, int from, int to, int size) {
  for (int i = 0; i < size; ++i) {
    s.a2[from + i] = s.a2[to + i];
    s.b2[from + i] = s.b2[to + i];
    s.c2[from + i] = s.c2[to + i];
  }
  for (int i = 0; i < size; ++i) {
    s.a2[to + i] = s.xv[to + i];
    s.b2[to + i] = s.xs[to + i];
    s.c2[to + i] = s.xh[to + i];
  }
}

// Trunks (radiancePredict.cu:385-437): fills comb[0..120) and pool[0..74).
__device__ __noinline__ void n_trunks(NetSIMT& s, const float* __restrict__ w, float g, float gamma) {
  s.tmp[6] = g;
  s.tmp[7] = gamma;
  s.pool[2 * kPOOL] = g;
  s.pool[2 * kPOOL + 1] = gamma;
  n_se<8>(s, w, -1, 0, 0, 0, WOFF(LSE01W), WOFF(LSE02W), WOFF(L01W), WOFF(L_Tr01W), WOFF(L_Hg01W));
  n_add3(s, 0, 0, 8);
  n_se<8>(s, w, 0, 8, 8, 3, WOFF(LSE11W), WOFF(LSE12W), WOFF(L11W), WOFF(L_Tr11W), WOFF(L_Hg11W));
  n_rep3(s, 0, 8, 8);
  n_se<16>(s, w, 0, 16, 16, 6, WOFF(LSE21W), WOFF(LSE22W), WOFF(L21W), WOFF(L_Tr21W), WOFF(L_Hg21W));
  n_add3(s, 16, 16, 16);
  n_se<16>(s, w, 16, 32, 32, 9, WOFF(LSE31W), WOFF(LSE32W), WOFF(L31W), WOFF(L_Tr31W), WOFF(L_Hg31W));
  n_add3(s, 32, 32, 16);
  n_se<16>(s, w, 32, 48, 48, 12, WOFF(LSE41W), WOFF(LSE42W), WOFF(L41W), WOFF(L_Tr41W), WOFF(L_Hg41W));
  n_rep3(s, 32, 48, 16);
  n_se<32>(s, w, 32, 64, 64, 15, WOFF(LSE51W), WOFF(LSE52W), WOFF(L51W), WOFF(L_Tr51W), WOFF(L_Hg51W));
  n_add3(s, 64, 64, 32);
  n_se<32>(s, w, 64, 96, 96, 18, WOFF(LSE61W), WOFF(LSE62W), WOFF(L61W), WOFF(L_Tr61W), WOFF(L_Hg61W));
  n_add3(s, 96, 96, 32);
  n_se<32>(s, w, 96, 128, 128, 21, WOFF(LSE71W), WOFF(LSE72W), WOFF(L71W), WOFF(L_Tr71W), WOFF(L_Hg71W));
  n_add3(s, 128, 128, 32);
  n_lin_relu<32, 32>(s.a2, s.comb, 128, 0, w + WOFF(L81W), w + WOFF(L81B));
  n_lin_relu<32, 32>(s.b2, s.comb, 128, 32, w + WOFF(L_Tr81W), w + WOFF(L_Tr81B));
  n_lin_relu<32, 32>(s.c2, s.comb, 128, 64, w + WOFF(L_Hg81W), w + WOFF(L_Hg81B));
  n_se<8>(s, w, -1, kDI + 0, 0, kP_DI + 0, WOFF(LDSE01W), WOFF(LDSE02W), WOFF(LD01W), WOFF(LD_Tr01W), WOFF(LD_Hg01W));
  n_add3(s, kDI + 0, 0, 8);
  n_se<8>(s, w, 0, kDI + 8, 8, kP_DI + 3, WOFF(LDSE11W), WOFF(LDSE12W), WOFF(LD11W), WOFF(LD_Tr11W), WOFF(LD_Hg11W));
  n_add3(s, kDI + 8, 8, 8);
  n_se<8>(s, w, 8, kDI + 16, 16, kP_DI + 6, WOFF(LDSE21W), WOFF(LDSE22W), WOFF(LD21W), WOFF(LD_Tr21W), WOFF(LD_Hg21W));
  n_add3(s, kDI + 16, 16, 8);
  n_se<8>(s, w, 16, kDI + 24, 24, kP_DI + 9, WOFF(LDSE31W), WOFF(LDSE32W), WOFF(LD31W), WOFF(LD_Tr31W), WOFF(LD_Hg31W));
  n_add3(s, kDI + 24, 24, 8);
  n_lin_relu<8, 8>(s.a2, s.comb, 24, 96, w + WOFF(LD41W), w + WOFF(LD41B));
  n_lin_relu<8, 8>(s.b2, s.comb, 24, 104, w + WOFF(LD_Tr41W), w + WOFF(LD_Tr41B));
  n_lin_relu<8, 8>(s.c2, s.comb, 24, 112, w + WOFF(LD_Hg41W), w + WOFF(LD_Hg41B));
}

// Head SC(p) (radiancePredict.cu:439-473) for one albedo channel.
__device__ __noinline__ float n_head(NetSIMT& s, const float* __restrict__ w, float srp) {
  s.pool[2 * kPOOL + 2] = srp;
  for (int i = 0; i < 120; ++i) s.a[i] = s.comb[i];
  n_lin_relu_bias_last(s.pool, s.a, 3, 8, 2 * kPOOL, 120, w + WOFF(LGGSW), w + WOFF(LGGSB));
  n_lin_relu_nobias(s.pool, s.sew, 75, 16, 0, 0, w + WOFF(LSEFin1W));
  n_lin_sigmoid_nobias(s.sew, s.sep, 16, 6, 0, 0, w + WOFF(LSEFin2W));
  for (int i = 0; i < 32; ++i) s.a[i] *= s.sep[0];
  for (int i = 0; i < 32; ++i) s.a[32 + i] *= s.sep[1];
  for (int i = 0; i < 32; ++i) s.a[64 + i] *= s.sep[2];
  for (int i = 0; i < 8; ++i) s.a[96 + i] *= s.sep[3];
  for (int i = 0; i < 8; ++i) s.a[104 + i] *= s.sep[4];
  for (int i = 0; i < 8; ++i) s.a[112 + i] *= s.sep[5];
  n_lin_relu<128, 128>(s.a, s.b, 0, 0, w + WOFF(LC0W), w + WOFF(LC0B));
  n_lin_relu<128, 64>(s.b, s.a, 0, 0, w + WOFF(LC1W), w + WOFF(LC1B));
  n_lin_relu<64, 32>(s.a, s.b, 0, 0, w + WOFF(LC2W), w + WOFF(LC2B));
  n_lin_relu<32, 16>(s.b, s.a, 0, 0, w + WOFF(LXW), w + WOFF(LXB));
  const int lx[12] = {WOFF(LX0W), WOFF(LX1W), WOFF(LX2W), WOFF(LX3W), WOFF(LX4W), WOFF(LX5W),
                      WOFF(LX6W), WOFF(LX7W), WOFF(LX8W), WOFF(LX9W), WOFF(LX10W), WOFF(LX11W)};
#pragma unroll 1
  for (int r = 0; r < 6; ++r) {
    n_lin_relu<16, 16>(s.a, s.b, 0, 0, w + lx[2 * r], w + lx[2 * r] + 256);
    n_lin_relu<16, 16>(s.b, s.c, 0, 0, w + lx[2 * r + 1], w + lx[2 * r + 1] + 256);
    for (int i = 0; i < 16; ++i) s.a[i] = s.a[i] + s.c[i];
  }
  n_lin_relu_bias_last(s.a, s.b, 16, 1, 0, 0, w + WOFF(LX12W), w + WOFF(LX12B));
  return s.b[0];
}

// Heads per distinct channel + output transform (radiancePredict.cu:475-485).
__device__ __forceinline__ F3 n_heads(NetSIMT& s, const float* __restrict__ w, F3 srp) {
  float X = n_head(s, w, srp.x), Y, Z;
  if (srp.y == srp.x) Y = X; else Y = n_head(s, w, srp.y);
  if (srp.z == srp.x) Z = X;
  else if (srp.z == srp.y) Z = Y;
  else Z = n_head(s, w, srp.z);
  return f3(fmaxf(expf(X) - 1.0f, 0.0f) * srp.x, fmaxf(expf(Y) - 1.0f, 0.0f) * srp.y,
            fmaxf(expf(Z) - 1.0f, 0.0f) * srp.z);
}

__host__ __device__ __forceinline__ F3 srp_of(F3 sr) {
  return f3((sr.x * sr.x) * (sr.x * sr.x), (sr.y * sr.y) * (sr.y * sr.y), (sr.z * sr.z) * (sr.z * sr.z));
}

}  // namespace mr
