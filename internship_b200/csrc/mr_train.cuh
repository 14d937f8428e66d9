// Training pieces shared by the fp32 training kernel (mr_train.cu) and the
// BF16 tensor-core head (mr_train_tc.cu): the offsets of the network's weight
// arrays per block, per-row dense layers with their backward passes, and the
// head's tail (core/radiancePredict.cu:370-485).
#pragma once
#include "mr_internal.h"
#include "mr_net_layout.cuh"

namespace mr {

struct TrainTables {
  int S[12], mode[12], from[12], pid[12], se0[12], se1[12], w[12][3], b[12][3];
  int l81w[3], l81b[3], ld41w[3], ld41b[3];
  int f1, f2, ggw, ggb, lc0w, lc0b, lc1w, lc1b, lc2w, lc2b, lxw, lxb, lxrw[12], lxrb[12], lx12w, lx12b;
};
constexpr TrainTables make_train_tables() {
  TrainTables t{};
  const WeightTable wt = make_weight_table();
  const int S[12] = {8, 8, 16, 16, 16, 32, 32, 32, 8, 8, 8, 8};
  const int mode[12] = {0, 2, 1, 1, 2, 1, 1, 1, 0, 1, 1, 1};
  const int from[12] = {0, 8, 16, 32, 48, 64, 96, 128, 160, 168, 176, 184};
  const int se0[12] = {MR_W_LSE01W, MR_W_LSE11W, MR_W_LSE21W, MR_W_LSE31W, MR_W_LSE41W, MR_W_LSE51W,
                       MR_W_LSE61W, MR_W_LSE71W, MR_W_LDSE01W, MR_W_LDSE11W, MR_W_LDSE21W, MR_W_LDSE31W};
  const int se1[12] = {MR_W_LSE02W, MR_W_LSE12W, MR_W_LSE22W, MR_W_LSE32W, MR_W_LSE42W, MR_W_LSE52W,
                       MR_W_LSE62W, MR_W_LSE72W, MR_W_LDSE02W, MR_W_LDSE12W, MR_W_LDSE22W, MR_W_LDSE32W};
  const int lw[12][3] = {{MR_W_L01W, MR_W_L_Tr01W, MR_W_L_Hg01W}, {MR_W_L11W, MR_W_L_Tr11W, MR_W_L_Hg11W},
                         {MR_W_L21W, MR_W_L_Tr21W, MR_W_L_Hg21W}, {MR_W_L31W, MR_W_L_Tr31W, MR_W_L_Hg31W},
                         {MR_W_L41W, MR_W_L_Tr41W, MR_W_L_Hg41W}, {MR_W_L51W, MR_W_L_Tr51W, MR_W_L_Hg51W},
                         {MR_W_L61W, MR_W_L_Tr61W, MR_W_L_Hg61W}, {MR_W_L71W, MR_W_L_Tr71W, MR_W_L_Hg71W},
                         {MR_W_LD01W, MR_W_LD_Tr01W, MR_W_LD_Hg01W}, {MR_W_LD11W, MR_W_LD_Tr11W, MR_W_LD_Hg11W},
                         {MR_W_LD21W, MR_W_LD_Tr21W, MR_W_LD_Hg21W}, {MR_W_LD31W, MR_W_LD_Tr31W, MR_W_LD_Hg31W}};
  const int lb[12][3] = {{MR_W_L01B, MR_W_L_Tr01B, MR_W_L_Hg01B}, {MR_W_L11B, MR_W_L_Tr11B, MR_W_L_Hg11B},
                         {MR_W_L21B, MR_W_L_Tr21B, MR_W_L_Hg21B}, {MR_W_L31B, MR_W_L_Tr31B, MR_W_L_Hg31B},
                         {MR_W_L41B, MR_W_L_Tr41B, MR_W_L_Hg41B}, {MR_W_L51B, MR_W_L_Tr51B, MR_W_L_Hg51B},
                         {MR_W_L61B, MR_W_L_Tr61B, MR_W_L_Hg61B}, {MR_W_L71B, MR_W_L_Tr71B, MR_W_L_Hg71B},
                         {MR_W_LD01B, MR_W_LD_Tr01B, MR_W_LD_Hg01B}, {MR_W_LD11B, MR_W_LD_Tr11B, MR_W_LD_Hg11B},
                         {MR_W_LD21B, MR_W_LD_Tr21B, MR_W_LD_Hg21B}, {MR_W_LD31B, MR_W_LD_Tr31B, MR_W_LD_Hg31B}};
  for (int i = 0; i < 12; ++i) {
    t.S[i] = S[i]; t.mode[i] = mode[i]; t.from[i] = from[i]; t.pid[i] = 3 * i;
    t.se0[i] = wt.off[se0[i]]; t.se1[i] = wt.off[se1[i]];
    for (int br = 0; br < 3; ++br) { t.w[i][br] = wt.off[lw[i][br]]; t.b[i][br] = wt.off[lb[i][br]]; }
  }
  const int l81w[3] = {MR_W_L81W, MR_W_L_Tr81W, MR_W_L_Hg81W}, l81b[3] = {MR_W_L81B, MR_W_L_Tr81B, MR_W_L_Hg81B};
  const int ld41w[3] = {MR_W_LD41W, MR_W_LD_Tr41W, MR_W_LD_Hg41W};
  const int ld41b[3] = {MR_W_LD41B, MR_W_LD_Tr41B, MR_W_LD_Hg41B};
  for (int br = 0; br < 3; ++br) {
    t.l81w[br] = wt.off[l81w[br]]; t.l81b[br] = wt.off[l81b[br]];
    t.ld41w[br] = wt.off[ld41w[br]]; t.ld41b[br] = wt.off[ld41b[br]];
  }
  t.f1 = wt.off[MR_W_LSEFin1W]; t.f2 = wt.off[MR_W_LSEFin2W];
  t.ggw = wt.off[MR_W_LGGSW]; t.ggb = wt.off[MR_W_LGGSB];
  t.lc0w = wt.off[MR_W_LC0W]; t.lc0b = wt.off[MR_W_LC0B]; t.lc1w = wt.off[MR_W_LC1W]; t.lc1b = wt.off[MR_W_LC1B];
  t.lc2w = wt.off[MR_W_LC2W]; t.lc2b = wt.off[MR_W_LC2B]; t.lxw = wt.off[MR_W_LXW]; t.lxb = wt.off[MR_W_LXB];
  const int rw[12] = {MR_W_LX0W, MR_W_LX1W, MR_W_LX2W, MR_W_LX3W, MR_W_LX4W, MR_W_LX5W,
                      MR_W_LX6W, MR_W_LX7W, MR_W_LX8W, MR_W_LX9W, MR_W_LX10W, MR_W_LX11W};
  const int rb[12] = {MR_W_LX0B, MR_W_LX1B, MR_W_LX2B, MR_W_LX3B, MR_W_LX4B, MR_W_LX5B,
                      MR_W_LX6B, MR_W_LX7B, MR_W_LX8B, MR_W_LX9B, MR_W_LX10B, MR_W_LX11B};
  for (int i = 0; i < 12; ++i) { t.lxrw[i] = wt.off[rw[i]]; t.lxrb[i] = wt.off[rb[i]]; }
  t.lx12w = wt.off[MR_W_LX12W]; t.lx12b = wt.off[MR_W_LX12B];
  return t;
}
static __constant__ TrainTables c_tt = make_train_tables();

__device__ __forceinline__ float relu(float x) { return x > 0.0f ? x : 0.0f; }
__device__ __forceinline__ float sigmoid(float x) { return 1.0f / (1.0f + expf(-x)); }

// Warp sum of v, added to G[idx] by lane 0. Every lane of the warp calls it
// with the same idx.
__device__ __forceinline__ void gacc(float* G, int idx, float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0 && v != 0.0f) atomicAdd(G + idx, v);
}

// ypre[o] = b[o] + sum_i W[o*K + i] x[i]
__device__ __forceinline__ void dense_fwd(const float* __restrict__ W, const float* __restrict__ B, const float* x,
                                          int K, int N, float* ypre) {
#pragma unroll 1
  for (int o = 0; o < N; ++o) {
    float a = 0.0f;
#pragma unroll 4
    for (int i = 0; i < K; ++i) a += x[i] * __ldg(W + o * K + i);
    ypre[o] = a + (B ? __ldg(B + o) : 0.0f);
  }
}
// Given dpre (N), input x (K): gradients of W (GW) and B (GB), and dx += W^T dpre
// (dx may be null).
__device__ __forceinline__ void dense_bwd(const float* __restrict__ W, float* GW, float* GB, const float* x,
                                          const float* dpre, float* dx, int K, int N) {
#pragma unroll 1
  for (int o = 0; o < N; ++o) {
    const float d = dpre[o];
    if (!__any_sync(0xffffffffu, d != 0.0f)) continue;  // dead unit for the whole warp
    if (GB) gacc(GB, o, d);
#pragma unroll 4
    for (int i = 0; i < K; ++i) gacc(GW, o * K + i, d * x[i]);
  }
  if (dx) {
#pragma unroll 1
    for (int i = 0; i < K; ++i) {
      float a = 0.0f;
#pragma unroll 4
      for (int o = 0; o < N; ++o) a += __ldg(W + o * K + i) * dpre[o];
      dx[i] += a;
    }
  }
}

// The head's tail (LX, the six residual pairs, LX12; radiancePredict.cu:454-473)
// for one row: forward from A3 (LC2's 32 outputs after ReLU), the loss
// (X - log(1 + label/srp))^2 / n summed over the warp into *loss, and the
// backward to d3 = dL/dA3; weight gradients go to G. Rows with valid false
// contribute nothing.
__device__ __forceinline__ void tail_fwd_bwd(const float* __restrict__ W, float* G, const TrainTables& T,
                                             const float* A3, float label, float srp, bool valid, float inv_batch,
                                             float* loss, float* d3) {
  float AXP[16];
  dense_fwd(W + T.lxw, W + T.lxb, A3, 32, 16, AXP);
  float AR[7][16], TP[6][16], TT[6][16], UP[6][16];
  for (int i = 0; i < 16; ++i) AR[0][i] = relu(AXP[i]);
#pragma unroll 1
  for (int r = 0; r < 6; ++r) {
    dense_fwd(W + T.lxrw[2 * r], W + T.lxrb[2 * r], AR[r], 16, 16, TP[r]);
    for (int i = 0; i < 16; ++i) TT[r][i] = relu(TP[r][i]);
    dense_fwd(W + T.lxrw[2 * r + 1], W + T.lxrb[2 * r + 1], TT[r], 16, 16, UP[r]);
    for (int i = 0; i < 16; ++i) AR[r + 1][i] = AR[r][i] + relu(UP[r][i]);
  }
  float OP;
  dense_fwd(W + T.lx12w, W + T.lx12b, AR[6], 16, 1, &OP);
  const float Xo = relu(OP);
  const float target = log1pf(fmaxf(label, 0.0f) / srp);
  const float err = valid ? Xo - target : 0.0f;
  {
    float l = err * err * inv_batch;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(loss, l);
  }
  float dOP = 2.0f * err * inv_batch * (OP > 0.0f ? 1.0f : 0.0f);
  float da[16];
  for (int i = 0; i < 16; ++i) da[i] = 0.0f;
  dense_bwd(W + T.lx12w, G + T.lx12w, G + T.lx12b, AR[6], &dOP, da, 16, 1);
#pragma unroll 1
  for (int r = 5; r >= 0; --r) {
    float du[16], dt[16], dtp[16];
    for (int i = 0; i < 16; ++i) { du[i] = UP[r][i] > 0.0f ? da[i] : 0.0f; dt[i] = 0.0f; }
    dense_bwd(W + T.lxrw[2 * r + 1], G + T.lxrw[2 * r + 1], G + T.lxrb[2 * r + 1], TT[r], du, dt, 16, 16);
    for (int i = 0; i < 16; ++i) dtp[i] = TP[r][i] > 0.0f ? dt[i] : 0.0f;
    dense_bwd(W + T.lxrw[2 * r], G + T.lxrw[2 * r], G + T.lxrb[2 * r], AR[r], dtp, da, 16, 16);  // da += W^T dtp
  }
  float dAX[16];
  for (int i = 0; i < 16; ++i) dAX[i] = AXP[i] > 0.0f ? da[i] : 0.0f;
  for (int i = 0; i < 32; ++i) d3[i] = 0.0f;
  dense_bwd(W + T.lxw, G + T.lxw, G + T.lxb, A3, dAX, d3, 32, 16);
}


}  // namespace mr
