// FP32 radiance-predictor network (core/radiancePredict.cu:370-485 in fp32),
// in four kernels over rows (tiles of 128 rows where shared state is tiled).
//
// Descriptors are read in chunks of 4 features: (row k, features 4j..4j+3) is
// the float4 at desc[k*rs + j*cs]; the render path passes chunk-of-4
// feature-major columns (rs = 4, cs = 4*capacity) so that a warp's 32 loads
// of one chunk are one coalesced transaction.
//
//  * k_simt_trunk (CUDA cores): the main trunk over a shared-memory tile,
//    column-major (feature f of tile row r at [f*128 + r]). The
//    squeeze-excitation statistics and gates and blocks 0 and 1 run per row
//    (one thread per row); the width-16 and width-32 layers and L81 (89 % of
//    the kernel's multiply-adds) run as register-tiled block GEMMs over the
//    tile, starting at the bias and adding the inputs in ascending order as
//    LinearReLU does, with their weights pre-transposed and double-buffered
//    in shared memory by cp.async.
//  * k_light_trunk (CUDA cores): the light-direction trunk and LD41, one
//    thread per row, weights as kernel parameters.
//  * k_tc32_head (tensor cores): the head. LC0 / LC1 / LC2 (53 % of all
//    multiply-adds) as tcgen05 MMAs whose every product is the sum of three
//    TF32 products (fp32-accurate); gates per row; LC2 outputs to staging.
//  * k_tc32_tail (CUDA cores): LX, the residual pairs, LX12 and the output,
//    one thread per row, weights as kernel parameters.
#include <algorithm>
#include <cstring>
#include <vector>

#include "mr_internal.h"
#include "mr_net_layout.cuh"
#include "mr_tcgen05.cuh"

namespace mr {

constexpr int kTile = 128;  // rows per tile

__device__ __forceinline__ float4 ldg4(const float* p) { return __ldg(reinterpret_cast<const float4*>(p)); }
__device__ __forceinline__ float relu0(float x) { return x >= 0.0f ? x : 0.0f; }

__device__ __forceinline__ void cp_async16(float* dst, const float* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"((unsigned)__cvta_generic_to_shared(dst)), "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }

// ---- weight image of the fp32 kernels -------------------------------------------------
// [trunk stages 0..6: blocks 2..7 of the main trunk and L81; per stage the
//  three branches' [in][out] weights, each followed by its bias]
constexpr int kTrunkStages = 7;
__host__ __device__ constexpr int stage_width(int g) { return g < 3 ? 16 : 32; }
__host__ __device__ constexpr int stage_floats(int g) { return 3 * (stage_width(g) * stage_width(g) + stage_width(g)); }
__host__ __device__ constexpr int stage_offset(int g) { return g <= 3 ? 816 * g : 2448 + 3168 * (g - 3); }
static_assert(stage_offset(1) == stage_floats(0) && stage_offset(4) == stage_offset(3) + stage_floats(3),
              "stage offsets");
// [squeeze-excitation blocks 0..11 (main trunk 0..7, light trunk 8..11): per
//  block kSeFloats = the LSEFin1 weights of its pool entries as [6][16] (mean
//  b0, max b0, mean b1, max b1, mean b2, max b2; 16 outputs), then SE1 8x8 and
//  SE2 3x8 row-major]
// [head per-row weights: LSEFin2 6x16, LSEFin1's albedo column (16), LGGS W
//  8x3 + B 8, LX12 W 16 + B 1, padded to kHeadRowFloats]
constexpr int kSeBlocks = 12, kSeFloats = 96 + 64 + 24;
constexpr int kSeOff = stage_offset(kTrunkStages);
constexpr int kHeadRowOff = kSeOff + kSeBlocks * kSeFloats;
constexpr int kHeadRowFloats = 96 + 16 + 32 + 20;
// [tensor-core head: LC0 / LC1 / LC2 as chunks of 32 input columns, each
//  chunk the TF32 part then the fp32 remainder of its N x 32 weights in the
//  canonical K-major layout (canon32); then the biases LC0B, LC1B, LC2B]
constexpr int kTcKC = 32;     // input columns per weight chunk
constexpr int kTcChunks = 10;  // per albedo channel: LC0 4, LC1 4, LC2 2
__host__ __device__ constexpr int tc_chunk_n(int c) { return c < 4 ? 128 : c < 8 ? 64 : 32; }
__host__ __device__ constexpr int tc_chunk_floats(int c) { return 2 * kTcKC * tc_chunk_n(c); }
__host__ __device__ constexpr int tc_chunk_off(int c) {
  return c < 4 ? 8192 * c : c < 8 ? 32768 + 4096 * (c - 4) : 49152 + 2048 * (c - 8);
}
constexpr int kTcHeadOff = (kHeadRowOff + kHeadRowFloats + 63) / 64 * 64;  // 256-byte aligned
constexpr int kTcBiasOff = kTcHeadOff + tc_chunk_off(kTcChunks);  // LC0B 128, LC1B 64, LC2B 32
constexpr int kSimtImage = kTcBiasOff + 224;
static_assert(kTcHeadOff % 64 == 0 && kTcBiasOff % 4 == 0, "image alignment");

// fp32 -> TF32 rounded to nearest, ties away from zero (cvt.rna.tf32.f32 on
// the device), for finite x.
static float tf32_rna(float x) {
  uint32_t u;
  std::memcpy(&u, &x, 4);
  u = (u + 0x1000u) & 0xFFFFE000u;
  float r;
  std::memcpy(&r, &u, 4);
  return r;
}
static_assert(kSeOff % 4 == 0 && kSeFloats % 4 == 0 && kHeadRowOff % 4 == 0, "float4 alignment");

void simt_weight_image(const float* w, std::vector<float>& img) {
  const WeightTable wt = make_weight_table();
  img.assign(kSimtImage, 0.0f);
  auto put_t = [&](size_t o, int id, int N, int K) {  // W[N][K] -> [K][N] at o
    const float* W = w + wt.off[id];
    for (int k = 0; k < K; ++k)
      for (int c = 0; c < N; ++c) img[o + (size_t)k * N + c] = W[(size_t)c * K + k];
  };
  const int ids[kTrunkStages][3][2] = {
      {{MR_W_L21W, MR_W_L21B}, {MR_W_L_Tr21W, MR_W_L_Tr21B}, {MR_W_L_Hg21W, MR_W_L_Hg21B}},
      {{MR_W_L31W, MR_W_L31B}, {MR_W_L_Tr31W, MR_W_L_Tr31B}, {MR_W_L_Hg31W, MR_W_L_Hg31B}},
      {{MR_W_L41W, MR_W_L41B}, {MR_W_L_Tr41W, MR_W_L_Tr41B}, {MR_W_L_Hg41W, MR_W_L_Hg41B}},
      {{MR_W_L51W, MR_W_L51B}, {MR_W_L_Tr51W, MR_W_L_Tr51B}, {MR_W_L_Hg51W, MR_W_L_Hg51B}},
      {{MR_W_L61W, MR_W_L61B}, {MR_W_L_Tr61W, MR_W_L_Tr61B}, {MR_W_L_Hg61W, MR_W_L_Hg61B}},
      {{MR_W_L71W, MR_W_L71B}, {MR_W_L_Tr71W, MR_W_L_Tr71B}, {MR_W_L_Hg71W, MR_W_L_Hg71B}},
      {{MR_W_L81W, MR_W_L81B}, {MR_W_L_Tr81W, MR_W_L_Tr81B}, {MR_W_L_Hg81W, MR_W_L_Hg81B}}};
  for (int g = 0; g < kTrunkStages; ++g) {
    const int S = stage_width(g);
    size_t o = stage_offset(g);
    for (int b = 0; b < 3; ++b) {
      put_t(o, ids[g][b][0], S, S);
      for (int c = 0; c < S; ++c) img[o + S * S + c] = w[wt.off[ids[g][b][1]] + c];
      o += S * S + S;
    }
  }
  const int se[kSeBlocks][2] = {{MR_W_LSE01W, MR_W_LSE02W}, {MR_W_LSE11W, MR_W_LSE12W}, {MR_W_LSE21W, MR_W_LSE22W},
                                {MR_W_LSE31W, MR_W_LSE32W}, {MR_W_LSE41W, MR_W_LSE42W}, {MR_W_LSE51W, MR_W_LSE52W},
                                {MR_W_LSE61W, MR_W_LSE62W}, {MR_W_LSE71W, MR_W_LSE72W}, {MR_W_LDSE01W, MR_W_LDSE02W},
                                {MR_W_LDSE11W, MR_W_LDSE12W}, {MR_W_LDSE21W, MR_W_LDSE22W},
                                {MR_W_LDSE31W, MR_W_LDSE32W}};
  const float* f1 = w + wt.off[MR_W_LSEFin1W];  // 16 x 75
  for (int blk = 0; blk < kSeBlocks; ++blk) {
    float* o = img.data() + kSeOff + blk * kSeFloats;
    const int pid = 3 * blk;
    for (int b = 0; b < 3; ++b)
      for (int j = 0; j < 16; ++j) {
        o[(2 * b) * 16 + j] = f1[j * 75 + pid + b];
        o[(2 * b + 1) * 16 + j] = f1[j * 75 + 36 + pid + b];
      }
    for (int i = 0; i < 64; ++i) o[96 + i] = w[wt.off[se[blk][0]] + i];
    for (int i = 0; i < 24; ++i) o[160 + i] = w[wt.off[se[blk][1]] + i];
  }
  float* hr = img.data() + kHeadRowOff;
  for (int i = 0; i < 96; ++i) hr[i] = w[wt.off[MR_W_LSEFin2W] + i];
  for (int j = 0; j < 16; ++j) hr[96 + j] = f1[j * 75 + 74];
  for (int i = 0; i < 24; ++i) hr[112 + i] = w[wt.off[MR_W_LGGSW] + i];
  for (int i = 0; i < 8; ++i) hr[136 + i] = w[wt.off[MR_W_LGGSB] + i];
  for (int i = 0; i < 16; ++i) hr[144 + i] = w[wt.off[MR_W_LX12W] + i];
  hr[160] = w[wt.off[MR_W_LX12B]];
  // tensor-core head
  const int lw[3] = {MR_W_LC0W, MR_W_LC1W, MR_W_LC2W}, lb[3] = {MR_W_LC0B, MR_W_LC1B, MR_W_LC2B};
  const int lk[3] = {128, 128, 64};
  int c = 0;
  for (int l = 0; l < 3; ++l) {
    const int N = tc_chunk_n(c), K = lk[l];
    const float* W = w + wt.off[lw[l]];  // W[N][K]
    for (int j = 0; j < K / kTcKC; ++j, ++c) {
      float* hi = img.data() + kTcHeadOff + tc_chunk_off(c);
      float* lo = hi + N * kTcKC;
      for (int nn = 0; nn < N; ++nn)
        for (int kl = 0; kl < kTcKC; ++kl) {
          const float x = W[(size_t)nn * K + kTcKC * j + kl], h = tf32_rna(x);
          hi[canon32(nn, kl, kTcKC) / 4] = h;
          lo[canon32(nn, kl, kTcKC) / 4] = x - h;
        }
    }
  }
  for (int i = 0; i < 128; ++i) img[kTcBiasOff + i] = w[wt.off[lb[0]] + i];
  for (int i = 0; i < 64; ++i) img[kTcBiasOff + 128 + i] = w[wt.off[lb[1]] + i];
  for (int i = 0; i < 32; ++i) img[kTcBiasOff + 192 + i] = w[wt.off[lb[2]] + i];
}

// ---- trunk ---------------------------------------------------------------------------

struct TrunkArgs {
  const float* __restrict__ w;
  const float* __restrict__ img;  // simt_weight_image
  const float* __restrict__ desc;
  const float* __restrict__ aux;
  long long rs, cs;    // desc strides (row, 4-feature chunk)
  long long ars, afs;  // aux strides
  int n;
  const unsigned* __restrict__ count;  // device row count (render path) or null
};

// Trunk outputs per row, handed from the trunk kernels to the head kernel:
// comb[0..120) (the L81 / LD41 outputs before gating), fin[0..16) (the
// LSEFin1 sums over pool[0..74), without the albedo term) and the head's
// gates of albedo channel 0 (6 + 2 unused, then the 8 LGGS outputs), 152
// values in chunks of 4: chunk c of row k is the float4 at t[k*rs + c*cs].
struct TrunkOut {
  float* t;
  long long rs, cs;
};

// One descriptor row; the address of each chunk is formed inside the asm so
// that the compiler does not keep a row address per feature live for reuse
// (each feature is read three times: statistics, block input, residual).
struct RowIO {
  const float* __restrict__ d;
  int cs16;  // chunk stride in bytes
  // features i..i+3, i a multiple of 4
  __device__ __forceinline__ float4 ld4(int i) const {
    float4 v;
    asm volatile(
        "{\n\t.reg .u64 a;\n\tmad.wide.s32 a, %4, %5, %6;\n\tld.global.nc.v4.f32 {%0,%1,%2,%3}, [a];\n\t}\n"
        : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
        : "r"(i >> 2), "r"(cs16), "l"(d));
    return v;
  }
};

// The running trunk state y of a row (3 branches x up to 32 values) in the
// tile, one column per thread: conflict-free.
struct YS {
  float* p;  // tile base + row
  __device__ __forceinline__ float& at(int b, int i) const { return p[(b * 32 + i) * kTile]; }
};

// yn = ReLU(B + W x) for one branch, S x S (bias stored after W): bias first,
// then ascending inputs (LinearReLU<S> order), four outputs interleaved.
template <int S>
__device__ __forceinline__ void dense1(const float* x, float* yn, const float* __restrict__ W) {
#pragma unroll
  for (int i0 = 0; i0 < S; i0 += 4) {
    float acc[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) acc[q] = __ldg(W + S * S + i0 + q);
#pragma unroll
    for (int j = 0; j < S; j += 4) {
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const float4 wv = ldg4(W + (i0 + q) * S + j);
        acc[q] += x[j] * wv.x;
        acc[q] += x[j + 1] * wv.y;
        acc[q] += x[j + 2] * wv.z;
        acc[q] += x[j + 3] * wv.w;
      }
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) yn[i0 + q] = relu0(acc[q]);
  }
}

// Squeeze-excitation of a block of width S (radiancePredict.cu:240-294):
// pooled statistics of the block input (mean, max per branch), which also go
// straight into the 16 LSEFin1 sums `fin` (pool[pid+b], pool[36+pid+b]), and
// the three branch gates.
template <int S>
__device__ __forceinline__ void se_gates(const RowIO& in, const float* __restrict__ sw, int from, float g,
                                         float gamma, float (&fin)[16], float (&gate)[3]) {
  float st[6];  // mean b0, max b0, mean b1, max b1, mean b2, max b2
#pragma unroll
  for (int b = 0; b < 3; ++b) {
    float s = 0.0f, m = -10000.0f;
#pragma unroll
    for (int i = 0; i < S; i += 4) {
      const float4 q = in.ld4(b * 192 + from + i);
      s += q.x; s += q.y; s += q.z; s += q.w;
      m = fmaxf(m, q.x); m = fmaxf(m, q.y); m = fmaxf(m, q.z); m = fmaxf(m, q.w);
    }
    st[2 * b] = s / (float)S;
    st[2 * b + 1] = m;
  }
  // LSEFin1 over this block's pool entries, in the order mean b, max b
#pragma unroll
  for (int k = 0; k < 6; ++k)
#pragma unroll
    for (int j = 0; j < 16; j += 4) {
      const float4 f = ldg4(sw + k * 16 + j);
      fin[j] += st[k] * f.x;
      fin[j + 1] += st[k] * f.y;
      fin[j + 2] += st[k] * f.z;
      fin[j + 3] += st[k] * f.w;
    }
  const float tmp[8] = {st[0], st[2], st[4], st[1], st[3], st[5], g, gamma};
  float h[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    float a = 0.0f;
#pragma unroll
    for (int j = 0; j < 8; j += 4) {
      const float4 q = ldg4(sw + 96 + i * 8 + j);
      a += tmp[j] * q.x;
      a += tmp[j + 1] * q.y;
      a += tmp[j + 2] * q.z;
      a += tmp[j + 3] * q.w;
    }
    h[i] = relu0(a);
  }
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    float a = 0.0f;
#pragma unroll
    for (int j = 0; j < 8; j += 4) {
      const float4 q = ldg4(sw + 160 + i * 8 + j);
      a += h[j] * q.x;
      a += h[j + 1] * q.y;
      a += h[j + 2] * q.z;
      a += h[j + 3] * q.w;
    }
    gate[i] = 1.0f / (1.0f + expf(-a));
  }
}

// Block of width 8, per row. MODE 0: SE + ADD3, 1: SERES + ADD3, 2: SERES +
// REP3. Weight offsets are runtime values so that blocks of equal mode share
// this code.
template <int MODE>
__device__ __forceinline__ void row_block8(const RowIO& in, const float* __restrict__ w, const float* __restrict__ sw,
                                           int from, int wa, int wb, int wc, float g, float gamma, const YS& y,
                                           float (&fin)[16]) {
  float gate[3];
  se_gates<8>(in, sw, from, g, gamma, fin, gate);
#pragma unroll 1
  for (int b = 0; b < 3; ++b) {
    const int wo = b == 0 ? wa : b == 1 ? wb : wc;
    const float gb = b == 0 ? gate[0] : b == 1 ? gate[1] : gate[2];
    float x[8], yn[8];
#pragma unroll
    for (int i = 0; i < 8; i += 4) {
      const float4 q = in.ld4(b * 192 + from + i);
      const float qv[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const float v = qv[u] * gb;
        x[i + u] = MODE == 0 ? v : v + y.at(b, i + u);
      }
    }
    dense1<8>(x, yn, w + wo);
#pragma unroll
    for (int i = 0; i < 8; i += 4) {
      const float4 q = in.ld4(b * 192 + from + i);
      const float qv[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        if (MODE == 2) {
          y.at(b, i + u) = yn[i + u];
          y.at(b, 8 + i + u) = qv[u];
        } else {
          y.at(b, i + u) = yn[i + u] + qv[u];
        }
      }
    }
  }
}

// Per-row half of a width-S SERES block run as a block GEMM: gates, then the
// layer input x = in * gate + y written over y in the tile.
template <int S>
__device__ __forceinline__ void row_gate_input(const RowIO& in, const float* __restrict__ sw, int from, float g,
                                               float gamma, const YS& y, float (&fin)[16]) {
  float gate[3];
  se_gates<S>(in, sw, from, g, gamma, fin, gate);
#pragma unroll
  for (int b = 0; b < 3; ++b) {
#pragma unroll 4
    for (int i = 0; i < S; i += 4) {
      const float4 q = in.ld4(b * 192 + from + i);
      const float qv[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const float v = qv[u] * gate[b];
        y.at(b, i + u) = v + y.at(b, i + u);
      }
    }
  }
}

// Trunk weight stage g into ring buffer g % 2 (one commit group per call,
// empty past the last stage).
__device__ __forceinline__ void trunk_stage_issue(const float* __restrict__ img, float* ring, int g) {
  if (g < kTrunkStages) {
    const float* src = img + stage_offset(g);
    float* dst = ring + (g & 1) * stage_floats(kTrunkStages - 1);
    const int pieces = stage_floats(g) / 4;
    for (int i = threadIdx.x; i < pieces; i += kTile) cp_async16(dst + 4 * i, src + 4 * i);
  }
  cp_async_commit();
}

// The three branch layers of a trunk stage of width S as block GEMMs over the
// tile: out_b = ReLU(B_b + W_b x_b), x_b = tile columns [32b, 32b+S). Thread
// t owns 4 consecutive columns (c0) and S/4 rows in quads: for S = 32 rows
// 4g..4g+3 and 64+4g..64+4g+3 (g = t % 16, c0 = 4 (t / 16)); for S = 16
// rows 4g..4g+3 (g = t % 32, c0 = 4 (t / 32)). Epilogue EPI 0: y = out + in
// (SERES + ADD3); 1: y[0..S) = out, y[S..2S) = in (SERES + REP3); 2: the
// outputs go to comb (L81).
template <int S, int EPI>
__device__ __forceinline__ void trunk_gemm(float* tile, const float* W, const float* __restrict__ desc, long long rs,
                                           long long cs, int row0, int n, int from, const TrunkOut& to) {
  constexpr int NQ = S / 16;            // row quads per thread
  constexpr int G = 32 / NQ;            // row groups
  constexpr int QS = kTile / NQ;        // distance between a thread's quads
  const int t = threadIdx.x, r0 = 4 * (t % G), c0 = 4 * (t / G);
#pragma unroll 1
  for (int b = 0; b < 3; ++b) {
    const float* X = tile + b * 32 * kTile;
    const float* Wb = W + b * (S * S + S);
    float acc[4 * NQ][4];
    {
      const float4 bias = *reinterpret_cast<const float4*>(Wb + S * S + c0);
#pragma unroll
      for (int i = 0; i < 4 * NQ; ++i) {
        acc[i][0] = bias.x; acc[i][1] = bias.y; acc[i][2] = bias.z; acc[i][3] = bias.w;
      }
    }
#pragma unroll 8
    for (int k = 0; k < S; ++k) {
      const float4 wv = *reinterpret_cast<const float4*>(Wb + k * S + c0);
      const float wa[4] = {wv.x, wv.y, wv.z, wv.w};
#pragma unroll
      for (int q = 0; q < NQ; ++q) {
        const float4 xv = *reinterpret_cast<const float4*>(X + k * kTile + q * QS + r0);
        const float xa[4] = {xv.x, xv.y, xv.z, xv.w};
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
          for (int j = 0; j < 4; ++j) acc[4 * q + i][j] = fmaf(xa[i], wa[j], acc[4 * q + i][j]);
      }
    }
    if (EPI != 2) __syncthreads();  // every read of x_b is done before y_b overwrites it
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
      const int rq = q * QS + r0;  // first of the quad's 4 rows
      float o[4][4];               // [row][column]
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) o[i][j] = relu0(acc[4 * q + i][j]);
      if (EPI == 2) {
#pragma unroll
        for (int i = 0; i < 4; ++i)
          if (row0 + rq + i < n)
            *reinterpret_cast<float4*>(to.t + (long long)(row0 + rq + i) * to.rs + (8 * b + c0 / 4) * to.cs) =
                make_float4(o[i][0], o[i][1], o[i][2], o[i][3]);
      } else {
        float iv[4][4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          const int row = row0 + rq + i, kr = row < n ? row : n - 1;
          const float4 v = ldg4(desc + (long long)kr * rs + ((b * 192 + from + c0) >> 2) * cs);
          iv[i][0] = v.x; iv[i][1] = v.y; iv[i][2] = v.z; iv[i][3] = v.w;
        }
        // one float4 of 4 rows per column: a quarter warp stores 128 contiguous bytes
        float* yc = tile + (b * 32 + c0) * kTile + rq;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          if (EPI == 0) {
            *reinterpret_cast<float4*>(yc + j * kTile) =
                make_float4(o[0][j] + iv[0][j], o[1][j] + iv[1][j], o[2][j] + iv[2][j], o[3][j] + iv[3][j]);
          } else {
            *reinterpret_cast<float4*>(yc + j * kTile) = make_float4(o[0][j], o[1][j], o[2][j], o[3][j]);
            *reinterpret_cast<float4*>(yc + (S + j) * kTile) = make_float4(iv[0][j], iv[1][j], iv[2][j], iv[3][j]);
          }
        }
      }
    }
  }
}

// L2 prefetch of descriptor features [f0, f1) of the three branches for the
// tile's rows, one bulk prefetch per 4-feature chunk (thread i issues chunk
// i), when each chunk's rows are contiguous (chunk-of-4 feature-major
// columns, rows 16 bytes apart).
__device__ __forceinline__ void desc_prefetch(const TrunkArgs& a, int row0, int n, int f0, int f1) {
  if (a.rs != 4) return;
  const int per = (f1 - f0) / 4, i = threadIdx.x;
  if (i >= 3 * per) return;
  const int chunk = (i / per) * 48 + f0 / 4 + i % per;
  const unsigned bytes = (unsigned)min(kTile, n - row0) * 16u;
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(a.desc + chunk * a.cs + row0 * 4), "r"(bytes)
               : "memory");
}

constexpr int kTrunkSmem = (96 * kTile + 2 * 3 * (32 * 32 + 32)) * (int)sizeof(float);

// Trunks of RadiancePredict (radiancePredict.cu:385-437) for a tile of 128
// rows, one thread per row in the per-row parts.
__device__ __forceinline__ void trunk_tile(const TrunkArgs& a, const TrunkOut& to, float* tile, float* ring, int row0,
                                           int n) {
  trunk_stage_issue(a.img, ring, 0);
  trunk_stage_issue(a.img, ring, 1);
  desc_prefetch(a, row0, n, 0, 48);  // blocks 0..3; each stage prefetches the block two stages ahead
  const int r = threadIdx.x, row = row0 + r;
  const int kr = row < n ? row : n - 1;
  const float* __restrict__ w = a.w;
  RowIO in{a.desc + (long long)kr * a.rs, (int)(a.cs * 4)};
  const float* ax = a.aux + (long long)kr * a.ars;
  const float g = __ldg(ax), gamma = __ldg(ax + a.afs);
  float fin[16];
#pragma unroll
  for (int j = 0; j < 16; ++j) fin[j] = 0.0f;
  const YS y{tile + r};
  // main trunk (radiancePredict.cu:396-421): blocks 0, 1 per row, 2..7 as GEMMs
  const float* __restrict__ sw = a.img + kSeOff;  // squeeze-excitation block weights
  row_block8<0>(in, w, sw, 0, WOFF(L01W), WOFF(L_Tr01W), WOFF(L_Hg01W), g, gamma, y, fin);
  row_block8<2>(in, w, sw + kSeFloats, 8, WOFF(L11W), WOFF(L_Tr11W), WOFF(L_Hg11W), g, gamma, y, fin);
#pragma unroll 1
  for (int st = 0; st < 6; ++st) {
    const int S = stage_width(st), from = st < 3 ? 16 + 16 * st : 64 + 32 * (st - 3);
    const float* sws = sw + (2 + st) * kSeFloats;
    if (st < 4) desc_prefetch(a, row0, n, st == 0 ? 48 : 32 * st + 32, st == 0 ? 64 : 32 * st + 64);
    if (S == 16)
      row_gate_input<16>(in, sws, from, g, gamma, y, fin);
    else
      row_gate_input<32>(in, sws, from, g, gamma, y, fin);
    asm volatile("cp.async.wait_group 1;\n" ::: "memory");
    __syncthreads();  // stage st's weights and every row's input are in the tile
    const float* W = ring + (st & 1) * stage_floats(kTrunkStages - 1);
    if (st < 2)
      trunk_gemm<16, 0>(tile, W, a.desc, a.rs, a.cs, row0, n, from, to);
    else if (st == 2)
      trunk_gemm<16, 1>(tile, W, a.desc, a.rs, a.cs, row0, n, from, to);
    else
      trunk_gemm<32, 0>(tile, W, a.desc, a.rs, a.cs, row0, n, from, to);
    trunk_stage_issue(a.img, ring, st + 2);  // ring buffer st % 2 is free: every thread passed the GEMM's barriers
    __syncthreads();                          // y complete for the per-row part
  }
  // L81 -> comb[0..96)
  asm volatile("cp.async.wait_group 1;\n" ::: "memory");
  __syncthreads();
  trunk_gemm<32, 2>(tile, ring + (6 & 1) * stage_floats(kTrunkStages - 1), a.desc, a.rs, a.cs, row0, n, 0, to);
  asm volatile("cp.async.wait_all;\n" ::: "memory");
  const bool valid = row < n;
  float* orow = to.t + (long long)row * to.rs;
  auto put4 = [&](int c, float x0, float x1, float x2, float x3) {
    if (valid) *reinterpret_cast<float4*>(orow + c * to.cs) = make_float4(x0, x1, x2, x3);
  };
  // the light-direction trunk (blocks 8..11, LD41) runs in k_light_trunk
  // LSEFin1's g and gamma columns (pool[72], pool[73]); the albedo column is
  // added per channel by the head
#pragma unroll
  for (int j = 0; j < 16; ++j)
    fin[j] += g * __ldg(w + WOFF(LSEFin1W) + j * 75 + 72) + gamma * __ldg(w + WOFF(LSEFin1W) + j * 75 + 73);
#pragma unroll
  for (int j0 = 0; j0 < 16; j0 += 4) put4(30 + j0 / 4, fin[j0], fin[j0 + 1], fin[j0 + 2], fin[j0 + 3]);
}

// One tile per block (a resident grid striding over the tiles measured
// slower: 0.948 against 0.930 ms for the network).
__global__ void __launch_bounds__(kTile, 3) k_simt_trunk(TrunkArgs a, TrunkOut to) {
  extern __shared__ __align__(16) float tsm[];
  const int n = a.count ? (int)min(*a.count, (unsigned)a.n) : a.n;
  const int row0 = blockIdx.x * kTile;
  if (row0 < n) trunk_tile(a, to, tsm, tsm + 96 * kTile, row0, n);  // block-uniform
}

// ---- light-direction trunk --------------------------------------------------------------
// Blocks 8..11 (SE + ADD3, then SERES + ADD3, width 8) and LD41
// (radiancePredict.cu:424-437) per row, after k_simt_trunk: comb[96..120)
// into trunk-output chunks 24..29 and the blocks' LSEFin1 terms added to the
// sums in chunks 30..33. One thread per row; the weights (squeeze-excitation
// of the four blocks, then the fifteen 8 -> 8 layers with their biases) are
// kernel parameters, uniform constant-bank operands.
struct LightParams {
  float se[4][kSeFloats];
  float dense[15][72];  // LD01, LD11, LD21, LD31, LD41; per block branches density, transmittance, phase
  float head[144];      // the head-row image's first 144 floats: LSEFin2, LSEFin1's albedo column, LGGS W, B
};
static_assert(sizeof(LightParams) + sizeof(TrunkArgs) + sizeof(TrunkOut) <= 32000, "kernel parameter space");

void light_param_image(const float* w, const std::vector<float>& img, std::vector<float>& out) {
  out.assign(sizeof(LightParams) / sizeof(float), 0.0f);
  std::copy(img.begin() + kSeOff + 8 * kSeFloats, img.begin() + kSeOff + 12 * kSeFloats, out.begin());
  const WeightTable wt = make_weight_table();
  const int ids[15] = {MR_W_LD01W, MR_W_LD_Tr01W, MR_W_LD_Hg01W, MR_W_LD11W, MR_W_LD_Tr11W, MR_W_LD_Hg11W,
                       MR_W_LD21W, MR_W_LD_Tr21W, MR_W_LD_Hg21W, MR_W_LD31W, MR_W_LD_Tr31W, MR_W_LD_Hg31W,
                       MR_W_LD41W, MR_W_LD_Tr41W, MR_W_LD_Hg41W};
  for (int d = 0; d < 15; ++d)
    std::copy(w + wt.off[ids[d]], w + wt.off[ids[d]] + 72, out.begin() + 4 * kSeFloats + 72 * d);
  std::copy(img.begin() + kHeadRowOff, img.begin() + kHeadRowOff + 144, out.begin() + 4 * kSeFloats + 15 * 72);
}

// 8 -> 8 layer, bias first then ascending inputs (dense1's order), weights
// from the parameter space.
__device__ __forceinline__ void dense8p(const float (&x)[8], float (&y)[8], const float* W) {
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    float acc = W[64 + q];
#pragma unroll
    for (int j = 0; j < 8; ++j) acc += x[j] * W[q * 8 + j];
    y[q] = relu0(acc);
  }
}

template <int B>
__device__ __forceinline__ void light_block(const RowIO& in, const LightParams& P, float g, float gamma,
                                            float (&y)[3][8], float (&fin)[16]) {
  constexpr int from = 160 + 8 * B;
  const float* sw = P.se[B];
  float st[6];
#pragma unroll
  for (int b = 0; b < 3; ++b) {
    float s = 0.0f, m = -10000.0f;
#pragma unroll
    for (int i = 0; i < 8; i += 4) {
      const float4 q = in.ld4(b * 192 + from + i);
      s += q.x; s += q.y; s += q.z; s += q.w;
      m = fmaxf(m, q.x); m = fmaxf(m, q.y); m = fmaxf(m, q.z); m = fmaxf(m, q.w);
    }
    st[2 * b] = s / 8.0f;
    st[2 * b + 1] = m;
  }
#pragma unroll
  for (int k = 0; k < 6; ++k)
#pragma unroll
    for (int j = 0; j < 16; ++j) fin[j] += st[k] * sw[k * 16 + j];
  const float tmp[8] = {st[0], st[2], st[4], st[1], st[3], st[5], g, gamma};
  float h[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    float a = 0.0f;
#pragma unroll
    for (int j = 0; j < 8; ++j) a += tmp[j] * sw[96 + i * 8 + j];
    h[i] = relu0(a);
  }
#pragma unroll
  for (int b = 0; b < 3; ++b) {
    float a = 0.0f;
#pragma unroll
    for (int j = 0; j < 8; ++j) a += h[j] * sw[160 + b * 8 + j];
    const float gate = 1.0f / (1.0f + expf(-a));
    float v[8], x[8], yn[8];  // the branch's block input (a second read, from L1)
#pragma unroll
    for (int i = 0; i < 8; i += 4) {
      const float4 q = in.ld4(b * 192 + from + i);
      v[i] = q.x; v[i + 1] = q.y; v[i + 2] = q.z; v[i + 3] = q.w;
    }
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const float xv = v[i] * gate;
      x[i] = B == 0 ? xv : xv + y[b][i];
    }
    dense8p(x, yn, P.dense[3 * B + b]);
#pragma unroll
    for (int i = 0; i < 8; ++i) y[b][i] = yn[i] + v[i];
  }
}

__device__ __forceinline__ void light_row(const TrunkArgs& a, const TrunkOut& to, const LightParams& P, int k) {
  const RowIO in{a.desc + (long long)k * a.rs, (int)(a.cs * 4)};
  const float* ax = a.aux + (long long)k * a.ars;
  const float g = __ldg(ax), gamma = __ldg(ax + a.afs);
  float y[3][8], fin[16];
#pragma unroll
  for (int j = 0; j < 16; ++j) fin[j] = 0.0f;
  light_block<0>(in, P, g, gamma, y, fin);
  light_block<1>(in, P, g, gamma, y, fin);
  light_block<2>(in, P, g, gamma, y, fin);
  light_block<3>(in, P, g, gamma, y, fin);
  float* orow = to.t + (long long)k * to.rs;
#pragma unroll
  for (int b = 0; b < 3; ++b) {  // LD41: comb[96..120)
    float c[8];
    dense8p(y[b], c, P.dense[12 + b]);
#pragma unroll
    for (int i = 0; i < 8; i += 4)
      *reinterpret_cast<float4*>(orow + ((96 + 8 * b + i) / 4) * to.cs) = make_float4(c[i], c[i + 1], c[i + 2], c[i + 3]);
  }
#pragma unroll
  for (int c = 0; c < 4; ++c) {  // LSEFin1 sums: the main trunk's (with the g, gamma columns) plus these blocks'
    float4* f = reinterpret_cast<float4*>(orow + (30 + c) * to.cs);
    const float4 q = *f;
    fin[4 * c] = q.x + fin[4 * c];
    fin[4 * c + 1] = q.y + fin[4 * c + 1];
    fin[4 * c + 2] = q.z + fin[4 * c + 2];
    fin[4 * c + 3] = q.w + fin[4 * c + 3];
    *f = make_float4(fin[4 * c], fin[4 * c + 1], fin[4 * c + 2], fin[4 * c + 3]);
  }
  // the head's gates of albedo channel 0 (radiancePredict.cu:439-452), in
  // k_tc32_head's arithmetic: sep[0..6) in chunks 34..35, LGGS x8 in 36..37
  const float* H = P.head;
  const float sc = __ldg(ax + 2 * a.afs);
  float sew[16], sep[6], x8[8];
#pragma unroll
  for (int j = 0; j < 16; ++j) sew[j] = relu0(fin[j] + sc * H[96 + j]);
#pragma unroll
  for (int i = 0; i < 6; ++i) {
    float acc = 0.0f;
#pragma unroll
    for (int j = 0; j < 16; ++j) acc += sew[j] * H[i * 16 + j];
    sep[i] = 1.0f / (1.0f + expf(-acc));
  }
#pragma unroll
  for (int i = 0; i < 8; ++i) {  // LGGS 3 -> 8, bias after the sum
    float acc = g * H[112 + 3 * i] + gamma * H[112 + 3 * i + 1] + sc * H[112 + 3 * i + 2];
    acc += H[136 + i];
    x8[i] = relu0(acc);
  }
  *reinterpret_cast<float4*>(orow + 34 * to.cs) = make_float4(sep[0], sep[1], sep[2], sep[3]);
  *reinterpret_cast<float4*>(orow + 35 * to.cs) = make_float4(sep[4], sep[5], 0.0f, 0.0f);
  *reinterpret_cast<float4*>(orow + 36 * to.cs) = make_float4(x8[0], x8[1], x8[2], x8[3]);
  *reinterpret_cast<float4*>(orow + 37 * to.cs) = make_float4(x8[4], x8[5], x8[6], x8[7]);
}

// One row per thread, no loop (see k_tc32_tail).
__global__ void __launch_bounds__(128, 6) k_light_trunk(TrunkArgs a, TrunkOut to, const LightParams P) {
  const int n = a.count ? (int)min(*a.count, (unsigned)a.n) : a.n;
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) light_row(a, to, P, k);
}

// ---- head --------------------------------------------------------------------------

constexpr int kHeadRows = kTile;   // rows (pixels) per tile
constexpr int kHeadThreads = 256;  // two threads per row
struct HeadArgs {
  const float* __restrict__ w;
  const float* __restrict__ wt;  // simt_weight_image
  const float* __restrict__ t;   // trunk outputs (TrunkOut layout)
  long long trs, tcs;
  const float* __restrict__ aux;
  long long ars, afs;
  int n;
  const unsigned* __restrict__ count;
  float* out;
  const int* __restrict__ pix;
  const float* __restrict__ trph;
  F3 light_color, scatter;
  const int* job;
  const BatchOut* bout;
  int* err;  // tensor-core head: set when a bounded wait gave up
  float* stg;  // LC2 outputs per albedo channel: chunk 8 ch + c of row k at stg[k*srs + c*scs]
  long long srs, scs;
};

// ---- head on the tensor cores (fp32-accurate) ---------------------------------------
// LC0 / LC1 / LC2 as M = 128 tcgen05 MMAs of kind::tf32 with FP32 accumulators
// in TMEM: every product is the sum of three TF32 products (A_hi W_hi + A_hi
// W_lo + A_lo W_hi, split_tf32), which carries about 22 bits of each operand,
// the accuracy of an fp32 dot product. Activations live in two canonical
// K-major tiles (TF32 part and fp32 remainder, 128 rows x K <= 128).
// Persistent blocks (one per SM) walk the row tiles. Thread 0 streams the
// split weight chunks (32 input columns each, the same 10-chunk sequence for
// every albedo channel) into a 3-slot shared-memory ring with bulk copies two
// chunks ahead of the MMAs that consume them (per-slot full / empty
// mbarriers), and issues the MMAs; the other threads only wait for a layer's
// MMAs before its epilogue, which runs per row on the TMEM lanes (bias, ReLU,
// split into the next layer's tiles). Gates, LX and the residual pairs stay
// per row on the CUDA cores.
constexpr int kTcSlots = 3;
constexpr int kTcStage = 2 * kTcKC * 128;  // floats per ring slot (largest chunk: 32 KB)
constexpr int kTcATile = 128 * 128;        // floats per A tile
constexpr int kTcHeadSmem = (2 * kTcATile + kTcSlots * kTcStage) * (int)sizeof(float) + 64;

struct TcFeed {  // thread 0's view of the weight ring
  const float* __restrict__ src;  // chunk images
  uint32_t ring, full, empty;     // shared addresses: slot 0, full[0], empty[0] (slots 8 B apart)
  int x;                          // next chunk to consume (running over channels and tiles)
  bool ok;
  __device__ __forceinline__ void load(int z) {  // chunk z into slot z % 3
    const int c = z % kTcChunks, s = z % kTcSlots;
    const uint32_t bytes = (uint32_t)tc_chunk_floats(c) * 4u;
    mbar_expect_tx(full + 8 * s, bytes);
    bulk_g2s(ring + (uint32_t)(s * kTcStage * 4), src + tc_chunk_off(c), bytes, full + 8 * s);
  }
};

// Thread 0: the MMAs of one head layer D[tmem] = A (128 x K) W^T (K -> N),
// K / 32 chunks of three TF32 products (4 MMAs of K = 8 each), refilling
// each consumed slot with the chunk three places later; then a commit on
// `done` that completes when every MMA of the layer has.
template <int N, int K>
__device__ __forceinline__ void tc_issue_layer(TcFeed& f, uint32_t tmem, uint32_t ahi, uint32_t alo, uint32_t done) {
  constexpr uint32_t id = idesc_tf32(128, N), sbo_a = (K / 4) * 128, sbo_b = (kTcKC / 4) * 128;
#pragma unroll 1
  for (int j = 0; j < K / kTcKC; ++j) {
    const int x = f.x, s = x % kTcSlots;
    if (f.ok && !mbar_wait(f.full + 8 * s, (uint32_t)(x / kTcSlots) & 1u)) f.ok = false;
    tc_fence_after();
    if (f.ok) {
      const uint32_t bh = f.ring + (uint32_t)(s * kTcStage * 4), bl = bh + N * kTcKC * 4;
#pragma unroll
      for (int term = 0; term < 3; ++term) {  // remainder terms first, then TF32 x TF32
        const uint32_t a = (term == 1 ? alo : ahi) + j * (kTcKC / 4) * 128, b = term == 0 ? bl : bh;
#pragma unroll
        for (int k8 = 0; k8 < kTcKC / 8; ++k8)
          umma_tf32(tmem, sdesc(a + k8 * 256, 128, sbo_a), sdesc(b + k8 * 256, 128, sbo_b), id,
                    (j | term | k8) ? 1u : 0u);
      }
    }
    umma_commit(f.empty + 8 * s);
    if (x >= 1) {  // chunk x - 1's MMAs are done with their slot: chunk x + 2 goes there
      const int y = x - 1, ys = y % kTcSlots;
      if (f.ok && !mbar_wait(f.empty + 8 * ys, (uint32_t)(y / kTcSlots) & 1u)) f.ok = false;
      if (f.ok) f.load(x + 2);
    }
    ++f.x;
  }
  umma_commit(done);
}

// All threads: the layer's MMAs are complete (bounded wait).
__device__ __forceinline__ void tc_layer_wait(uint32_t done, uint32_t& parity, bool& ok) {
  if (ok && !mbar_wait(done, parity)) ok = false;
  parity ^= 1u;
  tc_fence_after();
}

// 4 activations of row r at columns k..k+3 into the K-major split tiles.
__device__ __forceinline__ void put_split4(float* ahi, float* alo, int r, int k, int kp, float x0, float x1, float x2,
                                           float x3) {
  float4 h, l;
  split_tf32(x0, h.x, l.x);
  split_tf32(x1, h.y, l.y);
  split_tf32(x2, h.z, l.z);
  split_tf32(x3, h.w, l.w);
  const int o = canon32(r, k, kp) / 4;
  *reinterpret_cast<float4*>(ahi + o) = h;
  *reinterpret_cast<float4*>(alo + o) = l;
}

// Epilogue of a layer with N outputs: this thread's N/2 columns (half `h`) of
// its TMEM lane, ReLU(acc + bias), into the next layer's tiles (K = N).
template <int N>
__device__ __forceinline__ void tc_epi_split(uint32_t tl, const float* __restrict__ bias, float* ahi, float* alo, int r,
                                             int h) {
  static_assert(N % 64 == 0, "pairs of 16-column loads per thread");
#pragma unroll
  for (int q = 0; q < N / 32; q += 2) {  // two TMEM loads under one wait
    float v[2][16];
    tmem_ld16x2(tl + h * (N / 2) + 16 * q, tl + h * (N / 2) + 16 * (q + 1), v[0], v[1]);
#pragma unroll
    for (int p = 0; p < 2; ++p) {
      const int c0 = h * (N / 2) + 16 * (q + p);
#pragma unroll
      for (int i = 0; i < 16; i += 4) {
        const float4 b = ldg4(bias + c0 + i);
        put_split4(ahi, alo, r, c0 + i, N, relu0(v[p][i] + b.x), relu0(v[p][i + 1] + b.y), relu0(v[p][i + 2] + b.z),
                   relu0(v[p][i + 3] + b.w));
      }
    }
  }
}

// L2 prefetch of tile `tile`'s trunk outputs (rows below n): one range per
// 4-float chunk when rows are 16 bytes apart (render path), else one range of
// whole rows when the chunks of a row are contiguous.
__device__ __forceinline__ void prefetch_tile(const HeadArgs& a, int tile, int n) {
  const long long r0 = (long long)tile * kHeadRows;
  if (r0 >= n) return;
  const int rows = (int)min((long long)kHeadRows, n - r0);
  if (a.trs == 4) {
    for (int c = 0; c < 38; ++c)
      asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(a.t + r0 * 4 + c * a.tcs), "r"(rows * 16)
                   : "memory");
  } else if (a.tcs == 4 && a.trs % 4 == 0) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(a.t + r0 * a.trs),
                 "r"((unsigned)(rows * a.trs * 4))
                 : "memory");
  }
}

// Head SC(p) (radiancePredict.cu:439-473) per distinct albedo channel for
// tiles of 128 rows, LC0 / LC1 / LC2 on the tensor cores. Thread t serves
// row r = 32 (warp % 4) + lane (its TMEM lane) and column half warp / 4.
__global__ void __launch_bounds__(kHeadThreads, 1) k_tc32_head(HeadArgs a) {
  extern __shared__ __align__(1024) float tcsm[];
  float* Ahi = tcsm;
  float* Alo = tcsm + kTcATile;
  float* ring = tcsm + 2 * kTcATile;
  uint64_t* mb = reinterpret_cast<uint64_t*>(ring + kTcSlots * kTcStage);  // full[3], empty[3], done
  uint32_t* holder = reinterpret_cast<uint32_t*>(mb + 2 * kTcSlots + 1);
  const int n = a.count ? (int)min(*a.count, (unsigned)a.n) : a.n;
  const int ntiles = (n + kHeadRows - 1) / kHeadRows;
  if ((int)blockIdx.x >= ntiles) return;  // block-uniform
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int r = 32 * (warp & 3) + lane, half = warp >> 2;  // TMEM lane mapping
  const float* __restrict__ hr = a.wt + kHeadRowOff;
  const float* __restrict__ bias = a.wt + kTcBiasOff;
  const uint32_t done = smem_u32(mb + 2 * kTcSlots);
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(holder)),
                 "r"(128));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (threadIdx.x == 0) {
    for (int i = 0; i < 2 * kTcSlots + 1; ++i) mbar_init(smem_u32(mb + i), 1);
  }
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *holder;
  const uint32_t tl = tmem + ((uint32_t)(32 * (warp & 3)) << 16);
  const uint32_t ahi = smem_u32(Ahi), alo = smem_u32(Alo);
  TcFeed feed{a.wt + kTcHeadOff, smem_u32(ring), smem_u32(mb), smem_u32(mb + kTcSlots), 0, true};
  if (threadIdx.x == 0)
    for (int z = 0; z < kTcSlots; ++z) feed.load(z);
  uint32_t dpar = 0;
  bool ok = true;
#pragma unroll 1
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int row = tile * kHeadRows + r;
    const bool valid = row < n;
    const int kr = valid ? row : n - 1;
    const float* trow = a.t + (long long)kr * a.trs;
    const float* ax = a.aux + (long long)kr * a.ars;
    const float g = __ldg(ax), gamma = __ldg(ax + a.afs);
    const float srp[3] = {__ldg(ax + 2 * a.afs), __ldg(ax + 3 * a.afs), __ldg(ax + 4 * a.afs)};
    float fin[16];
    float4 tin[16];  // this thread's trunk-output chunks 16 half .. 16 half + 15 (those below 30)
#pragma unroll
    for (int i = 0; i < 16; ++i)
      if (16 * half + i < 30) tin[i] = __ldg(reinterpret_cast<const float4*>(trow + (16 * half + i) * a.tcs));
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const float4 q = __ldg(reinterpret_cast<const float4*>(trow + (30 + c) * a.tcs));
      fin[4 * c] = q.x; fin[4 * c + 1] = q.y; fin[4 * c + 2] = q.z; fin[4 * c + 3] = q.w;
    }
    // channel 0's gates, computed by k_light_trunk: sep in chunks 34..35, LGGS in 36..37
    const float4 gs0 = __ldg(reinterpret_cast<const float4*>(trow + 34 * a.tcs));
    const float4 gs1 = __ldg(reinterpret_cast<const float4*>(trow + 35 * a.tcs));
    float4 gx[2] = {make_float4(0.0f, 0.0f, 0.0f, 0.0f), make_float4(0.0f, 0.0f, 0.0f, 0.0f)};
    if (half) {  // LC0 input columns 120..127 belong to half 1
      gx[0] = __ldg(reinterpret_cast<const float4*>(trow + 36 * a.tcs));
      gx[1] = __ldg(reinterpret_cast<const float4*>(trow + 37 * a.tcs));
    }
    if (threadIdx.x == 0) prefetch_tile(a, tile + gridDim.x, n);  // the next tile's trunk outputs -> L2
    tc_fence_before();  // the previous tile's TMEM reads
    const bool need1 = __syncthreads_or(valid && srp[1] != srp[0]);
    const bool need2 = __syncthreads_or(valid && srp[2] != srp[0] && srp[2] != srp[1]);
#pragma unroll 1
    for (int ch = 0; ch < 3; ++ch) {
      if ((ch == 1 && !need1) || (ch == 2 && !need2)) continue;
      const float sc = ch == 0 ? srp[0] : ch == 1 ? srp[1] : srp[2];
      // gates of this channel (LGGS, LSEFin1's albedo column, LSEFin2)
      float sep[6] = {gs0.x, gs0.y, gs0.z, gs0.w, gs1.x, gs1.y};
      if (ch > 0) {
        float sew[16];
#pragma unroll
        for (int j = 0; j < 16; j += 4) {
          const float4 f = ldg4(hr + 96 + j);
          sew[j] = relu0(fin[j] + sc * f.x);
          sew[j + 1] = relu0(fin[j + 1] + sc * f.y);
          sew[j + 2] = relu0(fin[j + 2] + sc * f.z);
          sew[j + 3] = relu0(fin[j + 3] + sc * f.w);
        }
#pragma unroll
        for (int i = 0; i < 6; ++i) {
          float acc = 0.0f;
#pragma unroll
          for (int j = 0; j < 16; j += 4) {
            const float4 f = ldg4(hr + i * 16 + j);
            acc += sew[j] * f.x;
            acc += sew[j + 1] * f.y;
            acc += sew[j + 2] * f.z;
            acc += sew[j + 3] * f.w;
          }
          sep[i] = 1.0f / (1.0f + expf(-acc));
        }
      }
      // gated head input into the LC0 tiles: columns 64 half .. 64 half + 63
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        const int c = 16 * half + i;
        if (c < 30) {
          const float4 q = tin[i];
          const float s = c < 24 ? sep[c >> 3] : sep[3 + ((c - 24) >> 1)];
          put_split4(Ahi, Alo, r, 4 * c, 128, q.x * s, q.y * s, q.z * s, q.w * s);
        } else if (ch == 0) {
          const float4 q = gx[c - 30];
          put_split4(Ahi, Alo, r, 4 * c, 128, q.x, q.y, q.z, q.w);
        } else {
          float x[4];
#pragma unroll
          for (int u = 0; u < 4; ++u) {  // LGGS 3 -> 8, bias after the sum
            const int i = 4 * (c - 30) + u;
            float acc =
                g * __ldg(hr + 112 + 3 * i) + gamma * __ldg(hr + 112 + 3 * i + 1) + sc * __ldg(hr + 112 + 3 * i + 2);
            acc += __ldg(hr + 136 + i);
            x[u] = relu0(acc);
          }
          put_split4(Ahi, Alo, r, 4 * c, 128, x[0], x[1], x[2], x[3]);
        }
      }
      // LC0
      fence_async_smem();
      tc_fence_before();
      __syncthreads();
      if (threadIdx.x == 0) tc_issue_layer<128, 128>(feed, tmem, ahi, alo, done);
      tc_layer_wait(done, dpar, ok);
      tc_epi_split<128>(tl, bias, Ahi, Alo, r, half);
      // LC1
      fence_async_smem();
      tc_fence_before();
      __syncthreads();
      if (threadIdx.x == 0) tc_issue_layer<64, 128>(feed, tmem, ahi, alo, done);
      tc_layer_wait(done, dpar, ok);
      tc_epi_split<64>(tl, bias + 128, Ahi, Alo, r, half);
      // LC2
      fence_async_smem();
      tc_fence_before();
      __syncthreads();
      if (threadIdx.x == 0) tc_issue_layer<32, 64>(feed, tmem, ahi, alo, done);
      tc_layer_wait(done, dpar, ok);
      // LC2 outputs (bias, ReLU) of this channel to the staging columns; the
      // tail runs in k_tc32_tail
      {
        float v[16];
        tmem_ld16(tl + 16 * half, v);
        if (valid) {
          float* srow = a.stg + (long long)row * a.srs;
#pragma unroll
          for (int i = 0; i < 16; i += 4) {
            const float4 b = ldg4(bias + 192 + 16 * half + i);
            *reinterpret_cast<float4*>(srow + (8 * ch + (16 * half + i) / 4) * a.scs) =
                make_float4(relu0(v[i] + b.x), relu0(v[i + 1] + b.y), relu0(v[i + 2] + b.z), relu0(v[i + 3] + b.w));
          }
        }
      }
    }
  }
  // the two chunks loaded ahead of the last consumed one land before exit
  if (threadIdx.x == 0) {
    for (int z = feed.x; z < feed.x + 2; ++z)
      if (feed.ok && !mbar_wait(feed.full + 8 * (z % kTcSlots), (uint32_t)(z / kTcSlots) & 1u)) feed.ok = false;
    if (!feed.ok) ok = false;
  }
  if (!ok && a.err) atomicExch(a.err, 1);
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(128));
  }
}

// ---- tail of the head ----------------------------------------------------------------
// LX 32 -> 16, the six residual pairs of 16 -> 16 layers and LX12 16 -> 1
// (radiancePredict.cu:454-471) for each row and albedo channel, then the
// output (:472-483). One thread per row; the 3809 weights (LXW .. LX12B, in
// blob order) are kernel parameters, so each is a uniform constant-bank
// operand of its multiply-add and the layers issue no loads.
constexpr int kTailFloats = 512 + 16 + 12 * 272 + 16 + 1;
struct TailParams {
  float w[kTailFloats];
};
struct TailArgs {
  const float* __restrict__ stg;  // LC2 outputs (HeadArgs::stg layout)
  long long srs, scs;
  const float* __restrict__ aux;
  long long ars, afs;
  int n;
  const unsigned* __restrict__ count;
  float* out;
  const int* __restrict__ pix;
  const float* __restrict__ trph;
  F3 light_color, scatter;
  const int* job;
  const BatchOut* bout;
};

// Host image of TailParams: the blob's LXW .. LX12B, which are contiguous.
void tail_param_image(const float* w, std::vector<float>& out) {
  const WeightTable wt = make_weight_table();
  out.assign(w + wt.off[MR_W_LXW], w + wt.off[MR_W_LXW] + kTailFloats);
}
static_assert(sizeof(TailParams) + sizeof(TailArgs) <= 32000, "kernel parameter space");

// One row and channel: x = the channel's 32 LC2 outputs (chunks 8 ch .. 8 ch + 7).
__device__ __forceinline__ float tail_row(const float* srow, long long scs, int ch, const TailParams& P) {
  float x[32];
#pragma unroll
  for (int c = 0; c < 8; ++c) {
    const float4 q = __ldg(reinterpret_cast<const float4*>(srow + (8 * ch + c) * scs));
    x[4 * c] = q.x; x[4 * c + 1] = q.y; x[4 * c + 2] = q.z; x[4 * c + 3] = q.w;
  }
  float a16[16];
#pragma unroll
  for (int q = 0; q < 16; ++q) {  // LX, bias first, ascending inputs
    float acc = P.w[512 + q];
#pragma unroll
    for (int j = 0; j < 32; ++j) acc += x[j] * P.w[q * 32 + j];
    a16[q] = relu0(acc);
  }
#pragma unroll
  for (int rr = 0; rr < 6; ++rr) {
    const float* W1 = P.w + 528 + 272 * (2 * rr);
    const float* W2 = W1 + 272;
    float h16[16];
#pragma unroll
    for (int q = 0; q < 16; ++q) {
      float acc = W1[256 + q];
#pragma unroll
      for (int j = 0; j < 16; ++j) acc += a16[j] * W1[q * 16 + j];
      h16[q] = relu0(acc);
    }
#pragma unroll
    for (int q = 0; q < 16; ++q) {  // a16 is dead once h16 exists: the residual sum goes in place
      float acc = W2[256 + q];
#pragma unroll
      for (int j = 0; j < 16; ++j) acc += h16[j] * W2[q * 16 + j];
      a16[q] = a16[q] + relu0(acc);
    }
  }
  float o = 0.0f;  // LX12 16 -> 1, bias after the sum
#pragma unroll
  for (int i = 0; i < 16; ++i) o += a16[i] * P.w[3792 + i];
  o += P.w[3808];
  return relu0(o);
}

// Straight-line code per channel (a loop over the channels would let the
// compiler hoist the constant operands out of it into registers).
__device__ __forceinline__ void tail_one(const TailArgs& a, const TailParams& P, int k) {
  const float* ax = a.aux + (long long)k * a.ars;
  const float srp[3] = {__ldg(ax + 2 * a.afs), __ldg(ax + 3 * a.afs), __ldg(ax + 4 * a.afs)};
  const float* srow = a.stg + (long long)k * a.srs;
  float X[3];
  X[0] = tail_row(srow, a.scs, 0, P);
  X[1] = srp[1] != srp[0] ? tail_row(srow, a.scs, 1, P) : X[0];
  X[2] = srp[2] == srp[0] ? X[0] : srp[2] == srp[1] ? X[1] : tail_row(srow, a.scs, 2, P);
  const float o[3] = {fmaxf(expf(X[0]) - 1.0f, 0.0f) * srp[0], fmaxf(expf(X[1]) - 1.0f, 0.0f) * srp[1],
                      fmaxf(expf(X[2]) - 1.0f, 0.0f) * srp[2]};
  if (a.pix) {
    const int px = a.pix[k];
    const float tr = a.trph[k];
    F3 lc = a.light_color, scv = a.scatter;
    float* dst = a.out;
    if (a.job) {
      const BatchOut& bo = a.bout[a.job[k]];
      lc = bo.light_color;
      scv = bo.scatter;
      dst = bo.out;
    }
    dst[3 * (size_t)px + 0] = fmaxf(((o[0] + tr) * lc.x) * scv.x, 0.0f);
    dst[3 * (size_t)px + 1] = fmaxf(((o[1] + tr) * lc.y) * scv.y, 0.0f);
    dst[3 * (size_t)px + 2] = fmaxf(((o[2] + tr) * lc.z) * scv.z, 0.0f);
  } else {
#pragma unroll
    for (int c = 0; c < 3; ++c) a.out[3 * (size_t)k + c] = o[c];
  }
}

// One row per thread, no loop: around a loop the compiler would hoist the
// constant operands into registers.
__global__ void __launch_bounds__(128, 6) k_tc32_tail(TailArgs a, const TailParams P) {
  const int n = a.count ? (int)min(*a.count, (unsigned)a.n) : a.n;
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) tail_one(a, P, k);
}

int* mlp_error_word(const Network* net);  // mr_mlp_tc.cu

// Trunk kernel then head kernel. `tout` receives the trunk outputs (TrunkOut
// layout with strides trs / tcs): the render path passes its own descriptor
// columns, whose first 38 chunks of a row are no longer needed once that row's
// trunks are done.
int launch_mlp_simt(const Network* net, const float* desc, const float* aux, long long rs, long long cs,
                    long long ars, long long afs, int n, const unsigned* count, float* out, const int* pix,
                    const float* trph, F3 light_color, F3 scatter, cudaStream_t s, const int* job,
                    const BatchOut* bout, float* tout, long long trs, long long tcs, float* stg, long long srs,
                    long long scs, StageTimer* timer) {
  if (!tout || !stg) return set_error(MR_ERR_ARG, "fp32 network: no buffer for the trunk or LC2 outputs");
  if (net->h_tail.size() != (size_t)kTailFloats || net->h_light.size() * sizeof(float) != sizeof(LightParams))
    return set_error(MR_ERR_STATE, "network not packed");
  static DeviceCache attr;  // the attributes belong to each device's context
  int rc = attr.once([] {
    MR_CUDA(cudaFuncSetAttribute(k_tc32_head, cudaFuncAttributeMaxDynamicSharedMemorySize, kTcHeadSmem));
    MR_CUDA(cudaFuncSetAttribute(k_simt_trunk, cudaFuncAttributeMaxDynamicSharedMemorySize, kTrunkSmem));
    return (int)MR_OK;
  });
  if (rc) return rc;
  TrunkArgs a;
  a.w = net->w;
  a.img = net->simt_img;
  a.desc = desc;
  a.aux = aux;
  a.rs = rs;
  a.cs = cs;
  a.ars = ars;
  a.afs = afs;
  a.n = n;
  a.count = count;
  if (timer) timer->mark(ST_NN_TRUNK, s);
  k_simt_trunk<<<(unsigned)((n + kTile - 1) / kTile), kTile, kTrunkSmem, s>>>(a, TrunkOut{tout, trs, tcs});
  if (timer) timer->mark(ST_NN_TRUNK, s);
  MR_CUDA(cudaGetLastError());
  {
    LightParams LP;
    std::memcpy(&LP, net->h_light.data(), sizeof(LP));
    k_light_trunk<<<(unsigned)((n + 127) / 128), 128, 0, s>>>(a, TrunkOut{tout, trs, tcs}, LP);
    MR_CUDA(cudaGetLastError());
  }
  HeadArgs h;
  h.w = net->w;
  h.wt = net->simt_img;
  h.t = tout;
  h.trs = trs;
  h.tcs = tcs;
  h.aux = aux;
  h.ars = ars;
  h.afs = afs;
  h.n = n;
  h.count = count;
  h.out = out;
  h.pix = pix;
  h.trph = trph;
  h.light_color = light_color;
  h.scatter = scatter;
  h.job = job;
  h.bout = bout;
  h.err = mlp_error_word(net);
  h.stg = stg;
  h.srs = srs;
  h.scs = scs;
  const int tiles = (n + kHeadRows - 1) / kHeadRows;
  k_tc32_head<<<(unsigned)std::min(tiles, sm_count()), kHeadThreads, kTcHeadSmem, s>>>(h);
  MR_CUDA(cudaGetLastError());
  TailArgs t;
  t.stg = stg;
  t.srs = srs;
  t.scs = scs;
  t.aux = aux;
  t.ars = ars;
  t.afs = afs;
  t.n = n;
  t.count = count;
  t.out = out;
  t.pix = pix;
  t.trph = trph;
  t.light_color = light_color;
  t.scatter = scatter;
  t.job = job;
  t.bout = bout;
  TailParams P;
  std::memcpy(P.w, net->h_tail.data(), sizeof(P.w));
  k_tc32_tail<<<(unsigned)((n + 127) / 128), 128, 0, s>>>(t, P);
  MR_CUDA(cudaGetLastError());
  return MR_OK;
}

}  // namespace mr
