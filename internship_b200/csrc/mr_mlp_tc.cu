// Radiance-predictor network on the 5th-generation tensor cores (tcgen05).
//
// The network of core/radiancePredict.cu:370-485 is evaluated for tiles of
// 128 pixels: every linear layer wider than 3 inputs is one M=128 x N x K
// tcgen05.mma (BF16 operands from shared memory, FP32 accumulators in tensor
// memory); the per-pixel work between layers (bias, ReLU, squeeze-excitation
// gates, residual adds, pooling) runs in FP32 with one thread per pixel row,
// which is exactly the row a warp reads back from its TMEM lane quarter.
//
// Layout: persistent kernel, one CTA per SM, kGroups tile groups of 4 warps.
// The packed BF16 weight image (canonical K-major, no swizzle: 8x16-byte core
// matrices, row groups SBO apart, K halves LBO = 128 B apart) is loaded into
// shared memory once per CTA and shared by the groups. Each group owns a
// 32 KB A region (three 128 x 32 branch tiles in the trunks, one 128 x 128
// tile in the head), 128 TMEM columns and an mbarrier signalled by
// tcgen05.commit.
// Only the elected thread 0 of a group issues MMAs. Every wait is bounded.
#include <cuda_bf16.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "mr_internal.h"
#include "mr_net_layout.cuh"
#include "mr_tcgen05.cuh"

namespace mr {

// ---- layer table -----------------------------------------------------------------
struct TcLayer { int w, b, n, k; };  // weight / bias ids (MR_W_*), true out / in sizes

#define L3(a, b, c, n) {MR_W_##a##W, MR_W_##a##B, n, n}, {MR_W_##b##W, MR_W_##b##B, n, n}, {MR_W_##c##W, MR_W_##c##B, n, n}
constexpr TcLayer kTc[] = {
    L3(L01, L_Tr01, L_Hg01, 8),  L3(L11, L_Tr11, L_Hg11, 8),  L3(L21, L_Tr21, L_Hg21, 16),
    L3(L31, L_Tr31, L_Hg31, 16), L3(L41, L_Tr41, L_Hg41, 16), L3(L51, L_Tr51, L_Hg51, 32),
    L3(L61, L_Tr61, L_Hg61, 32), L3(L71, L_Tr71, L_Hg71, 32), L3(L81, L_Tr81, L_Hg81, 32),
    L3(LD01, LD_Tr01, LD_Hg01, 8), L3(LD11, LD_Tr11, LD_Hg11, 8), L3(LD21, LD_Tr21, LD_Hg21, 8),
    L3(LD31, LD_Tr31, LD_Hg31, 8), L3(LD41, LD_Tr41, LD_Hg41, 8),
    {MR_W_LC0W, MR_W_LC0B, 128, 128}, {MR_W_LC1W, MR_W_LC1B, 64, 128}, {MR_W_LC2W, MR_W_LC2B, 32, 64},
    {MR_W_LXW, MR_W_LXB, 16, 32},
    {MR_W_LX0W, MR_W_LX0B, 16, 16}, {MR_W_LX1W, MR_W_LX1B, 16, 16}, {MR_W_LX2W, MR_W_LX2B, 16, 16},
    {MR_W_LX3W, MR_W_LX3B, 16, 16}, {MR_W_LX4W, MR_W_LX4B, 16, 16}, {MR_W_LX5W, MR_W_LX5B, 16, 16},
    {MR_W_LX6W, MR_W_LX6B, 16, 16}, {MR_W_LX7W, MR_W_LX7B, 16, 16}, {MR_W_LX8W, MR_W_LX8B, 16, 16},
    {MR_W_LX9W, MR_W_LX9B, 16, 16}, {MR_W_LX10W, MR_W_LX10B, 16, 16}, {MR_W_LX11W, MR_W_LX11B, 16, 16},
};
#undef L3
constexpr int kTcLayers = sizeof(kTc) / sizeof(kTc[0]);
static_assert(kTcLayers == 58, "layer count");
enum { TC_MAIN = 0, TC_L81 = 24, TC_DI = 27, TC_LD41 = 39, TC_LC0 = 42, TC_LC1 = 43, TC_LC2 = 44, TC_LX = 45,
       TC_LXR = 46 };

constexpr int pad16(int x) { return x < 16 ? 16 : (x + 15) / 16 * 16; }
constexpr int tc_bytes(int i) { return pad16(kTc[i].n) * pad16(kTc[i].k) * 2; }
constexpr int tc_offset(int i) { int o = 0; for (int j = 0; j < i; ++j) o += tc_bytes(j); return o; }
constexpr int kWBytes = tc_offset(kTcLayers);
static_assert(kWBytes == 100352, "packed weight image size");

// fp32 arrays read by the per-row code of the head (SEFin, LGGS, LX12) and
// the biases of the MMA layers, compacted into an image that is
// passed in the kernel's parameter space: uniform constant-bank operands
// instead of one load instruction per weight and row.
constexpr bool rowwise_used(int id) {
  for (int i = 0; i < kTcLayers; ++i)
    if (kTc[i].b == id) return true;
  constexpr int ids[] = {MR_W_LSEFin1W, MR_W_LSEFin2W, MR_W_LGGSW, MR_W_LGGSB, MR_W_LX12W, MR_W_LX12B};
  for (int x : ids)
    if (x == id) return true;
  return false;
}
struct RowTable { int off[MR_W_COUNT]; int total; };
constexpr RowTable make_row_table() {
  RowTable t{};
  const WeightTable wt = make_weight_table();
  int o = 0;
  for (int i = 0; i < MR_W_COUNT; ++i) {
    t.off[i] = rowwise_used(i) ? o : -1;
    if (rowwise_used(i)) o += (wt.size[i] + 3) / 4 * 4;  // every array 16-byte aligned: float4 reads
  }
  t.total = o;
  return t;
}
constexpr int kRowFloats = make_row_table().total;
template <int ID>
struct ROff {
  static constexpr int value = make_row_table().off[ID];
  static_assert(value >= 0, "weight array not in the row-wise image");
};
#define ROFF(name) (::mr::ROff<MR_W_##name>::value)

// Squeeze-excitation record of each trunk block (its gates and LSEFin1 terms,
// radiancePredict.cu:240-294), 192 floats read as float4 kernel parameters:
// [16 x (LSEFin1 weights of the block's 3 means, then its 3 maxima)],
// [SE1 8 x 8], [SE2 3 x 8], zero padding. Order of the records: the light
// trunk's blocks 0..3, then the main trunk's blocks 0..7.
constexpr int kSeRecFloats = 192, kSeRecs = 12;
struct SeRecSrc { int pid, se1, se2; };
constexpr SeRecSrc kSeRecSrc[kSeRecs] = {
    {24, MR_W_LDSE01W, MR_W_LDSE02W}, {27, MR_W_LDSE11W, MR_W_LDSE12W}, {30, MR_W_LDSE21W, MR_W_LDSE22W},
    {33, MR_W_LDSE31W, MR_W_LDSE32W}, {0, MR_W_LSE01W, MR_W_LSE02W},    {3, MR_W_LSE11W, MR_W_LSE12W},
    {6, MR_W_LSE21W, MR_W_LSE22W},    {9, MR_W_LSE31W, MR_W_LSE32W},    {12, MR_W_LSE41W, MR_W_LSE42W},
    {15, MR_W_LSE51W, MR_W_LSE52W},   {18, MR_W_LSE61W, MR_W_LSE62W},   {21, MR_W_LSE71W, MR_W_LSE72W},
};

// E4M3 image: rows of K padded to a multiple of 32 one-byte elements (the
// K of one f8f6f4 MMA), N padded to 16.
constexpr int kp8(int k) { return k <= 32 ? 32 : (k + 31) / 32 * 32; }
constexpr int tc_bytes8(int i) { return pad16(kTc[i].n) * kp8(kTc[i].k); }
constexpr int tc_offset8(int i) { int o = 0; for (int j = 0; j < i; ++j) o += tc_bytes8(j); return o; }
constexpr int kW8Bytes = tc_offset8(kTcLayers);

struct TcTables { int woff[kTcLayers]; int woff8[kTcLayers]; int boff[kTcLayers]; };
constexpr TcTables make_tc_tables() {
  TcTables t{};
  const RowTable rt = make_row_table();
  for (int i = 0; i < kTcLayers; ++i) {
    t.woff[i] = tc_offset(i);
    t.woff8[i] = tc_offset8(i);
    t.boff[i] = rt.off[kTc[i].b];
  }
  return t;
}
__constant__ TcTables c_tc = make_tc_tables();
__device__ __forceinline__ int tc_offset_dev(int i) { return c_tc.woff[i]; }
template <bool F8>
__device__ __forceinline__ int tc_off(int i) { return F8 ? c_tc.woff8[i] : c_tc.woff[i]; }
__device__ __forceinline__ int kTcBias(int i) { return c_tc.boff[i]; }

constexpr int kGroups = 4;
constexpr int kTrunkBytes = 3 * 128 * 32 * 2;  // 24 KB
constexpr int kHeadBytes = 128 * 128 * 2;      // 32 KB
// The trunk tiles and the head tile of a group share one region: every
// layer's MMA has completed (mbarrier) before its epilogue overwrites it.
constexpr int kGroupBytes = kHeadBytes;
static_assert(kTrunkBytes <= kHeadBytes, "trunk tiles alias the head tile");
template <bool F8>
constexpr int smem_bytes() { return (F8 ? kW8Bytes : kWBytes) + kGroups * kGroupBytes + 64 * kGroups + 16; }
constexpr int kSmemBytes = smem_bytes<false>();
constexpr int kTmemCols = 512;  // 128 per group (power of two allocation)
static_assert(128 * kGroups <= kTmemCols, "tensor memory budget");
static_assert(kSmemBytes <= 232448, "shared memory budget");


__device__ __forceinline__ void group_bar(int g) { asm volatile("bar.sync %0, 128;" ::"r"(g + 1) : "memory"); }

__device__ __forceinline__ uint32_t pack_bf16(float a, float b) {
  __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<uint32_t*>(&h);
}
// Row `row` of a K-major tile with KP columns from x[0..KP) (fp32 -> bf16).
template <int KP>
__device__ __forceinline__ void store_row(uint8_t* tile, int row, const float* x) {
#pragma unroll
  for (int kg = 0; kg < KP / 8; ++kg) {
    uint4 q;
    q.x = pack_bf16(x[8 * kg + 0], x[8 * kg + 1]);
    q.y = pack_bf16(x[8 * kg + 2], x[8 * kg + 3]);
    q.z = pack_bf16(x[8 * kg + 4], x[8 * kg + 5]);
    q.w = pack_bf16(x[8 * kg + 6], x[8 * kg + 7]);
    *reinterpret_cast<uint4*>(tile + canon_off(row, 8 * kg, KP)) = q;
  }
}
// N columns starting at column k0 (a multiple of 8) of row `row`.
template <int KP, int N>
__device__ __forceinline__ void store_cols(uint8_t* tile, int row, int k0, const float* x) {
#pragma unroll
  for (int kg = 0; kg < N / 8; ++kg) {
    uint4 q;
    q.x = pack_bf16(x[8 * kg + 0], x[8 * kg + 1]);
    q.y = pack_bf16(x[8 * kg + 2], x[8 * kg + 3]);
    q.z = pack_bf16(x[8 * kg + 4], x[8 * kg + 5]);
    q.w = pack_bf16(x[8 * kg + 6], x[8 * kg + 7]);
    *reinterpret_cast<uint4*>(tile + canon_off(row, k0 + 8 * kg, KP)) = q;
  }
}
template <int KP>
__device__ __forceinline__ void load_row(const uint8_t* tile, int row, float* x) {
#pragma unroll
  for (int kg = 0; kg < KP / 8; ++kg) {
    uint4 q = *reinterpret_cast<const uint4*>(tile + canon_off(row, 8 * kg, KP));
    uint32_t w[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      x[8 * kg + 2 * j] = __uint_as_float(w[j] << 16);
      x[8 * kg + 2 * j + 1] = __uint_as_float(w[j] & 0xFFFF0000u);
    }
  }
}

// Issue D[tmem] = A[128 x KP] * W[NP x KP]^T as KP/16 MMAs.
template <int NP, int KP>
__device__ __forceinline__ void issue_layer(uint32_t tmem_d, uint32_t a_addr, uint32_t w_addr) {
  constexpr uint32_t id = idesc_bf16(128, NP);
#pragma unroll
  for (int s = 0; s < KP / 16; ++s) {
    uint64_t da = sdesc(a_addr + s * 256, 128, (KP / 8) * 128);
    uint64_t db = sdesc(w_addr + s * 256, 128, (KP / 8) * 128);
    umma_bf16(tmem_d, da, db, id, s > 0 ? 1u : 0u);
  }
}

// ---- E4M3 operands (MR_PREC_FP8) ------------------------------------------------
// 8-bit K-major tiles keep the byte structure of the BF16 ones: 16-byte
// core-matrix rows (16 elements), 8-row groups SBO apart, K halves of one MMA
// (K = 32) 128 bytes apart. Values are stored multiplied by a power-of-two
// scale chosen per row and operand (max |x| -> at most 448, the largest
// E4M3 value); the epilogue multiplies the FP32 accumulator by the inverse
// row scale and the layer's inverse weight scale.
template <bool F8>
__host__ __device__ constexpr int qoff(int row, int k, int kp) {
  return F8 ? ((row >> 3) * (kp >> 4) + (k >> 4)) * 128 + (row & 7) * 16 + (k & 15) : canon_off(row, k, kp);
}
template <bool F8>
__host__ __device__ constexpr int qkp(int k) { return F8 ? kp8(k) : pad16(k); }

// two floats -> E4M3x2 (first value in the low byte), round to nearest, saturating
__device__ __forceinline__ uint32_t pack_e4m3x2(float lo, float hi) {
  uint16_t r;
  asm("{\n\t.reg .b16 t;\n\tcvt.rn.satfinite.e4m3x2.f32 t, %2, %1;\n\tmov.b16 %0, t;\n\t}\n"
      : "=h"(r) : "f"(lo), "f"(hi));
  return r;
}
// Power-of-two scale mapping max |x| = m to at most 448.
__device__ __forceinline__ float q_scale(float m) {
  if (!(m > 0.0f)) return 1.0f;
  const float e = fminf(fmaxf(floorf(log2f(448.0f / m)), -24.0f), 24.0f);
  return exp2f(e);
}
// N (multiple of 8) values x[0..N) to columns k0.. (multiple of 8) of a row;
// `s` scales the values of an 8-bit tile.
template <bool F8, int KP, int N>
__device__ __forceinline__ void store_q(uint8_t* tile, int row, int k0, const float* x, float s) {
#pragma unroll
  for (int kg = 0; kg < N / 8; ++kg) {
    const float* v = x + 8 * kg;
    if constexpr (F8) {
      uint2 q;
      q.x = pack_e4m3x2(v[0] * s, v[1] * s) | (pack_e4m3x2(v[2] * s, v[3] * s) << 16);
      q.y = pack_e4m3x2(v[4] * s, v[5] * s) | (pack_e4m3x2(v[6] * s, v[7] * s) << 16);
      *reinterpret_cast<uint2*>(tile + qoff<true>(row, k0 + 8 * kg, KP)) = q;
    } else {
      uint4 q;
      q.x = pack_bf16(v[0], v[1]);
      q.y = pack_bf16(v[2], v[3]);
      q.z = pack_bf16(v[4], v[5]);
      q.w = pack_bf16(v[6], v[7]);
      *reinterpret_cast<uint4*>(tile + canon_off(row, k0 + 8 * kg, KP)) = q;
    }
  }
}
// Whole row of KP values with its own scale; returns the inverse scale (1 for BF16).
template <bool F8, int KP>
__device__ __forceinline__ float store_row_q(uint8_t* tile, int row, const float* x) {
  float s = 1.0f;
  if constexpr (F8) {
    float m = 0.0f;
#pragma unroll
    for (int i = 0; i < KP; ++i) m = fmaxf(m, fabsf(x[i]));
    s = q_scale(m);
  }
  store_q<F8, KP, KP>(tile, row, 0, x, s);
  return 1.0f / s;
}

__device__ __forceinline__ void umma_f8(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f8f6f4 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"(acc)
      : "memory");
}
// Instruction descriptor: E4M3 x E4M3 -> FP32, A and B K-major, M x N.
__host__ __device__ constexpr uint32_t idesc_e4m3(int m, int n) {
  return (1u << 4) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}
// D[tmem] = A[128 x KP] * W[NP x KP]^T; KP in elements of the operand type.
template <bool F8, int NP, int KP>
__device__ __forceinline__ void issue_q(uint32_t tmem_d, uint32_t a_addr, uint32_t w_addr) {
  if constexpr (F8) {
    static_assert(KP % 32 == 0, "E4M3 K step is 32");
    constexpr uint32_t id = idesc_e4m3(128, NP);
#pragma unroll
    for (int s = 0; s < KP / 32; ++s) {
      uint64_t da = sdesc(a_addr + s * 256, 128, (KP / 16) * 128);
      uint64_t db = sdesc(w_addr + s * 256, 128, (KP / 16) * 128);
      umma_f8(tmem_d, da, db, id, s > 0 ? 1u : 0u);
    }
  } else {
    issue_layer<NP, KP>(tmem_d, a_addr, w_addr);
  }
}

__device__ __forceinline__ float sigm(float x) { return 1.0f / (1.0f + expf(-x)); }

// Read of the row-wise weight image (kernel parameter space).
__device__ __forceinline__ float ldw(const float* p) { return *p; }

struct TcArgs {
  const uint8_t* __restrict__ wpack;  // kWBytes packed bf16 image
  const float* __restrict__ w;        // fp32 blob
  const float* __restrict__ desc;     // row k, chunk j (features 4j..4j+3) at desc[k*rs + j*cs]
  long long rs, cs, ars, afs;         // descriptor / aux strides
  const float* __restrict__ aux;      // n x 5
  int n;
  float* out;                         // n x 3, or image when pix != null
  const int* __restrict__ pix;        // compose mode: pixel index per record
  const float* __restrict__ trph;     // compose mode: single-scatter term
  const unsigned* __restrict__ count; // compose mode: number of records (device)
  F3 light_color, scatter;
  const int* __restrict__ job;        // batched compose: job of each record (null: single image)
  const BatchOut* __restrict__ bout;  // batched compose: per-job outputs
  float* spill;                       // 120 x spill_cap ungated head columns (multi-channel tiles)
  long long spill_cap;
  int* err;                           // set on a wait timeout
  const uint8_t* __restrict__ wpack8; // kW8Bytes packed E4M3 image (MR_PREC_FP8)
  float winv[kTcLayers];              // inverse per-layer weight scales (1 for BF16)
  float4 se[kSeRecs * kSeRecFloats / 4];  // squeeze-excitation records (kSeRecSrc)
  alignas(16) float rw[kRowFloats];   // row-wise fp32 weights (make_row_table)
};

static_assert(sizeof(TcArgs) <= 32764, "kernel parameter space");

// One descriptor row in chunk-of-4 order: features i..i+3 (i a multiple of
// 4) are the float4 at p + (i/4)*cs, cs = 4*capacity for the render path's
// chunked columns and 4 for row-major input. The address is formed inside
// the asm so that the compiler cannot keep hundreds of row addresses live
// across the MMA waits.
struct DIn {
  const float* __restrict__ p;
  int cs16;  // chunk stride in bytes
  __device__ __forceinline__ float4 ld4(int i) const {
    float4 v;
    asm volatile(
        "{\n\t.reg .u64 a;\n\tmad.wide.s32 a, %4, %5, %6;\n\tld.global.nc.v4.f32 {%0,%1,%2,%3}, [a];\n\t}\n"
        : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
        : "r"(i >> 2), "r"(cs16), "l"(p));
    return v;
  }
};

struct GroupCtx {
  uint8_t* trunk;   // 3 x (128 x 32) tiles
  uint8_t* head;    // 128 x 128 tile
  uint32_t tmem;    // this group's column base
  uint32_t tlane;   // this warp's TMEM lane quarter (lane << 16)
  uint32_t mbar;
  uint32_t phase;
  int g, t;         // group, row (0..127)
  const uint8_t* wsm;
  bool ok;
};

// One MMA round: make A visible, issue (thread 0), wait for completion.
template <typename IssueFn>
__device__ __forceinline__ void mma_round(GroupCtx& c, IssueFn issue) {
  fence_async_smem();
  tc_fence_before();
  group_bar(c.g);
  if (c.t == 0) {
    tc_fence_after();
    issue();
    umma_commit(c.mbar);
  }
  // A thread that timed out once stops waiting but keeps the group's barrier
  // sequence, so the group never deadlocks; the error word is set at exit.
  if (c.ok && !mbar_wait(c.mbar, c.phase)) c.ok = false;
  c.phase ^= 1u;
  tc_fence_after();
}

// Reads back N (<= 32) columns at TMEM column `col`, adds the bias and
// applies ReLU.
template <int N>
__device__ __forceinline__ void epi_relu(const GroupCtx& c, int col, const float* __restrict__ bias, float* y,
                                         float sc = 1.0f) {
  float v[16];
#pragma unroll
  for (int h = 0; h < (N + 15) / 16; ++h) {
    tmem_ld16(c.tmem + c.tlane + col + 16 * h, v);
#pragma unroll
    for (int i = 0; i < 16; ++i)
      if (16 * h + i < N) {
        float a = ldw(bias + 16 * h + i) + v[i] * sc;
        y[16 * h + i] = a >= 0.0f ? a : 0.0f;
      }
  }
}

// Split MMA round: issue (after making this group's A rows visible to the
// tensor core), then wait. Work between the two overlaps the MMA.
template <typename IssueFn>
__device__ __forceinline__ void mma_issue(GroupCtx& c, IssueFn issue) {
  fence_async_smem();
  tc_fence_before();
  group_bar(c.g);
  if (c.t == 0) {
    tc_fence_after();
    issue();
    umma_commit(c.mbar);
  }
}
__device__ __forceinline__ void mma_wait(GroupCtx& c) {
  if (c.ok && !mbar_wait(c.mbar, c.phase)) c.ok = false;
  c.phase ^= 1u;
  tc_fence_after();
}

// 8 fp32 values to / from this thread's TMEM lane (columns col..col+7).
__device__ __forceinline__ void tmem_st8(uint32_t taddr, const float* v) {
  asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};\n" ::"r"(taddr),
               "r"(__float_as_uint(v[0])), "r"(__float_as_uint(v[1])), "r"(__float_as_uint(v[2])),
               "r"(__float_as_uint(v[3])), "r"(__float_as_uint(v[4])), "r"(__float_as_uint(v[5])),
               "r"(__float_as_uint(v[6])), "r"(__float_as_uint(v[7]))
               : "memory");
  asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
}
// 8 columns; load and wait in one asm statement, so that no use of the
// loaded registers is scheduled before the wait.
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float* v) {
  uint32_t r[8];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];\n\t"
               "tcgen05.wait::ld.sync.aligned;\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
               : "r"(taddr)
               : "memory");
#pragma unroll
  for (int i = 0; i < 8; ++i) v[i] = __uint_as_float(r[i]);
}

constexpr int kBr = 128 * 32 * 2;  // bytes of one branch tile (K <= 32)

// Pooled statistics of one trunk block's three descriptor segments
// (radiancePredict.cu:240-294): mean and max, their LSEFin1 contributions
// (pool[pid+br], pool[36+pid+br]) and the block's squeeze-excitation gates.
// Depends only on the descriptor, g and gamma, so it runs while the previous
// layer's MMA is in flight.
template <int S>
__device__ __forceinline__ void block_prep(const DIn& d, const float4* __restrict__ rec, int from, float g, float gamma,
                                           float* fin, float* gate) {
  float mean[3], mx[3];
#pragma unroll
  for (int br = 0; br < 3; ++br) {
    float s = 0.0f, m = -10000.0f;
#pragma unroll
    for (int i = 0; i < S; i += 4) {
      const float4 q = d.ld4(br * 192 + from + i);
      s += q.x; s += q.y; s += q.z; s += q.w;
      m = fmaxf(fmaxf(m, q.x), fmaxf(q.y, fmaxf(q.z, q.w)));
    }
    mean[br] = s / (float)S;
    mx[br] = m;
  }
  // LSEFin1 terms: per output j the weights of (mean b0..b2, max b0..b2)
#pragma unroll
  for (int j = 0; j < 16; j += 2) {
    const float4 q0 = rec[3 * (j / 2)], q1 = rec[3 * (j / 2) + 1], q2 = rec[3 * (j / 2) + 2];
    const float wa[12] = {q0.x, q0.y, q0.z, q0.w, q1.x, q1.y, q1.z, q1.w, q2.x, q2.y, q2.z, q2.w};
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      float a = fin[j + u];
#pragma unroll
      for (int br = 0; br < 3; ++br) {
        a += mean[br] * wa[6 * u + br];
        a += mx[br] * wa[6 * u + 3 + br];
      }
      fin[j + u] = a;
    }
  }
  const float tmp[8] = {mean[0], mean[1], mean[2], mx[0], mx[1], mx[2], g, gamma};
  float h[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const float4 q0 = rec[24 + 2 * i], q1 = rec[25 + 2 * i];
    const float wr[8] = {q0.x, q0.y, q0.z, q0.w, q1.x, q1.y, q1.z, q1.w};
    float a = 0.0f;
#pragma unroll
    for (int j = 0; j < 8; ++j) a += tmp[j] * wr[j];
    h[i] = a >= 0.0f ? a : 0.0f;
  }
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    const float4 q0 = rec[40 + 2 * i], q1 = rec[41 + 2 * i];
    const float wr[8] = {q0.x, q0.y, q0.z, q0.w, q1.x, q1.y, q1.z, q1.w};
    float a = 0.0f;
#pragma unroll
    for (int j = 0; j < 8; ++j) a += h[j] * wr[j];
    gate[i] = sigm(a);
  }
}

// A rows of a block that starts a trunk (SE, no residual input): seg * gate.
template <bool F8, int S>
__device__ __forceinline__ void store_first(GroupCtx& c, const DIn& d, int from, const float* gate, float* ainv) {
  constexpr int KP = qkp<F8>(S);
#pragma unroll
  for (int br = 0; br < 3; ++br) {
    float x[KP];
#pragma unroll
    for (int i = 0; i < KP; i += 4) {
      if (i < S) {
        const float4 q = d.ld4(br * 192 + from + i);
        x[i] = q.x * gate[br]; x[i + 1] = q.y * gate[br]; x[i + 2] = q.z * gate[br]; x[i + 3] = q.w * gate[br];
      } else {
        x[i] = x[i + 1] = x[i + 2] = x[i + 3] = 0.0f;
      }
    }
    ainv[br] = store_row_q<F8, KP>(c.trunk + br * kBr, c.t, x);
  }
}

// Epilogue of trunk block (S, MODE) at descriptor offset `from`:
// yn = ReLU(acc + b); y = yn + seg (ADD3) or [yn, seg] (REP3, MODE 2).
// next_y false: writes the next block's A rows seg2 * gate2 + y (SERES input,
// radiancePredict.cu:259-294); true: writes y (input of L81 / LD41).
template <bool F8, int S, int MODE>
__device__ __forceinline__ void block_epi(GroupCtx& c, const DIn& d, const float* __restrict__ w, int layer0, int from,
                                          int from2, bool next_y, const float* gate2, float* ainv, const float* winv) {
  constexpr int W = MODE == 2 ? 2 * S : S;
  constexpr int KP = qkp<F8>(W);
#pragma unroll
  for (int br = 0; br < 3; ++br) {
    const float4* bias = reinterpret_cast<const float4*>(w + kTcBias(layer0 + br));  // 16-byte aligned
    const float sc = F8 ? ainv[br] * winv[layer0 + br] : 1.0f;
    float y[KP];
#pragma unroll
    for (int h = 0; h < (S + 15) / 16; ++h) {
      float v[16];
      tmem_ld16(c.tmem + c.tlane + 32 * br + 16 * h, v);
#pragma unroll
      for (int i = 0; i < 16; i += 4)
        if (16 * h + i < S) {
          const float4 bq = bias[(16 * h + i) / 4];
          const float bb[4] = {bq.x, bq.y, bq.z, bq.w};
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            const float a = v[i + u] * sc + bb[u];
            y[16 * h + i + u] = a >= 0.0f ? a : 0.0f;
          }
        }
    }
#pragma unroll
    for (int i = 0; i < S; i += 4) {
      const float4 q = d.ld4(br * 192 + from + i);
      const float sv[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        if (MODE == 2) y[S + i + u] = sv[u];
        else y[i + u] = y[i + u] + sv[u];
      }
    }
#pragma unroll
    for (int i = W; i < KP; ++i) y[i] = 0.0f;
    if (!next_y) {
#pragma unroll
      for (int i = 0; i < W; i += 4) {
        const float4 q = d.ld4(br * 192 + from2 + i);
        y[i] = q.x * gate2[br] + y[i];
        y[i + 1] = q.y * gate2[br] + y[i + 1];
        y[i + 2] = q.z * gate2[br] + y[i + 2];
        y[i + 3] = q.w * gate2[br] + y[i + 3];
      }
    }
    ainv[br] = store_row_q<F8, KP>(c.trunk + br * kBr, c.t, y);
  }
}

// Three branch MMAs of a trunk layer with S outputs and S inputs.
template <bool F8, int S>
__device__ __forceinline__ void issue_trunk(GroupCtx& c, int layer0) {
  const uint32_t tb = smem_u32(c.trunk), wb = smem_u32(c.wsm);
  mma_issue(c, [&]() {
#pragma unroll
    for (int br = 0; br < 3; ++br)
      issue_q<F8, pad16(S), qkp<F8>(S)>(c.tmem + 32 * br, tb + br * kBr, wb + tc_off<F8>(layer0 + br));
  });
}

// The trunks as a sequence of MMA rounds (radiancePredict.cu:396-437): round
// r computes the squeeze-excitation gates of the block it issues (prep),
// waits for the previous round's MMAs, writes their epilogue as this block's
// A rows (or, for a trunk's first block, the gated descriptor segment), and
// issues the block's three branch MMAs. The rounds run from this table in
// one rolled loop, so that every round executes the same few instantiations
// (three widths) instead of a straight-line copy per block: the four tile
// groups of a CTA, each at its own round, then share a small instruction
// working set.
enum { TS_FIRST = 0, TS_EPI = 1, TS_LD41 = 2 };
struct TrunkStep {
  short prep_from, rec, prep_s;              // prep_s 0: no gates to compute; rec: kSeRecSrc index
  short kind, epi_layer, epi_s, cat, next_y, from, from2;
  short layer, s;                            // the block issued
};
#define TS_PREP(f, rec, S) f, rec, S
#define TS_NOPREP 0, 0, 0
__constant__ TrunkStep c_trunk[14] = {
    // light-direction trunk: blocks at 160, 168, 176, 184, then LD41
    {TS_PREP(160, 0, 8), TS_FIRST, 0, 0, 0, 0, 160, 0, TC_DI + 0, 8},
    {TS_PREP(168, 1, 8), TS_EPI, TC_DI + 0, 8, 0, 0, 160, 168, TC_DI + 3, 8},
    {TS_PREP(176, 2, 8), TS_EPI, TC_DI + 3, 8, 0, 0, 168, 176, TC_DI + 6, 8},
    {TS_PREP(184, 3, 8), TS_EPI, TC_DI + 6, 8, 0, 0, 176, 184, TC_DI + 9, 8},
    {TS_PREP(0, 4, 8), TS_EPI, TC_DI + 9, 8, 0, 1, 184, 0, TC_LD41, 8},
    // main trunk: LD41 parked in TMEM, then blocks 0..7 and L81
    {TS_NOPREP, TS_LD41, 0, 0, 0, 0, 0, 0, TC_MAIN + 0, 8},
    {TS_PREP(8, 5, 8), TS_EPI, TC_MAIN + 0, 8, 0, 0, 0, 8, TC_MAIN + 3, 8},
    {TS_PREP(16, 6, 16), TS_EPI, TC_MAIN + 3, 8, 1, 0, 8, 16, TC_MAIN + 6, 16},
    {TS_PREP(32, 7, 16), TS_EPI, TC_MAIN + 6, 16, 0, 0, 16, 32, TC_MAIN + 9, 16},
    {TS_PREP(48, 8, 16), TS_EPI, TC_MAIN + 9, 16, 0, 0, 32, 48, TC_MAIN + 12, 16},
    {TS_PREP(64, 9, 32), TS_EPI, TC_MAIN + 12, 16, 1, 0, 48, 64, TC_MAIN + 15, 32},
    {TS_PREP(96, 10, 32), TS_EPI, TC_MAIN + 15, 32, 0, 0, 64, 96, TC_MAIN + 18, 32},
    {TS_PREP(128, 11, 32), TS_EPI, TC_MAIN + 18, 32, 0, 0, 96, 128, TC_MAIN + 21, 32},
    {TS_NOPREP, TS_EPI, TC_MAIN + 21, 32, 0, 1, 128, 0, TC_L81, 32},
};
#undef TS_PREP
#undef TS_NOPREP

__device__ __forceinline__ void prep_any(int S, const DIn& d, const float4* __restrict__ rec, int from, float g,
                                         float gamma, float* fin, float* gate) {
  if (S == 8) block_prep<8>(d, rec, from, g, gamma, fin, gate);
  else if (S == 16) block_prep<16>(d, rec, from, g, gamma, fin, gate);
  else block_prep<32>(d, rec, from, g, gamma, fin, gate);
}
template <bool F8>
__device__ __forceinline__ void epi_any(int S, bool cat, GroupCtx& c, const DIn& d, const float* __restrict__ w,
                                        int layer0, int from, int from2, bool next_y, const float* gate2, float* ainv,
                                        const float* winv) {
  if (S == 8) {
    if (cat) block_epi<F8, 8, 2>(c, d, w, layer0, from, from2, next_y, gate2, ainv, winv);
    else block_epi<F8, 8, 1>(c, d, w, layer0, from, from2, next_y, gate2, ainv, winv);
  } else if (S == 16) {
    if (cat) block_epi<F8, 16, 2>(c, d, w, layer0, from, from2, next_y, gate2, ainv, winv);
    else block_epi<F8, 16, 1>(c, d, w, layer0, from, from2, next_y, gate2, ainv, winv);
  } else {
    block_epi<F8, 32, 1>(c, d, w, layer0, from, from2, next_y, gate2, ainv, winv);
  }
}
template <bool F8>
__device__ __forceinline__ void issue_any(int S, GroupCtx& c, int layer0) {
  if (S == 8) issue_trunk<F8, 8>(c, layer0);
  else if (S == 16) issue_trunk<F8, 16>(c, layer0);
  else issue_trunk<F8, 32>(c, layer0);
}

// Channel-dependent head gates: LGGS(g, gamma, srp) -> x8 (head columns
// 120..127) and the six SEFin gates sep (radiancePredict.cu:439-452).
__device__ __forceinline__ void head_gates(const float* __restrict__ w, const float* fin, float g, float gamma,
                                           float srp, float* x8, float* sep) {
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    float a = g * ldw(w + ROFF(LGGSW) + 3 * i) + gamma * ldw(w + ROFF(LGGSW) + 3 * i + 1) +
              srp * ldw(w + ROFF(LGGSW) + 3 * i + 2);
    a += ldw(w + ROFF(LGGSB) + i);
    x8[i] = a >= 0.0f ? a : 0.0f;
  }
  float sew[16];
  const float* f1 = w + ROFF(LSEFin1W);
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    const float a = fin[j] + g * ldw(f1 + j * 75 + 72) + gamma * ldw(f1 + j * 75 + 73) + srp * ldw(f1 + j * 75 + 74);
    sew[j] = a >= 0.0f ? a : 0.0f;
  }
#pragma unroll
  for (int i = 0; i < 6; ++i) {
    float a = 0.0f;
#pragma unroll
    for (int j = 0; j < 16; ++j) a += sew[j] * ldw(w + ROFF(LSEFin2W) + j + i * 16);
    sep[i] = sigm(a);
  }
}

// Head SC(p) (radiancePredict.cu:439-473) for one albedo channel; the
// gated 128-wide input is already in c.head (inverse row scale ainv for E4M3).
// Returns the output X. With E4M3 operands every layer's outputs get a new row
// scale before they are stored as the next layer's A rows (a first pass over
// TMEM finds the row maximum where the outputs do not fit in registers).
template <bool F8>
__device__ __forceinline__ float head_chain(GroupCtx& c, const float* __restrict__ w, const float* winv, float ainv) {
  const uint32_t hb = smem_u32(c.head), tb = smem_u32(c.trunk), wb = smem_u32(c.wsm);
  float v[32];
  // LC0 128 -> 128, read back and re-stored 32 columns at a time
  mma_round(c, [&]() { issue_q<F8, 128, 128>(c.tmem, hb, wb + tc_off<F8>(TC_LC0)); });
  float sc = F8 ? ainv * winv[TC_LC0] : 1.0f, s = 1.0f;
  if constexpr (F8) {
    float m = 0.0f;
#pragma unroll 1
    for (int h = 0; h < 4; ++h) {
      epi_relu<32>(c, 32 * h, w + ROFF(LC0B) + 32 * h, v, sc);
#pragma unroll
      for (int i = 0; i < 32; ++i) m = fmaxf(m, v[i]);
    }
    s = q_scale(m);
  }
#pragma unroll 1
  for (int h = 0; h < 4; ++h) {
    epi_relu<32>(c, 32 * h, w + ROFF(LC0B) + 32 * h, v, sc);
    store_q<F8, 128, 32>(c.head, c.t, 32 * h, v, s);
  }
  ainv = 1.0f / s;
  // LC1 128 -> 64
  mma_round(c, [&]() { issue_q<F8, 64, 128>(c.tmem, hb, wb + tc_off<F8>(TC_LC1)); });
  sc = F8 ? ainv * winv[TC_LC1] : 1.0f;
  if constexpr (F8) {
    float m = 0.0f;
#pragma unroll 1
    for (int h = 0; h < 2; ++h) {
      epi_relu<32>(c, 32 * h, w + ROFF(LC1B) + 32 * h, v, sc);
#pragma unroll
      for (int i = 0; i < 32; ++i) m = fmaxf(m, v[i]);
    }
    s = q_scale(m);
  }
#pragma unroll 1
  for (int h = 0; h < 2; ++h) {
    epi_relu<32>(c, 32 * h, w + ROFF(LC1B) + 32 * h, v, sc);
    store_q<F8, 64, 32>(c.trunk, c.t, 32 * h, v, s);
  }
  ainv = 1.0f / s;
  // LC2 64 -> 32
  mma_round(c, [&]() { issue_q<F8, 32, 64>(c.tmem, tb, wb + tc_off<F8>(TC_LC2)); });
  epi_relu<32>(c, 0, w + ROFF(LC2B), v, F8 ? ainv * winv[TC_LC2] : 1.0f);
  ainv = store_row_q<F8, 32>(c.trunk, c.t, v);
  // LX 32 -> 16
  mma_round(c, [&]() { issue_q<F8, 16, 32>(c.tmem, tb, wb + tc_off<F8>(TC_LX)); });
  float a[16], b[32];
  epi_relu<16>(c, 0, w + ROFF(LXB), a, F8 ? ainv * winv[TC_LX] : 1.0f);
  constexpr int K16 = qkp<F8>(16);
#pragma unroll
  for (int i = 16; i < 32; ++i) b[i] = 0.0f;
  // six residual pairs (:454-471)
#pragma unroll 1
  for (int r = 0; r < 6; ++r) {
#pragma unroll
    for (int i = 0; i < 16; ++i) b[i] = a[i];
    ainv = store_row_q<F8, K16>(c.trunk, c.t, b);
    int l0 = TC_LXR + 2 * r, l1 = l0 + 1;
    mma_round(c, [&]() { issue_q<F8, 16, K16>(c.tmem, tb, wb + tc_off<F8>(l0)); });
    epi_relu<16>(c, 0, w + kTcBias(l0), b, F8 ? ainv * winv[l0] : 1.0f);
    ainv = store_row_q<F8, K16>(c.trunk, c.t, b);
    mma_round(c, [&]() { issue_q<F8, 16, K16>(c.tmem, tb, wb + tc_off<F8>(l1)); });
    epi_relu<16>(c, 0, w + kTcBias(l1), b, F8 ? ainv * winv[l1] : 1.0f);
#pragma unroll
    for (int i = 0; i < 16; ++i) a[i] = a[i] + b[i];
  }
  // LX12 16 -> 1, bias after the sum (LinearReLU, :41-56)
  float o = 0.0f;
#pragma unroll
  for (int i = 0; i < 16; ++i) o += a[i] * ldw(w + ROFF(LX12W) + i);
  o += ldw(w + ROFF(LX12B));
  return o >= 0.0f ? o : 0.0f;
}

// Head input of a further albedo channel, from the ungated head columns the
// first pass spilled (feature-major, comb[i] at spill[i*cap + row]); returns
// the inverse row scale of the stored row.
template <bool F8>
__device__ __forceinline__ float head_input_spilled(GroupCtx& c, const float* __restrict__ w, const float* spill,
                                                    long long cap, int row, const float* fin, float g, float gamma,
                                                    float srp) {
  float x8[8], sep[6];
  head_gates(w, fin, g, gamma, srp, x8, sep);
  float s = 1.0f;
  if constexpr (F8) {
    float m = 0.0f;
#pragma unroll
    for (int i = 0; i < 8; ++i) m = fmaxf(m, x8[i]);
#pragma unroll 1
    for (int i = 0; i < 120; ++i) m = fmaxf(m, spill[i * cap + row] * sep[i < 96 ? i / 32 : 3 + (i - 96) / 8]);
    s = q_scale(m);
  }
  store_q<F8, 128, 8>(c.head, c.t, 120, x8, s);
#pragma unroll 1
  for (int g8 = 0; g8 < 15; ++g8) {
    const float sg = sep[g8 < 12 ? g8 / 4 : g8 - 9];
#pragma unroll
    for (int i = 0; i < 8; ++i) x8[i] = spill[(8 * g8 + i) * cap + row] * sg;
    store_q<F8, 128, 8>(c.head, c.t, 8 * g8, x8, s);
  }
  return 1.0f / s;
}

// Group-wide OR of a per-row flag (named barrier g+1 with reduction).
__device__ __forceinline__ bool group_any(int g, bool x) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\tsetp.ne.u32 p, %1, 0;\n\tbar.red.or.pred q, %2, 128, p;\n\tselp.u32 %0, 1, 0, q;\n\t}\n"
      : "=r"(r)
      : "r"((uint32_t)x), "r"(g + 1)
      : "memory");
  return r != 0;
}

template <bool F8>
__global__ void __launch_bounds__(128 * kGroups, 1) k_mlp_tc(const __grid_constant__ TcArgs a) {
  constexpr int WB = F8 ? kW8Bytes : kWBytes;
  extern __shared__ __align__(1024) uint8_t smem[];
  uint8_t* wsm = smem;
  uint8_t* gbase = smem + WB;
  uint64_t* mbars = reinterpret_cast<uint64_t*>(smem + WB + kGroups * kGroupBytes);
  uint32_t* tmem_holder = reinterpret_cast<uint32_t*>(mbars + kGroups);
  const int tid = threadIdx.x, warp = tid >> 5;
  const int g = tid >> 7, t = tid & 127;
  // weights -> shared memory (16-byte vectors)
  const uint4* wsrc = reinterpret_cast<const uint4*>(F8 ? a.wpack8 : a.wpack);
  for (int i = tid; i < WB / 16; i += blockDim.x) reinterpret_cast<uint4*>(wsm)[i] = __ldg(wsrc + i);
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_holder)),
                 "r"(kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (t == 0) mbar_init(smem_u32(mbars + g), 1);
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  fence_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();

  GroupCtx c;
  c.trunk = gbase + g * kGroupBytes;
  c.head = c.trunk;
  c.tmem = *tmem_holder + (uint32_t)(128 * g);
  c.tlane = (uint32_t)(32 * (warp & 3)) << 16;
  c.mbar = smem_u32(mbars + g);
  c.phase = 0;
  c.g = g;
  c.t = t;
  c.wsm = wsm;
  c.ok = true;
  const float* __restrict__ w = a.rw;
  const int n = a.pix ? (int)min(*a.count, (unsigned)a.n) : a.n;
  // TMEM columns 96..119 of the group hold the light trunk's LD41 output
  // while the main trunk (columns 0..95) runs.
  const uint32_t tcomb = c.tmem + c.tlane + 96;

  for (int it = 0;; ++it) {
    // static tile striding over (CTA, group)
    const int tile = (it * (int)gridDim.x + (int)blockIdx.x) * kGroups + g;
    if (tile * 128 >= n) break;  // group-uniform exit
    const int row = tile * 128 + t;
    const int kk = row < n ? row : n - 1;
    const DIn d{a.desc + (long long)kk * a.rs, (int)(a.cs * 4)};
    const float* ax = a.aux + (long long)kk * a.ars;
    const float gg = __ldg(ax), gamma = __ldg(ax + a.afs);
    float srp[3] = {__ldg(ax + 2 * a.afs), __ldg(ax + 3 * a.afs), __ldg(ax + 4 * a.afs)};
    // further heads (radiancePredict.cu:478-483), decided for the whole tile
    const bool need1 = group_any(g, srp[1] != srp[0]);
    const bool need2 = group_any(g, srp[2] != srp[0] && srp[2] != srp[1]);
    float fin[16];
#pragma unroll
    for (int j = 0; j < 16; ++j) fin[j] = 0.0f;
    float gate[3], ainv[3];  // ainv: inverse E4M3 row scales of the three branch A rows (1 for BF16)
    const float* winv = a.winv;

#pragma unroll 1
    for (int r = 0; r < 14; ++r) {
      const TrunkStep& st = c_trunk[r];
      if (st.prep_s) prep_any(st.prep_s, d, a.se + st.rec * (kSeRecFloats / 4), st.prep_from, gg, gamma, fin, gate);
      if (st.kind != TS_FIRST) mma_wait(c);
      if (st.kind == TS_EPI) {
        epi_any<F8>(st.epi_s, st.cat != 0, c, d, w, st.epi_layer, st.from, st.from2, st.next_y != 0, gate, ainv,
                    winv);
      } else {
        if (st.kind == TS_LD41) {
          // LD41 -> comb[96..120), parked in TMEM
#pragma unroll
          for (int br = 0; br < 3; ++br) {
            float v[8];
            tmem_ld8(c.tmem + c.tlane + 32 * br, v);
            const float* bias = w + kTcBias(TC_LD41 + br);
            const float sc = F8 ? ainv[br] * winv[TC_LD41 + br] : 1.0f;
#pragma unroll
            for (int i = 0; i < 8; ++i) {
              const float x = v[i] * sc + ldw(bias + i);
              v[i] = x >= 0.0f ? x : 0.0f;
            }
            tmem_st8(tcomb + 8 * br, v);
          }
        }
        store_first<F8, 8>(c, d, st.from, gate, ainv);  // a trunk's first block: seg * gate
      }
      issue_any<F8>(st.s, c, st.layer);
    }
    // channel-0 head gates while L81 runs (fin is complete)
    float x8[8], sep[6];
    head_gates(w, fin, gg, gamma, srp[0], x8, sep);
    mma_wait(c);
    // L81 -> comb[0..96); gated head input for channel 0 (:439-452)
    const bool spill = (need1 || need2) && a.spill != nullptr;
    const long long cap = a.spill_cap;
    float hs = 1.0f;  // E4M3 scale of the head row
    if constexpr (F8) {
      float m = 0.0f;
#pragma unroll
      for (int i = 0; i < 8; ++i) m = fmaxf(m, x8[i]);
#pragma unroll
      for (int br = 0; br < 3; ++br) {
        const float* bias = w + kTcBias(TC_L81 + br);
        const float sc = ainv[br] * winv[TC_L81 + br];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          float v[16];
          tmem_ld16(c.tmem + c.tlane + 32 * br + 16 * h, v);
#pragma unroll
          for (int i = 0; i < 16; ++i) m = fmaxf(m, fmaxf(v[i] * sc + ldw(bias + 16 * h + i), 0.0f) * sep[br]);
        }
        float v8[8];
        tmem_ld8(tcomb + 8 * br, v8);
#pragma unroll
        for (int i = 0; i < 8; ++i) m = fmaxf(m, v8[i] * sep[3 + br]);
      }
      hs = q_scale(m);
    }
#pragma unroll
    for (int br = 0; br < 3; ++br) {
      const float* bias = w + kTcBias(TC_L81 + br);
      const float sc = F8 ? ainv[br] * winv[TC_L81 + br] : 1.0f;
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        float v[16];
        tmem_ld16(c.tmem + c.tlane + 32 * br + 16 * h, v);
#pragma unroll
        for (int i = 0; i < 16; ++i) {
          const float x = v[i] * sc + ldw(bias + 16 * h + i);
          v[i] = x >= 0.0f ? x : 0.0f;
        }
        if (spill && row < n) {
#pragma unroll
          for (int i = 0; i < 16; ++i) a.spill[(32 * br + 16 * h + i) * cap + row] = v[i];
        }
#pragma unroll
        for (int i = 0; i < 16; ++i) v[i] *= sep[br];
        store_q<F8, 128, 16>(c.head, c.t, 32 * br + 16 * h, v, hs);
      }
    }
#pragma unroll
    for (int br = 0; br < 3; ++br) {
      float v[8];
      tmem_ld8(tcomb + 8 * br, v);
      if (spill && row < n) {
#pragma unroll
        for (int i = 0; i < 8; ++i) a.spill[(96 + 8 * br + i) * cap + row] = v[i];
      }
#pragma unroll
      for (int i = 0; i < 8; ++i) v[i] *= sep[3 + br];
      store_q<F8, 128, 8>(c.head, c.t, 96 + 8 * br, v, hs);
    }
    store_q<F8, 128, 8>(c.head, c.t, 120, x8, hs);
    // heads: channel 0, then the further distinct channels of the tile
    float X[3] = {0.0f, 0.0f, 0.0f};
#pragma unroll 1
    for (int ch = 0; ch < 3; ++ch) {
      if ((ch == 1 && !need1) || (ch == 2 && !need2)) continue;
      if (ch > 0) {
        if (a.spill == nullptr) {  // host contract: multi-channel tiles need the spill buffer
          c.ok = false;
          break;
        }
        hs = 1.0f / head_input_spilled<F8>(c, w, a.spill, cap, row < n ? row : 0, fin, gg, gamma,
                                               ch == 1 ? srp[1] : srp[2]);
      }
      const float x = head_chain<F8>(c, w, winv, 1.0f / hs);
      if (ch == 0) X[0] = x;
      else if (ch == 1) X[1] = x;
      else X[2] = x;
    }
    if (srp[1] == srp[0]) X[1] = X[0];
    if (srp[2] == srp[0]) X[2] = X[0];
    else if (srp[2] == srp[1]) X[2] = X[1];
    if (row < n) {
      float o[3];
#pragma unroll
      for (int ch = 0; ch < 3; ++ch) o[ch] = fmaxf(expf(X[ch]) - 1.0f, 0.0f) * srp[ch];
      if (a.pix) {
        const int px = a.pix[row];
        const float tr = a.trph[row];
        F3 lcv = a.light_color, scv = a.scatter;
        float* dst = a.out;
        if (a.job) {
          const BatchOut& bo = a.bout[a.job[row]];
          lcv = bo.light_color;
          scv = bo.scatter;
          dst = bo.out;
        }
        const float lc[3] = {lcv.x, lcv.y, lcv.z};
        const float sc[3] = {scv.x, scv.y, scv.z};
#pragma unroll
        for (int ch = 0; ch < 3; ++ch) dst[3 * (size_t)px + ch] = fmaxf(((o[ch] + tr) * lc[ch]) * sc[ch], 0.0f);
      } else {
#pragma unroll
        for (int ch = 0; ch < 3; ++ch) a.out[3 * (size_t)row + ch] = o[ch];
      }
    }
  }
  if (!c.ok) atomicExch(a.err, 1);
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(*tmem_holder), "r"(kTmemCols));
  }
}
// Failure path of the bounded waits: allocates tensor memory, initialises an
// mbarrier that nothing will ever arrive on, waits for it with a limit of
// limit_ns, records the timeout in *err with the time waited, and frees the
// tensor memory on the way out, as every kernel of this file does when a wait
// gives up.
__global__ void __launch_bounds__(128, 1) k_tc_wait_selftest(uint64_t limit_ns, int* err,
                                                             unsigned long long* waited_ns) {
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t holder;
  const int t = threadIdx.x, warp = t >> 5;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&holder)),
                 "r"(128));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (t == 0) mbar_init(smem_u32(&mbar), 1);
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = holder;
  const uint64_t t0 = globaltimer();
  const bool ok = mbar_wait(smem_u32(&mbar), 0, limit_ns);  // no arrival: runs out
  const uint64_t t1 = globaltimer();
  if (!ok && t == 0) {
    atomicExch(err, 1);
    *waited_ns = t1 - t0;
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(128));
  }
}

// One tile through the same descriptors: D[128 x N] = A[128 x K] * B[N x K]^T.
template <int N, int K>
__global__ void __launch_bounds__(128, 1) k_tc_selftest(const uint16_t* __restrict__ A, const uint16_t* __restrict__ B,
                                                        float* __restrict__ D, int* err) {
  extern __shared__ __align__(1024) uint8_t dsm[];
  uint8_t* sa = dsm;
  uint8_t* sb = dsm + 128 * K * 2;
  uint64_t& mbar = *reinterpret_cast<uint64_t*>(dsm + 128 * K * 2 + N * K * 2);
  uint32_t& holder = *reinterpret_cast<uint32_t*>(dsm + 128 * K * 2 + N * K * 2 + 8);
  const int t = threadIdx.x, warp = t >> 5;
  for (int k = 0; k < K; ++k) {
    *reinterpret_cast<uint16_t*>(sa + canon_off(t, k, K)) = A[t * K + k];
    if (t < N) *reinterpret_cast<uint16_t*>(sb + canon_off(t, k, K)) = B[t * K + k];
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&holder)),
                 "r"(128));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (t == 0) mbar_init(smem_u32(&mbar), 1);
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  fence_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = holder;
  if (t == 0) {
    issue_layer<N, K>(tmem, smem_u32(sa), smem_u32(sb));
    umma_commit(smem_u32(&mbar));
  }
  const bool ok = mbar_wait(smem_u32(&mbar), 0);
  tc_fence_after();
  if (ok) {
    float v[16];
#pragma unroll
    for (int h = 0; h < N / 16; ++h) {
      tmem_ld16(tmem + ((uint32_t)(32 * warp) << 16) + 16 * h, v);
#pragma unroll
      for (int i = 0; i < 16; ++i) D[t * N + 16 * h + i] = v[i];
    }
  } else if (t == 0) {
    atomicExch(err, 1);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(128));
  }
}

// D[tmem] (+)= A_hi W_hi^T + A_hi W_lo^T + A_lo W_hi^T over KP columns: the
// small terms first, then the large one.
template <int NP, int KP>
__device__ __forceinline__ void issue_tf32x3(uint32_t tmem_d, uint32_t a_hi, uint32_t a_lo, uint32_t w_hi,
                                             uint32_t w_lo, bool accumulate) {
  constexpr uint32_t id = idesc_tf32(128, NP);
  constexpr uint32_t sbo = (KP / 4) * 128;
#pragma unroll
  for (int term = 0; term < 3; ++term) {
    const uint32_t a = term == 1 ? a_lo : a_hi, w = term == 0 ? w_lo : w_hi;
#pragma unroll
    for (int s = 0; s < KP / 8; ++s)
      umma_tf32(tmem_d, sdesc(a + s * 256, 128, sbo), sdesc(w + s * 256, 128, sbo), id,
                (accumulate || term > 0 || s > 0) ? 1u : 0u);
  }
}

// Self-test of the fp32-accurate TF32 path: D[128 x N] = A[128 x K] * B[N x K]^T
// as three TF32 products per element (split 1) or one (split 0).
template <int N, int K>
__global__ void __launch_bounds__(128, 1) k_tc_selftest32(const float* __restrict__ A, const float* __restrict__ B,
                                                          float* __restrict__ D, int* err, int split) {
  extern __shared__ __align__(1024) uint8_t dsm[];
  uint8_t* ah = dsm;
  uint8_t* al = ah + 128 * K * 4;
  uint8_t* bh = al + 128 * K * 4;
  uint8_t* bl = bh + N * K * 4;
  uint64_t& mbar = *reinterpret_cast<uint64_t*>(bl + N * K * 4);
  uint32_t& holder = *reinterpret_cast<uint32_t*>(bl + N * K * 4 + 8);
  const int t = threadIdx.x, warp = t >> 5;
  for (int k = 0; k < K; ++k) {
    float h, l;
    split_tf32(A[t * K + k], h, l);
    *reinterpret_cast<float*>(ah + canon32(t, k, K)) = split ? h : A[t * K + k];
    *reinterpret_cast<float*>(al + canon32(t, k, K)) = l;
    if (t < N) {
      split_tf32(B[t * K + k], h, l);
      *reinterpret_cast<float*>(bh + canon32(t, k, K)) = split ? h : B[t * K + k];
      *reinterpret_cast<float*>(bl + canon32(t, k, K)) = l;
    }
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&holder)),
                 "r"(128));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (t == 0) mbar_init(smem_u32(&mbar), 1);
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  fence_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = holder;
  if (t == 0) {
    if (split) {
      issue_tf32x3<N, K>(tmem, smem_u32(ah), smem_u32(al), smem_u32(bh), smem_u32(bl), false);
    } else {
#pragma unroll
      for (int s = 0; s < K / 8; ++s)
        umma_tf32(tmem, sdesc(smem_u32(ah) + s * 256, 128, (K / 4) * 128),
                  sdesc(smem_u32(bh) + s * 256, 128, (K / 4) * 128), idesc_tf32(128, N), s > 0 ? 1u : 0u);
    }
    umma_commit(smem_u32(&mbar));
  }
  const bool ok = mbar_wait(smem_u32(&mbar), 0);
  tc_fence_after();
  if (ok) {
    float v[16];
#pragma unroll
    for (int h = 0; h < N / 16; ++h) {
      tmem_ld16(tmem + ((uint32_t)(32 * warp) << 16) + 16 * h, v);
#pragma unroll
      for (int i = 0; i < 16; ++i) D[t * N + 16 * h + i] = v[i];
    }
  } else if (t == 0) {
    atomicExch(err, 1);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(128));
  }
}

// The same through the E4M3 path: D[128 x N] = A[128 x K] * B[N x K]^T with
// 8-bit operands (kind::f8f6f4).
template <int N, int K>
__global__ void __launch_bounds__(128, 1) k_tc_selftest8(const uint8_t* __restrict__ A, const uint8_t* __restrict__ B,
                                                         float* __restrict__ D, int* err) {
  extern __shared__ __align__(1024) uint8_t dsm[];
  uint8_t* sa = dsm;
  uint8_t* sb = dsm + 128 * K;
  uint64_t& mbar = *reinterpret_cast<uint64_t*>(dsm + 128 * K + N * K);
  uint32_t& holder = *reinterpret_cast<uint32_t*>(dsm + 128 * K + N * K + 8);
  const int t = threadIdx.x, warp = t >> 5;
  for (int k = 0; k < K; ++k) {
    sa[qoff<true>(t, k, K)] = A[t * K + k];
    if (t < N) sb[qoff<true>(t, k, K)] = B[t * K + k];
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&holder)),
                 "r"(128));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (t == 0) mbar_init(smem_u32(&mbar), 1);
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  fence_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = holder;
  if (t == 0) {
    issue_q<true, N, K>(tmem, smem_u32(sa), smem_u32(sb));
    umma_commit(smem_u32(&mbar));
  }
  const bool ok = mbar_wait(smem_u32(&mbar), 0);
  tc_fence_after();
  if (ok) {
    float v[16];
#pragma unroll
    for (int h = 0; h < N / 16; ++h) {
      tmem_ld16(tmem + ((uint32_t)(32 * warp) << 16) + 16 * h, v);
#pragma unroll
      for (int i = 0; i < 16; ++i) D[t * N + 16 * h + i] = v[i];
    }
  } else if (t == 0) {
    atomicExch(err, 1);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(128));
  }
}

// ---- host ----------------------------------------------------------------------
static uint16_t to_bf16_bits(float f) {
  uint32_t u;
  std::memcpy(&u, &f, 4);
  if ((u & 0x7F800000u) == 0x7F800000u) return (uint16_t)(u >> 16);  // inf / nan
  u += 0x7FFFu + ((u >> 16) & 1u);  // round to nearest even
  return (uint16_t)(u >> 16);
}

// OCP FP8 E4M3 encoding of f (1 sign, 4 exponent bits with bias 7, 3 mantissa
// bits; no infinities; largest finite 448), round to nearest even,
// saturating. Written from the format definition.
static uint8_t to_e4m3(float f) {
  const uint8_t sign = std::signbit(f) ? 0x80 : 0x00;
  const float a = std::fabs(f);
  if (std::isnan(f)) return 0x7f;
  if (a >= 448.0f) return sign | 0x7e;
  if (a < 0.015625f) {  // below 2^-6: subnormal, units of 2^-9
    const int q = (int)std::nearbyint(a * 512.0f);  // 0..8; 8 is the smallest normal (exponent field 1)
    return sign | (uint8_t)q;
  }
  int e;
  std::frexp(a, &e);                                  // a = m 2^e, m in [0.5, 1)
  const float mant = std::ldexp(a, 1 - e);            // [1, 2)
  int q = (int)std::nearbyint((mant - 1.0f) * 8.0f);  // 0..8
  int E = e + 6;                                      // biased exponent of 2^(e-1)
  if (q == 8) { q = 0; ++E; }
  if (E > 15 || (E == 15 && q == 7)) return sign | 0x7e;
  return sign | (uint8_t)((E << 3) | q);
}

void simt_weight_image(const float* w, std::vector<float>& img);  // mr_mlp_simt.cu
void tail_param_image(const float* w, std::vector<float>& out);   // mr_mlp_simt.cu
void light_param_image(const float* w, const std::vector<float>& img, std::vector<float>& out);

int pack_network(Network* n) {
  std::vector<float> w(MR_WEIGHT_TOTAL);
  if (cudaMemcpy(w.data(), n->w, MR_WEIGHT_TOTAL * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess)
    return set_error(MR_ERR_CUDA, "pack_network: weight read-back failed");
  std::vector<uint8_t> img(kWBytes, 0), img8(kW8Bytes, 0);
  const WeightTable wt = make_weight_table();
  // E4M3 image: per layer, weights times a power-of-two scale that maps the
  // largest |w| to at most 448
  n->h_winv8.assign(kTcLayers, 1.0f);
  for (int i = 0; i < kTcLayers; ++i) {
    const TcLayer& L = kTc[i];
    const float* W = w.data() + wt.off[L.w];
    float m = 0.0f;
    for (int j = 0; j < L.n * L.k; ++j) m = std::max(m, std::fabs(W[j]));
    const float sc = m > 0.0f ? std::ldexp(1.0f, (int)std::floor(std::log2(448.0f / m))) : 1.0f;
    n->h_winv8[i] = 1.0f / sc;
    const int kp = kp8(L.k);
    uint8_t* base = img8.data() + tc_offset8(i);
    for (int r = 0; r < L.n; ++r)
      for (int k = 0; k < L.k; ++k) base[qoff<true>(r, k, kp)] = to_e4m3(W[k + r * L.k] * sc);
  }
  for (int i = 0; i < kTcLayers; ++i) {
    const TcLayer& L = kTc[i];
    const int kp = pad16(L.k);
    uint8_t* base = img.data() + tc_offset(i);
    const float* W = w.data() + wt.off[L.w];
    for (int r = 0; r < L.n; ++r)
      for (int k = 0; k < L.k; ++k) {
        uint16_t b = to_bf16_bits(W[k + r * L.k]);
        std::memcpy(base + canon_off(r, k, kp), &b, 2);
      }
  }
  // row-wise fp32 image for the kernel parameters
  const RowTable rt = make_row_table();
  n->h_rowwise.assign(kRowFloats, 0.0f);
  for (int id = 0; id < MR_W_COUNT; ++id)
    if (rt.off[id] >= 0) std::memcpy(&n->h_rowwise[rt.off[id]], w.data() + wt.off[id], wt.size[id] * sizeof(float));
  // squeeze-excitation records of the tensor-core trunk
  n->h_se.assign(kSeRecs * kSeRecFloats, 0.0f);
  for (int r = 0; r < kSeRecs; ++r) {
    float* o = &n->h_se[r * kSeRecFloats];
    const float* f1 = w.data() + wt.off[MR_W_LSEFin1W];
    for (int j = 0; j < 16; ++j)
      for (int b = 0; b < 3; ++b) {
        o[6 * j + b] = f1[j * 75 + kSeRecSrc[r].pid + b];
        o[6 * j + 3 + b] = f1[j * 75 + 36 + kSeRecSrc[r].pid + b];
      }
    std::memcpy(o + 96, w.data() + wt.off[kSeRecSrc[r].se1], 64 * sizeof(float));
    std::memcpy(o + 160, w.data() + wt.off[kSeRecSrc[r].se2], 24 * sizeof(float));
  }
  // weight image of the fp32 kernels
  {
    std::vector<float> si;
    simt_weight_image(w.data(), si);
    tail_param_image(w.data(), n->h_tail);
    light_param_image(w.data(), si, n->h_light);
    cudaError_t e = cudaMalloc(&n->simt_img, si.size() * sizeof(float));
    if (e == cudaSuccess) e = cudaMemcpy(n->simt_img, si.data(), si.size() * sizeof(float), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return set_error(MR_ERR_NOMEM, "pack_network: %s", cudaGetErrorString(e));
  }
  // [BF16 image | error word (256 B) | E4M3 image]
  cudaError_t e = cudaMalloc(&n->packed, kWBytes + 256 + kW8Bytes);
  if (e == cudaSuccess) e = cudaMemcpy(n->packed, img.data(), kWBytes, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset((uint8_t*)n->packed + kWBytes, 0, 256);
  if (e == cudaSuccess)
    e = cudaMemcpy((uint8_t*)n->packed + kWBytes + 256, img8.data(), kW8Bytes, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return set_error(MR_ERR_NOMEM, "pack_network: %s", cudaGetErrorString(e));
  n->packed_bytes = kWBytes;
  return MR_OK;
}

void free_packed(Network* n) {
  if (n->simt_img) cudaFree(n->simt_img);
  n->simt_img = nullptr;
  if (n->packed) cudaFree(n->packed);
  n->packed = nullptr;
  n->packed_bytes = 0;
}

// Launch the tensor-core network. pix/trph/count != null selects compose
// mode (out = image). `spill` (120 x n floats) is required when rows may have
// distinct albedo channels; the kernel reports a missing one through the
// error word. The error word lives after the packed image.
int launch_mlp_tc(const Network* net, const float* desc, const float* aux, long long rs, long long cs,
                  long long ars, long long afs, int n, float* out, const int* pix, const float* trph,
                  const unsigned* count, F3 light_color, F3 scatter, float* spill, bool f8, cudaStream_t s,
                  const int* job, const BatchOut* bout) {
  if (cs * 4 > 0x7FFFFFFFll || n > (1 << 28))
    return set_error(MR_ERR_ARG, "tensor-core network: %d rows / chunk stride %lld out of range", n, cs);
  static DeviceCache attr;  // the attributes belong to each device's context
  int rc = attr.once([] {
    MR_CUDA(cudaFuncSetAttribute(k_mlp_tc<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_bytes<false>()));
    MR_CUDA(cudaFuncSetAttribute(k_mlp_tc<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_bytes<true>()));
    return (int)MR_OK;
  });
  if (rc) return rc;
  TcArgs a;
  a.wpack = (const uint8_t*)net->packed;
  a.w = net->w;
  a.desc = desc;
  a.aux = aux;
  a.rs = rs;
  a.cs = cs;
  a.ars = ars;
  a.afs = afs;
  a.n = n;
  a.out = out;
  a.pix = pix;
  a.trph = trph;
  a.count = count;
  a.light_color = light_color;
  a.scatter = scatter;
  a.spill = spill;
  a.spill_cap = n;
  a.job = job;
  a.bout = bout;
  if (net->h_rowwise.size() != (size_t)kRowFloats) return set_error(MR_ERR_STATE, "network not packed");
  std::memcpy(a.rw, net->h_rowwise.data(), sizeof(a.rw));
  if (net->h_se.size() * sizeof(float) != sizeof(a.se)) return set_error(MR_ERR_STATE, "network not packed");
  std::memcpy(a.se, net->h_se.data(), sizeof(a.se));
  a.wpack8 = (const uint8_t*)net->packed + kWBytes + 256;
  for (int i = 0; i < kTcLayers; ++i) a.winv[i] = f8 ? net->h_winv8[i] : 1.0f;
  a.err = (int*)((uint8_t*)net->packed + kWBytes);
  int tiles = (n + 127) / 128;
  int grid = std::min(sm_count(), std::max(1, (tiles + kGroups - 1) / kGroups));
  if (f8) k_mlp_tc<true><<<grid, 128 * kGroups, smem_bytes<true>(), s>>>(a);
  else k_mlp_tc<false><<<grid, 128 * kGroups, smem_bytes<false>(), s>>>(a);
  MR_CUDA(cudaGetLastError());
  return MR_OK;
}

// The network's error word (set by a kernel whose bounded wait gave up).
int* mlp_error_word(const Network* net) { return (int*)((uint8_t*)net->packed + kWBytes); }

int mlp_tc_error(const Network* net, bool reset) {
  int e = 0;
  int* p = (int*)((uint8_t*)net->packed + kWBytes);
  MR_CUDA(cudaMemcpy(&e, p, sizeof(int), cudaMemcpyDeviceToHost));
  if (reset) MR_CUDA(cudaMemset(p, 0, sizeof(int)));
  return e ? set_error(MR_ERR_TIMEOUT, "tensor-core network: an mbarrier wait timed out") : MR_OK;
}

}  // namespace mr

using namespace mr;

extern "C" int mr_tc_selftest(int32_t n, int32_t k, const uint16_t* host_a, const uint16_t* host_b, float* host_d) {
  clear_error();
  if (!host_a || !host_b || !host_d) return set_error(MR_ERR_ARG, "mr_tc_selftest: NULL argument");
  uint16_t *a = nullptr, *b = nullptr;
  float* d = nullptr;
  int* err = nullptr;
  MR_CUDA(cudaMalloc(&a, 128 * k * 2));
  MR_CUDA(cudaMalloc(&b, n * k * 2));
  MR_CUDA(cudaMalloc(&d, 128 * n * 4));
  MR_CUDA(cudaMalloc(&err, 4));
  MR_CUDA(cudaMemset(err, 0, 4));
  MR_CUDA(cudaMemcpy(a, host_a, 128 * k * 2, cudaMemcpyHostToDevice));
  MR_CUDA(cudaMemcpy(b, host_b, n * k * 2, cudaMemcpyHostToDevice));
  int rc = MR_OK;
  const int sm = 128 * k * 2 + n * k * 2 + 16;
#define MR_SELFTEST(NN, KK)                                                                      \
  if (n == NN && k == KK) {                                                                      \
    cudaFuncSetAttribute(k_tc_selftest<NN, KK>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm); \
    k_tc_selftest<NN, KK><<<1, 128, sm>>>(a, b, d, err);                                          \
  } else
  MR_SELFTEST(16, 16) MR_SELFTEST(32, 32) MR_SELFTEST(16, 32) MR_SELFTEST(32, 64) MR_SELFTEST(64, 128)
  MR_SELFTEST(128, 128) rc = set_error(MR_ERR_ARG, "mr_tc_selftest: shape %dx%d not built", n, k);
#undef MR_SELFTEST
  if (rc == MR_OK) {
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) rc = cuda_error(e, "tc selftest");
  }
  int he = 0;
  if (rc == MR_OK) cudaMemcpy(&he, err, 4, cudaMemcpyDeviceToHost);
  if (rc == MR_OK && he) rc = set_error(MR_ERR_TIMEOUT, "tc selftest: mbarrier wait timed out");
  if (rc == MR_OK) cudaMemcpy(host_d, d, 128 * n * 4, cudaMemcpyDeviceToHost);
  cudaFree(a);
  cudaFree(b);
  cudaFree(d);
  cudaFree(err);
  return rc;
}

extern "C" int mr_tc_wait_selftest(int32_t limit_us, int64_t* host_waited_ns) {
  clear_error();
  if (limit_us <= 0 || limit_us > 1000000) return set_error(MR_ERR_ARG, "mr_tc_wait_selftest: limit %d us", limit_us);
  int* err = nullptr;
  unsigned long long* waited = nullptr;
  MR_CUDA(cudaMalloc(&err, 4));
  MR_CUDA(cudaMalloc(&waited, 8));
  MR_CUDA(cudaMemset(err, 0, 4));
  MR_CUDA(cudaMemset(waited, 0, 8));
  k_tc_wait_selftest<<<1, 128>>>((uint64_t)limit_us * 1000ull, err, waited);
  int rc = MR_OK;
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e != cudaSuccess) rc = cuda_error(e, "wait selftest");
  int he = 0;
  unsigned long long w = 0;
  if (rc == MR_OK) {
    cudaMemcpy(&he, err, 4, cudaMemcpyDeviceToHost);
    cudaMemcpy(&w, waited, 8, cudaMemcpyDeviceToHost);
    if (host_waited_ns) *host_waited_ns = (int64_t)w;
    rc = he ? set_error(MR_ERR_TIMEOUT, "wait selftest: the mbarrier wait gave up after %llu ns", w)
            : set_error(MR_ERR_STATE, "wait selftest: the wait completed although nothing arrived");
  }
  cudaFree(err);
  cudaFree(waited);
  return rc;
}

extern "C" int mr_tc_selftest_tf32(int32_t n, int32_t k, const float* host_a, const float* host_b, float* host_d,
                                   int32_t split) {
  clear_error();
  if (!host_a || !host_b || !host_d) return set_error(MR_ERR_ARG, "mr_tc_selftest_tf32: NULL argument");
  float *a = nullptr, *b = nullptr, *d = nullptr;
  int* err = nullptr;
  MR_CUDA(cudaMalloc(&a, 128 * k * 4));
  MR_CUDA(cudaMalloc(&b, n * k * 4));
  MR_CUDA(cudaMalloc(&d, 128 * n * 4));
  MR_CUDA(cudaMalloc(&err, 4));
  MR_CUDA(cudaMemset(err, 0, 4));
  MR_CUDA(cudaMemcpy(a, host_a, 128 * k * 4, cudaMemcpyHostToDevice));
  MR_CUDA(cudaMemcpy(b, host_b, n * k * 4, cudaMemcpyHostToDevice));
  int rc = MR_OK;
  const int sm = 2 * (128 * k + n * k) * 4 + 16;
#define MR_SELFTEST32(NN, KK)                                                                       \
  if (n == NN && k == KK) {                                                                         \
    cudaFuncSetAttribute(k_tc_selftest32<NN, KK>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm); \
    k_tc_selftest32<NN, KK><<<1, 128, sm>>>(a, b, d, err, split ? 1 : 0);                           \
  } else
  MR_SELFTEST32(16, 16) MR_SELFTEST32(32, 32) MR_SELFTEST32(32, 64) MR_SELFTEST32(64, 128)
  rc = set_error(MR_ERR_ARG, "mr_tc_selftest_tf32: shape %dx%d not built", n, k);
#undef MR_SELFTEST32
  if (rc == MR_OK) {
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) rc = cuda_error(e, "tc selftest tf32");
  }
  int he = 0;
  if (rc == MR_OK) cudaMemcpy(&he, err, 4, cudaMemcpyDeviceToHost);
  if (rc == MR_OK && he) rc = set_error(MR_ERR_TIMEOUT, "tc selftest tf32: mbarrier wait timed out");
  if (rc == MR_OK) cudaMemcpy(host_d, d, 128 * n * 4, cudaMemcpyDeviceToHost);
  cudaFree(a);
  cudaFree(b);
  cudaFree(d);
  cudaFree(err);
  return rc;
}

extern "C" int mr_tc_selftest_fp8(int32_t n, int32_t k, const uint8_t* host_a, const uint8_t* host_b, float* host_d) {
  clear_error();
  if (!host_a || !host_b || !host_d) return set_error(MR_ERR_ARG, "mr_tc_selftest_fp8: NULL argument");
  uint8_t *a = nullptr, *b = nullptr;
  float* d = nullptr;
  int* err = nullptr;
  MR_CUDA(cudaMalloc(&a, 128 * k));
  MR_CUDA(cudaMalloc(&b, n * k));
  MR_CUDA(cudaMalloc(&d, 128 * n * 4));
  MR_CUDA(cudaMalloc(&err, 4));
  MR_CUDA(cudaMemset(err, 0, 4));
  MR_CUDA(cudaMemcpy(a, host_a, 128 * k, cudaMemcpyHostToDevice));
  MR_CUDA(cudaMemcpy(b, host_b, n * k, cudaMemcpyHostToDevice));
  int rc = MR_OK;
  const int sm = 128 * k + n * k + 16;
#define MR_SELFTEST8(NN, KK)                                                                       \
  if (n == NN && k == KK) {                                                                        \
    cudaFuncSetAttribute(k_tc_selftest8<NN, KK>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm); \
    k_tc_selftest8<NN, KK><<<1, 128, sm>>>(a, b, d, err);                                          \
  } else
  MR_SELFTEST8(16, 32) MR_SELFTEST8(32, 32) MR_SELFTEST8(64, 128) MR_SELFTEST8(128, 128)
  rc = set_error(MR_ERR_ARG, "mr_tc_selftest_fp8: shape %dx%d not built", n, k);
#undef MR_SELFTEST8
  if (rc == MR_OK) {
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) rc = cuda_error(e, "tc selftest fp8");
  }
  int he = 0;
  if (rc == MR_OK) cudaMemcpy(&he, err, 4, cudaMemcpyDeviceToHost);
  if (rc == MR_OK && he) rc = set_error(MR_ERR_TIMEOUT, "tc selftest fp8: mbarrier wait timed out");
  if (rc == MR_OK) cudaMemcpy(host_d, d, 128 * n * 4, cudaMemcpyDeviceToHost);
  cudaFree(a);
  cudaFree(b);
  cudaFree(d);
  cudaFree(err);
  return rc;
}

extern "C" int mr_network_check(const mr_network* net, int32_t reset) {
  clear_error();
  if (!net) return set_error(MR_ERR_ARG, "mr_network_check: NULL network");
  return mlp_tc_error(&net->n, reset != 0);
}
