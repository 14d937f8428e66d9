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

struct TcTables { int woff[kTcLayers]; int boff[kTcLayers]; };
constexpr TcTables make_tc_tables() {
  TcTables t{};
  WeightTable wt = make_weight_table();
  for (int i = 0; i < kTcLayers; ++i) { t.woff[i] = tc_offset(i); t.boff[i] = wt.off[kTc[i].b]; }
  return t;
}
__constant__ TcTables c_tc = make_tc_tables();
__device__ __forceinline__ int tc_offset_dev(int i) { return c_tc.woff[i]; }
__device__ __forceinline__ int kTcBias(int i) { return c_tc.boff[i]; }

constexpr int kGroups = 3;
constexpr int kTrunkBytes = 3 * 128 * 32 * 2;  // 24 KB
constexpr int kHeadBytes = 128 * 128 * 2;      // 32 KB
// The trunk tiles and the head tile of a group share one region: every
// layer's MMA has completed (mbarrier) before its epilogue overwrites it.
constexpr int kGroupBytes = kHeadBytes;
static_assert(kTrunkBytes <= kHeadBytes, "trunk tiles alias the head tile");
constexpr int kSmemBytes = kWBytes + kGroups * kGroupBytes + 64 * kGroups + 16;
constexpr int kTmemCols = 512;  // 128 per group (power of two allocation)
static_assert(128 * kGroups <= kTmemCols, "tensor memory budget");
static_assert(kSmemBytes <= 232448, "shared memory budget");

// Byte offset of element (row, k) of a K-major tile with KP columns.
__host__ __device__ constexpr int canon_off(int row, int k, int kp) {
  return ((row >> 3) * (kp >> 3) + (k >> 3)) * 128 + (row & 7) * 16 + (k & 7) * 2;
}

// ---- PTX wrappers ----------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor: K-major, no swizzle, Blackwell version 1.
__device__ __forceinline__ uint64_t sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = (uint64_t)((addr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}
// Instruction descriptor: BF16 x BF16 -> FP32, A and B K-major, M x N.
__host__ __device__ constexpr uint32_t idesc_bf16(int m, int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}
__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"(acc)
      : "memory");
}
__device__ __forceinline__ void umma_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar) : "memory");
}
__device__ __forceinline__ void mbar_init(uint32_t mbar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(count) : "memory");
}
__device__ __forceinline__ uint64_t globaltimer() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
// Bounded wait for the mbarrier phase with the given parity (2 s limit).
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity) {
  uint64_t t0 = 0;
  for (uint32_t it = 0;; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}\n"
        : "=r"(done)
        : "r"(mbar), "r"(parity)
        : "memory");
    if (done) return true;
    if (it == 0) t0 = globaltimer();
    else if ((it & 63) == 0 && globaltimer() - t0 > 2000000000ull) return false;
  }
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void group_bar(int g) { asm volatile("bar.sync %0, 128;" ::"r"(g + 1) : "memory"); }

// 16 consecutive fp32 columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

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

__device__ __forceinline__ float sigm(float x) { return 1.0f / (1.0f + expf(-x)); }

struct TcArgs {
  const uint8_t* __restrict__ wpack;  // kWBytes packed bf16 image
  const float* __restrict__ w;        // fp32 blob (biases, SE and small layers)
  const float* __restrict__ desc;     // row k feature i at desc[k*rs + i*fs]
  long long rs, fs, ars, afs;         // descriptor / aux strides
  const float* __restrict__ aux;      // n x 5
  int n;
  float* out;                         // n x 3, or image when pix != null
  const int* __restrict__ pix;        // compose mode: pixel index per record
  const float* __restrict__ trph;     // compose mode: single-scatter term
  const unsigned* __restrict__ count; // compose mode: number of records (device)
  F3 light_color, scatter;
  int* err;                           // set on a wait timeout
};

// One descriptor row: feature i at p[i*fs] (fs = 1 row-major, fs = capacity
// feature-major).
struct DIn {
  const float* __restrict__ p;
  long long fs;
  __device__ __forceinline__ float operator[](int i) const { return __ldg(p + i * fs); }
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
__device__ __forceinline__ void epi_relu(const GroupCtx& c, int col, const float* __restrict__ bias, float* y) {
  float v[16];
#pragma unroll
  for (int h = 0; h < (N + 15) / 16; ++h) {
    tmem_ld16(c.tmem + c.tlane + col + 16 * h, v);
#pragma unroll
    for (int i = 0; i < 16; ++i)
      if (16 * h + i < N) {
        float a = __ldg(bias + 16 * h + i) + v[i];
        y[16 * h + i] = a >= 0.0f ? a : 0.0f;
      }
  }
}

// SE / SERES block of the trunks (radiancePredict.cu:240-294) for branch
// width S on the descriptor row d, pooling into the SEFin1 accumulators.
// MODE: 0 = SE, then ADD3; 1 = SERES, then ADD3; 2 = SERES, then REP3.
template <int S, int MODE>
__device__ __noinline__ void trunk_block(GroupCtx& c, const DIn& d, const float* __restrict__ w,
                                            int from, int pid, int sew0, int sew1, int layer0, float g, float gamma,
                                            float (&y)[3][32], float* fin) {
  constexpr int KP = S < 16 ? 16 : S;
  // pooled statistics of the three descriptor segments
  float mean[3], mx[3];
#pragma unroll
  for (int br = 0; br < 3; ++br) {
    float s = 0.0f, m = -10000.0f;
#pragma unroll
    for (int i = 0; i < S; ++i) {
      float v = d[br * 192 + from + i];
      s += v;
      m = fmaxf(m, v);
    }
    mean[br] = s / (float)S;
    mx[br] = m;
  }
  // LSEFin1 (16 x 75) contributions of pool[pid+br] and pool[36+pid+br]
  const float* f1 = w + WOFF(LSEFin1W);
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    float a = fin[j];
#pragma unroll
    for (int br = 0; br < 3; ++br) {
      a += mean[br] * __ldg(f1 + j * 75 + pid + br);
      a += mx[br] * __ldg(f1 + j * 75 + 36 + pid + br);
    }
    fin[j] = a;
  }
  // squeeze-excitation gates
  float tmp[8] = {mean[0], mean[1], mean[2], mx[0], mx[1], mx[2], g, gamma};
  float h[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    float a = 0.0f;
#pragma unroll
    for (int j = 0; j < 8; ++j) a += tmp[j] * __ldg(w + sew0 + j + i * 8);
    h[i] = a >= 0.0f ? a : 0.0f;
  }
  float gate[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    float a = 0.0f;
#pragma unroll
    for (int j = 0; j < 8; ++j) a += h[j] * __ldg(w + sew1 + j + i * 8);
    gate[i] = sigm(a);
  }
  // layer inputs x = seg * gate (+ previous output)
#pragma unroll
  for (int br = 0; br < 3; ++br) {
    float x[KP];
#pragma unroll
    for (int i = 0; i < KP; ++i) {
      float v = 0.0f;
      if (i < S) {
        v = d[br * 192 + from + i] * gate[br];
        if (MODE != 0) v = v + y[br][i];
      }
      x[i] = v;
    }
    store_row<KP>(c.trunk + br * (128 * 32 * 2), c.t, x);
  }
  const uint32_t tb = smem_u32(c.trunk), wb = smem_u32(c.wsm);
  mma_round(c, [&]() {
#pragma unroll
    for (int br = 0; br < 3; ++br)
      issue_layer<KP, KP>(c.tmem + 32 * br, tb + br * (128 * 32 * 2), wb + tc_offset_dev(layer0 + br));
  });
  // epilogue: ReLU(W x + b), then ADD3 / REP3
#pragma unroll
  for (int br = 0; br < 3; ++br) {
    float yn[32];
    epi_relu<S>(c, 32 * br, w + kTcBias(layer0 + br), yn);
#pragma unroll
    for (int i = 0; i < S; ++i) {
      float s = d[br * 192 + from + i];
      if (MODE == 2) {
        y[br][i] = yn[i];
        y[br][S + i] = s;
      } else {
        y[br][i] = yn[i] + s;
      }
    }
  }
}

// Head SC(p) (radiancePredict.cu:439-473) for one albedo channel; the
// gated 128-wide input is already in c.head (bf16). Returns the output X.
__device__ __noinline__ float head_chain(GroupCtx& c, const float* __restrict__ w) {
  const uint32_t hb = smem_u32(c.head), tb = smem_u32(c.trunk), wb = smem_u32(c.wsm);
  float v[32];
  // LC0 128 -> 128, read back and re-stored 32 columns at a time
  mma_round(c, [&]() { issue_layer<128, 128>(c.tmem, hb, wb + tc_offset(TC_LC0)); });
#pragma unroll 1
  for (int h = 0; h < 4; ++h) {
    epi_relu<32>(c, 32 * h, w + WOFF(LC0B) + 32 * h, v);
    store_cols<128, 32>(c.head, c.t, 32 * h, v);
  }
  // LC1 128 -> 64
  mma_round(c, [&]() { issue_layer<64, 128>(c.tmem, hb, wb + tc_offset(TC_LC1)); });
#pragma unroll 1
  for (int h = 0; h < 2; ++h) {
    epi_relu<32>(c, 32 * h, w + WOFF(LC1B) + 32 * h, v);
    store_cols<64, 32>(c.trunk, c.t, 32 * h, v);
  }
  // LC2 64 -> 32
  mma_round(c, [&]() { issue_layer<32, 64>(c.tmem, tb, wb + tc_offset(TC_LC2)); });
  epi_relu<32>(c, 0, w + WOFF(LC2B), v);
  store_row<32>(c.trunk, c.t, v);
  // LX 32 -> 16
  mma_round(c, [&]() { issue_layer<16, 32>(c.tmem, tb, wb + tc_offset(TC_LX)); });
  float a[16], b[16];
  epi_relu<16>(c, 0, w + WOFF(LXB), a);
  // six residual pairs (:454-471)
#pragma unroll 1
  for (int r = 0; r < 6; ++r) {
    store_row<16>(c.trunk, c.t, a);
    int l0 = TC_LXR + 2 * r, l1 = l0 + 1;
    mma_round(c, [&]() { issue_layer<16, 16>(c.tmem, tb, wb + tc_offset_dev(l0)); });
    epi_relu<16>(c, 0, w + kTcBias(l0), b);
    store_row<16>(c.trunk, c.t, b);
    mma_round(c, [&]() { issue_layer<16, 16>(c.tmem, tb, wb + tc_offset_dev(l1)); });
    epi_relu<16>(c, 0, w + kTcBias(l1), b);
#pragma unroll
    for (int i = 0; i < 16; ++i) a[i] = a[i] + b[i];
  }
  // LX12 16 -> 1, bias after the sum (LinearReLU, :41-56)
  float o = 0.0f;
#pragma unroll
  for (int i = 0; i < 16; ++i) o += a[i] * __ldg(w + WOFF(LX12W) + i);
  o += __ldg(w + WOFF(LX12B));
  return o >= 0.0f ? o : 0.0f;
}

// Builds the gated head input for albedo channel value srp into c.head.
__device__ __noinline__ void head_input(GroupCtx& c, const float* __restrict__ w, const float* comb_raw,
                                           const float* fin, float g, float gamma, float srp) {
  // pool[72..74] = g, gamma, srp: LGGS (3 -> 8, bias last) and LSEFin1's last columns
  float x8[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    float a = g * __ldg(w + WOFF(LGGSW) + 3 * i) + gamma * __ldg(w + WOFF(LGGSW) + 3 * i + 1) +
              srp * __ldg(w + WOFF(LGGSW) + 3 * i + 2);
    a += __ldg(w + WOFF(LGGSB) + i);
    x8[i] = a >= 0.0f ? a : 0.0f;
  }
  store_cols<128, 8>(c.head, c.t, 120, x8);
  float sew[16];
  const float* f1 = w + WOFF(LSEFin1W);
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    float a = fin[j] + g * __ldg(f1 + j * 75 + 72) + gamma * __ldg(f1 + j * 75 + 73) + srp * __ldg(f1 + j * 75 + 74);
    sew[j] = a >= 0.0f ? a : 0.0f;
  }
  float sep[6];
#pragma unroll
  for (int i = 0; i < 6; ++i) {
    float a = 0.0f;
#pragma unroll
    for (int j = 0; j < 16; ++j) a += sew[j] * __ldg(w + WOFF(LSEFin2W) + j + i * 16);
    sep[i] = sigm(a);
  }
  // gated comb, 8 columns at a time: segments [0,32) [32,64) [64,96) use
  // gates 0..2, [96,104) [104,112) [112,120) gates 3..5
#pragma unroll 1
  for (int g8 = 0; g8 < 15; ++g8) {
    const float s = sep[g8 < 12 ? g8 / 4 : g8 - 9];
#pragma unroll
    for (int i = 0; i < 8; ++i) x8[i] = comb_raw[8 * g8 + i] * s;
    store_cols<128, 8>(c.head, c.t, 8 * g8, x8);
  }
}

// Light-direction trunk block (width 8).
template <int MODE>
__device__ __forceinline__ void di_block(GroupCtx& c, const DIn& d, const float* __restrict__ w,
                                         int blk, float g, float gamma, float (&y)[3][32], float* fin) {
  const int sew0[4] = {WOFF(LDSE01W), WOFF(LDSE11W), WOFF(LDSE21W), WOFF(LDSE31W)};
  const int sew1[4] = {WOFF(LDSE02W), WOFF(LDSE12W), WOFF(LDSE22W), WOFF(LDSE32W)};
  trunk_block<8, MODE>(c, d, w, 160 + 8 * blk, 24 + 3 * blk, sew0[blk], sew1[blk], TC_DI + 3 * blk, g, gamma, y, fin);
}

__global__ void __launch_bounds__(128 * kGroups, 1) k_mlp_tc(TcArgs a) {
  extern __shared__ __align__(1024) uint8_t smem[];
  uint8_t* wsm = smem;
  uint8_t* gbase = smem + kWBytes;
  uint64_t* mbars = reinterpret_cast<uint64_t*>(smem + kWBytes + kGroups * kGroupBytes);
  uint32_t* tmem_holder = reinterpret_cast<uint32_t*>(mbars + kGroups);
  volatile unsigned* need_slot = tmem_holder + 1;  // kGroups slots
  const int tid = threadIdx.x, warp = tid >> 5;
  const int g = tid >> 7, t = tid & 127;
  // weights -> shared memory (16-byte vectors)
  for (int i = tid; i < kWBytes / 16; i += blockDim.x)
    reinterpret_cast<uint4*>(wsm)[i] = __ldg(reinterpret_cast<const uint4*>(a.wpack) + i);
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
  const float* __restrict__ w = a.w;
  const int n = a.pix ? (int)min(*a.count, (unsigned)a.n) : a.n;

  for (int it = 0;; ++it) {
    // static tile striding over (CTA, group)
    const int tile = (it * (int)gridDim.x + (int)blockIdx.x) * kGroups + g;
    if (tile * 128 >= n) break;  // group-uniform exit
    const int row = tile * 128 + t;
    const int kk = row < n ? row : n - 1;
    const DIn d{a.desc + (long long)kk * a.rs, a.fs};
    const float* ax = a.aux + (long long)kk * a.ars;
    const float gg = __ldg(ax), gamma = __ldg(ax + a.afs);
    float srp[3] = {__ldg(ax + 2 * a.afs), __ldg(ax + 3 * a.afs), __ldg(ax + 4 * a.afs)};
    float fin[16];
#pragma unroll
    for (int j = 0; j < 16; ++j) fin[j] = 0.0f;
    float y[3][32];
    // comb (the head input before gating) lives in local memory through an
    // opaque offset; it is written in chunks and read once per head.
    float comb_store[120];
    int zero = 0;
    asm volatile("" : "+r"(zero));
    float* comb = comb_store + zero;
    // main trunk (radiancePredict.cu:396-421)
    trunk_block<8, 0>(c, d, w, 0, 0, WOFF(LSE01W), WOFF(LSE02W), TC_MAIN + 0, gg, gamma, y, fin);
    trunk_block<8, 2>(c, d, w, 8, 3, WOFF(LSE11W), WOFF(LSE12W), TC_MAIN + 3, gg, gamma, y, fin);
    trunk_block<16, 1>(c, d, w, 16, 6, WOFF(LSE21W), WOFF(LSE22W), TC_MAIN + 6, gg, gamma, y, fin);
    trunk_block<16, 1>(c, d, w, 32, 9, WOFF(LSE31W), WOFF(LSE32W), TC_MAIN + 9, gg, gamma, y, fin);
    trunk_block<16, 2>(c, d, w, 48, 12, WOFF(LSE41W), WOFF(LSE42W), TC_MAIN + 12, gg, gamma, y, fin);
    trunk_block<32, 1>(c, d, w, 64, 15, WOFF(LSE51W), WOFF(LSE52W), TC_MAIN + 15, gg, gamma, y, fin);
    trunk_block<32, 1>(c, d, w, 96, 18, WOFF(LSE61W), WOFF(LSE62W), TC_MAIN + 18, gg, gamma, y, fin);
    trunk_block<32, 1>(c, d, w, 128, 21, WOFF(LSE71W), WOFF(LSE72W), TC_MAIN + 21, gg, gamma, y, fin);
    {  // L81 per branch -> comb[0..96)
#pragma unroll
      for (int br = 0; br < 3; ++br) store_row<32>(c.trunk + br * (128 * 32 * 2), c.t, y[br]);
      const uint32_t tb = smem_u32(c.trunk), wb = smem_u32(c.wsm);
      mma_round(c, [&]() {
#pragma unroll
        for (int br = 0; br < 3; ++br)
          issue_layer<32, 32>(c.tmem + 32 * br, tb + br * (128 * 32 * 2), wb + tc_offset(TC_L81) + 2048 * br);
      });
#pragma unroll
      for (int br = 0; br < 3; ++br) epi_relu<32>(c, 32 * br, w + kTcBias(TC_L81 + br), comb + 32 * br);
    }
    // light-direction trunk (:424-437)
    di_block<0>(c, d, w, 0, gg, gamma, y, fin);
    di_block<1>(c, d, w, 1, gg, gamma, y, fin);
    di_block<1>(c, d, w, 2, gg, gamma, y, fin);
    di_block<1>(c, d, w, 3, gg, gamma, y, fin);
    {  // LD41 per branch -> comb[96..120)
#pragma unroll
      for (int br = 0; br < 3; ++br) {
        float x[16];
#pragma unroll
        for (int i = 0; i < 16; ++i) x[i] = i < 8 ? y[br][i] : 0.0f;
        store_row<16>(c.trunk + br * (128 * 32 * 2), c.t, x);
      }
      const uint32_t tb = smem_u32(c.trunk), wb = smem_u32(c.wsm);
      mma_round(c, [&]() {
#pragma unroll
        for (int br = 0; br < 3; ++br)
          issue_layer<16, 16>(c.tmem + 32 * br, tb + br * (128 * 32 * 2), wb + tc_offset(TC_LD41) + 512 * br);
      });
#pragma unroll
      for (int br = 0; br < 3; ++br) epi_relu<8>(c, 32 * br, w + kTcBias(TC_LD41 + br), comb + 96 + 8 * br);
    }
    // heads per distinct albedo channel (group-uniform decision)
    float X[3];
    head_input(c, w, comb, fin, gg, gamma, srp[0]);
    X[0] = head_chain(c, w);
#pragma unroll 1
    for (int ch = 1; ch < 3; ++ch) {
      // The head runs for the whole tile if any row's channel differs from
      // the channels already evaluated (radiancePredict.cu:478-483).
      const bool same = srp[ch] == srp[0] || (ch == 2 && srp[2] == srp[1]);
      if (t == 0) need_slot[g] = 0u;
      group_bar(g);
      if (!same) need_slot[g] = 1u;
      group_bar(g);
      const bool any = need_slot[g] != 0u;
      group_bar(g);
      if (any) {
        head_input(c, w, comb, fin, gg, gamma, srp[ch]);
        X[ch] = head_chain(c, w);
      } else {
        X[ch] = srp[ch] == srp[0] ? X[0] : X[1];
      }
    }
    if (row < n) {
      float o[3];
#pragma unroll
      for (int ch = 0; ch < 3; ++ch) o[ch] = fmaxf(expf(X[ch]) - 1.0f, 0.0f) * srp[ch];
      if (a.pix) {
        const int px = a.pix[row];
        const float tr = a.trph[row];
        const float lc[3] = {a.light_color.x, a.light_color.y, a.light_color.z};
        const float sc[3] = {a.scatter.x, a.scatter.y, a.scatter.z};
#pragma unroll
        for (int ch = 0; ch < 3; ++ch) a.out[3 * (size_t)px + ch] = fmaxf(((o[ch] + tr) * lc[ch]) * sc[ch], 0.0f);
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

// ---- host ----------------------------------------------------------------------
static uint16_t to_bf16_bits(float f) {
  uint32_t u;
  std::memcpy(&u, &f, 4);
  if ((u & 0x7F800000u) == 0x7F800000u) return (uint16_t)(u >> 16);  // inf / nan
  u += 0x7FFFu + ((u >> 16) & 1u);  // round to nearest even
  return (uint16_t)(u >> 16);
}

int pack_network(Network* n) {
  std::vector<float> w(MR_WEIGHT_TOTAL);
  if (cudaMemcpy(w.data(), n->w, MR_WEIGHT_TOTAL * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess)
    return set_error(MR_ERR_CUDA, "pack_network: weight read-back failed");
  std::vector<uint8_t> img(kWBytes, 0);
  const WeightTable wt = make_weight_table();
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
  cudaError_t e = cudaMalloc(&n->packed, kWBytes + 256);
  if (e == cudaSuccess) e = cudaMemcpy(n->packed, img.data(), kWBytes, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset((uint8_t*)n->packed + kWBytes, 0, 256);
  if (e != cudaSuccess) return set_error(MR_ERR_NOMEM, "pack_network: %s", cudaGetErrorString(e));
  n->packed_bytes = kWBytes;
  return MR_OK;
}

void free_packed(Network* n) {
  if (n->packed) cudaFree(n->packed);
  n->packed = nullptr;
  n->packed_bytes = 0;
}

// Launch the tensor-core network. pix/trph/count != null selects compose
// mode (out = image). The error word lives after the packed image.
int launch_mlp_tc(const Network* net, const float* desc, const float* aux, long long rs, long long fs,
                  long long ars, long long afs, int n, float* out, const int* pix, const float* trph,
                  const unsigned* count, F3 light_color, F3 scatter, cudaStream_t s) {
  static bool attr = false;
  if (!attr) {
    MR_CUDA(cudaFuncSetAttribute(k_mlp_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes));
    attr = true;
  }
  TcArgs a;
  a.wpack = (const uint8_t*)net->packed;
  a.w = net->w;
  a.desc = desc;
  a.aux = aux;
  a.rs = rs;
  a.fs = fs;
  a.ars = ars;
  a.afs = afs;
  a.n = n;
  a.out = out;
  a.pix = pix;
  a.trph = trph;
  a.count = count;
  a.light_color = light_color;
  a.scatter = scatter;
  a.err = (int*)((uint8_t*)net->packed + kWBytes);
  int tiles = (n + 127) / 128;
  int grid = std::min(sm_count(), std::max(1, (tiles + kGroups - 1) / kGroups));
  k_mlp_tc<<<grid, 128 * kGroups, kSmemBytes, s>>>(a);
  MR_CUDA(cudaGetLastError());
  return MR_OK;
}

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

extern "C" int mr_network_check(const mr_network* net, int32_t reset) {
  clear_error();
  if (!net) return set_error(MR_ERR_ARG, "mr_network_check: NULL network");
  return mlp_tc_error(&net->n, reset != 0);
}
