// BF16 tensor-core training of the network's head (LC0, LC1, LC2 of
// core/radiancePredict.cu:454-471): the forward products and both backward
// products (dX = dY W, dW = dY^T X) of every head layer as tcgen05 MMAs with
// FP32 accumulation in tensor memory.
//
// The backward products read the forward tiles transposed. A BF16 tile stored
// in the canonical K-major layout of [rows][cols] is, byte for byte, the
// canonical MN-major layout of its transpose: a core matrix is 8 rows of 16
// contiguous bytes either way. dW = dY^T X therefore takes dY's and X's
// forward tiles as MN-major operands (K = the tile's rows), and dX = dY W takes
// the forward weight image W [out][in] as an MN-major B operand (N = in,
// K = out); no transposed copies are made.
#include <cuda_bf16.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "mr_internal.h"
#include "mr_tcgen05.cuh"
#include "mr_train.cuh"

namespace mr {

// Instruction descriptor with the operand majors: a_mn / b_mn = 1 reads A / B
// MN-major (bits 15 / 16 of the kind::f16 instruction descriptor).
__host__ __device__ constexpr uint32_t idesc_bf16_mn(int m, int n, int a_mn, int b_mn) {
  return idesc_bf16(m, n) | ((uint32_t)a_mn << 15) | ((uint32_t)b_mn << 16);
}

// Descriptor of an operand with MNP elements along M (or N) and K elements
// along K, the 16-wide K slice s (MMA step s): K-major tiles are stored as
// canon_off(mn, k, K), MN-major tiles as canon_off(k, mn, MNP). For an
// MN-major operand without swizzle the leading-byte-offset field carries the
// step between groups of 8 K rows ((MNP/8)*128 B) and the stride-byte-offset
// field the step between core matrices along MN (128 B); the opposite
// assignment gives wrong products (mr_tc_selftest_mn).
__device__ __forceinline__ uint64_t operand_desc(uint32_t base, int mn_major, int mnp, int kk, int s) {
  if (!mn_major) return sdesc(base + s * 256, 128, (kk / 8) * 128);
  const uint32_t kstep = (uint32_t)(mnp / 8) * 128;  // 8 K rows
  return sdesc(base + s * 2 * kstep, kstep, 128);
}

// D[128 x N] = A[128 x K] B[N x K]^T with either operand MN-major; inputs
// row-major (A: 128 x K, B: N x K). Each operand has a 64 KB region of shared
// memory, so that a descriptor with its strides swapped would still read
// inside it.
template <int N, int K>
__global__ void __launch_bounds__(128, 1) k_tc_selftest_mn(const uint16_t* __restrict__ A,
                                                           const uint16_t* __restrict__ B, float* __restrict__ D,
                                                           int a_mn, int b_mn, int* err) {
  extern __shared__ __align__(1024) uint8_t dsm[];
  uint8_t* sa = dsm;
  uint8_t* sb = dsm + 65536;
  uint64_t& mbar = *reinterpret_cast<uint64_t*>(dsm + 131072);
  uint32_t& holder = *reinterpret_cast<uint32_t*>(dsm + 131072 + 8);
  const int t = threadIdx.x, warp = t >> 5;
  for (int i = t; i < 65536 * 2 / 16; i += 128) reinterpret_cast<uint4*>(dsm)[i] = make_uint4(0, 0, 0, 0);
  __syncthreads();
  for (int k = 0; k < K; ++k) {
    *reinterpret_cast<uint16_t*>(sa + (a_mn ? canon_off(k, t, 128) : canon_off(t, k, K))) = A[t * K + k];
    if (t < N) *reinterpret_cast<uint16_t*>(sb + (b_mn ? canon_off(k, t, N) : canon_off(t, k, K))) = B[t * K + k];
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
    const uint32_t id = idesc_bf16_mn(128, N, a_mn, b_mn);
#pragma unroll
    for (int s = 0; s < K / 16; ++s)
      umma_bf16(tmem, operand_desc(smem_u32(sa), a_mn, 128, K, s), operand_desc(smem_u32(sb), b_mn, N, K, s), id,
                s > 0 ? 1u : 0u);
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

// Descriptors of the training head's operands: K-major tiles [mn][k] with K
// columns, and MN-major views of K-major tiles [k][mn] with MNP columns.
__device__ __forceinline__ uint64_t kdesc(uint32_t base, int kk, int s) { return operand_desc(base, 0, 0, kk, s); }
__device__ __forceinline__ uint64_t mndesc(uint32_t base, int mnp, int s) { return operand_desc(base, 1, mnp, 0, s); }

// ---- the training head ----------------------------------------------------------
// Shared memory: the BF16 weight image [LC0 128x128 | LC1 64x128 | LC2 32x64]
// (canonical K-major, rows = outputs), the forward tiles kept for the weight
// gradients (head input H0, A1, A2), and one working tile for the backward
// products' A operands (dA3, dA2, dA1 in turn).
constexpr int kImgW0 = 0, kImgW1 = 128 * 128 * 2, kImgW2 = kImgW1 + 64 * 128 * 2;
constexpr int kHeadImgBytes = kImgW2 + 32 * 64 * 2;
constexpr int kOffH0 = kHeadImgBytes, kOffA1 = kOffH0 + 32768, kOffA2 = kOffA1 + 32768, kOffWk = kOffA2 + 16384;
// The working tile's slot is 64 KB: an MN-major read of it with M padded to
// 128 (LC1 and LC2 have 64 and 32 outputs) spans up to 60 KB of descriptor
// extent, all of it inside the slot.
constexpr int kWkSlot = 65536;
constexpr int kHeadTrainSmem = kOffWk + kWkSlot + 16;
static_assert(kHeadImgBytes % 1024 == 0 && kOffWk % 1024 == 0, "tile alignment");
static_assert(kHeadTrainSmem <= 232448, "shared memory budget");
// Tensor memory (512 columns): the working accumulator, then the weight
// gradients of LC0 (128 x 128), LC1 (rows 0..63 of 128 x 128) and LC2 (rows
// 0..31 of 128 x 64), accumulated over all of the CTA's tiles.
constexpr uint32_t kColWork = 0, kColG0 = 128, kColG1 = 256, kColG2 = 384;

// fp32 master weights -> the BF16 image (round to nearest even).
__global__ void k_pack_head(const float* __restrict__ w, uint8_t* __restrict__ img) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  int o, k, K, base, src;
  if (i < 128 * 128) { o = i / 128; k = i % 128; K = 128; base = kImgW0; src = WOFF(LC0W); }
  else if (i < 128 * 128 + 64 * 128) { const int j = i - 128 * 128; o = j / 128; k = j % 128; K = 128; base = kImgW1; src = WOFF(LC1W); }
  else if (i < kHeadImgBytes / 2) { const int j = i - 128 * 128 - 64 * 128; o = j / 64; k = j % 64; K = 64; base = kImgW2; src = WOFF(LC2W); }
  else return;
  const __nv_bfloat16 b = __float2bfloat16_rn(w[src + o * K + k]);
  *reinterpret_cast<__nv_bfloat16*>(img + base + canon_off(o, k, K)) = b;
}

struct HeadTrainArgs {
  const uint8_t* img;   // kHeadImgBytes BF16 image (k_pack_head)
  const float* w;       // fp32 master weights (biases, the tail)
  float* grad;          // fp32 gradient (blob layout)
  const float* h0;      // head input per row, n x 128
  float* dh0;           // its gradient per row, n x 128
  const float* aux;     // n x 5 (g, gamma, srp.xyz)
  const float* label;   // n
  int n;
  float inv_batch;
  float* loss;
  int* err;             // set when a bounded wait gives up
};

// 16 consecutive values of a row -> BF16 at columns c0..c0+15 of a K-major tile.
__device__ __forceinline__ void put16(uint8_t* tile, int row, int c0, int kp, const float* v) {
  uint32_t p[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    __nv_bfloat162 h = __floats2bfloat162_rn(v[2 * i], v[2 * i + 1]);
    p[i] = *reinterpret_cast<uint32_t*>(&h);
  }
  *reinterpret_cast<uint4*>(tile + canon_off(row, c0, kp)) = make_uint4(p[0], p[1], p[2], p[3]);
  *reinterpret_cast<uint4*>(tile + canon_off(row, c0 + 8, kp)) = make_uint4(p[4], p[5], p[6], p[7]);
}

// The head of the training step for tiles of 128 rows, one thread per row
// (TMEM lane): LC0 -> LC1 -> LC2 forward as MMAs, the tail and the loss on
// the CUDA cores (tail_fwd_bwd), then per layer one MMA round with the input
// gradient (dY W, W read MN-major) and the weight gradient (dY^T X, both
// tiles read MN-major) accumulated in tensor memory; the head-input gradient
// goes to dh0 for the trunks' backward.
__global__ void __launch_bounds__(128, 1) k_train_head_tc(const __grid_constant__ HeadTrainArgs a) {
  extern __shared__ __align__(1024) uint8_t sm[];
  uint8_t* img = sm;
  uint8_t* tH0 = sm + kOffH0;
  uint8_t* tA1 = sm + kOffA1;
  uint8_t* tA2 = sm + kOffA2;
  uint8_t* tWk = sm + kOffWk;
  uint64_t* mbar = reinterpret_cast<uint64_t*>(sm + kOffWk + kWkSlot);
  uint32_t* holder = reinterpret_cast<uint32_t*>(sm + kOffWk + kWkSlot + 8);
  const int t = threadIdx.x, warp = t >> 5;
  for (int i = t; i < kHeadImgBytes / 16; i += 128)
    reinterpret_cast<uint4*>(img)[i] = __ldg(reinterpret_cast<const uint4*>(a.img) + i);
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(holder)),
                 "r"(512));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (t == 0) mbar_init(smem_u32(mbar), 1);
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  fence_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tm = *holder, lane = (uint32_t)(32 * warp) << 16;
  const uint32_t sW0 = smem_u32(img + kImgW0), sW1 = smem_u32(img + kImgW1), sW2 = smem_u32(img + kImgW2);
  const uint32_t sH0 = smem_u32(tH0), sA1 = smem_u32(tA1), sA2 = smem_u32(tA2), sWk = smem_u32(tWk);
  const TrainTables& T = c_tt;
  const float* __restrict__ W = a.w;
  float* G = a.grad;
  uint32_t phase = 0;
  bool ok = true, first = true;
  // one MMA round: the tile writes visible to the tensor core, issue, wait
  auto round = [&](auto issue) {
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    if (t == 0) {
      tc_fence_after();
      issue();
      umma_commit(smem_u32(mbar));
    }
    if (ok && !mbar_wait(smem_u32(mbar), phase)) ok = false;
    phase ^= 1u;
    tc_fence_after();
  };
  const int tiles = (a.n + 127) / 128;
  for (int tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
    const int row = tile * 128 + t;
    const bool valid = row < a.n;
    const int k = valid ? row : a.n - 1;
    // H0 -> BF16 tile
    {
      const float4* src = reinterpret_cast<const float4*>(a.h0 + (size_t)k * 128);
#pragma unroll 1
      for (int c = 0; c < 128; c += 16) {
        float v[16];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const float4 x = src[c / 4 + q];
          v[4 * q] = x.x; v[4 * q + 1] = x.y; v[4 * q + 2] = x.z; v[4 * q + 3] = x.w;
        }
        put16(tH0, t, c, 128, v);
      }
    }
    const uint32_t fw = idesc_bf16_mn(128, 128, 0, 0);
    round([&] {
      for (int s = 0; s < 8; ++s) umma_bf16(tm + kColWork, kdesc(sH0, 128, s), kdesc(sW0, 128, s), fw, s > 0);
    });
    // A1 = ReLU(LC0 H0 + b)
    uint32_t m1[4] = {0u, 0u, 0u, 0u};
#pragma unroll 1
    for (int h = 0; h < 8; ++h) {
      float v[16];
      tmem_ld16(tm + lane + kColWork + 16 * h, v);
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        const float x = v[i] + __ldg(W + T.lc0b + 16 * h + i);
        if (x > 0.0f) m1[h / 2] |= 1u << ((16 * h + i) & 31);
        v[i] = x > 0.0f ? x : 0.0f;
      }
      put16(tA1, t, 16 * h, 128, v);
    }
    round([&] {
      const uint32_t id = idesc_bf16_mn(128, 64, 0, 0);
      for (int s = 0; s < 8; ++s) umma_bf16(tm + kColWork, kdesc(sA1, 128, s), kdesc(sW1, 128, s), id, s > 0);
    });
    // A2 = ReLU(LC1 A1 + b)
    uint32_t m2[2] = {0u, 0u};
#pragma unroll 1
    for (int h = 0; h < 4; ++h) {
      float v[16];
      tmem_ld16(tm + lane + kColWork + 16 * h, v);
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        const float x = v[i] + __ldg(W + T.lc1b + 16 * h + i);
        if (x > 0.0f) m2[h / 2] |= 1u << ((16 * h + i) & 31);
        v[i] = x > 0.0f ? x : 0.0f;
      }
      put16(tA2, t, 16 * h, 64, v);
    }
    round([&] {
      const uint32_t id = idesc_bf16_mn(128, 32, 0, 0);
      for (int s = 0; s < 4; ++s) umma_bf16(tm + kColWork, kdesc(sA2, 64, s), kdesc(sW2, 64, s), id, s > 0);
    });
    // A3 = ReLU(LC2 A2 + b), the tail, the loss and the tail's backward
    float A3[32], d3[32];
    uint32_t m3 = 0u;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      float v[16];
      tmem_ld16(tm + lane + kColWork + 16 * h, v);
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        const float x = v[i] + __ldg(W + T.lc2b + 16 * h + i);
        if (x > 0.0f) m3 |= 1u << (16 * h + i);
        A3[16 * h + i] = x > 0.0f ? x : 0.0f;
      }
    }
    const float srp = a.aux[5 * (size_t)k + 2];
    tail_fwd_bwd(W, G, T, A3, a.label[k], srp, valid, a.inv_batch, a.loss, d3);
    // dA3 -> working tile; LC2's input and weight gradients
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      float v[16];
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        v[i] = (m3 >> (16 * h + i)) & 1u ? d3[16 * h + i] : 0.0f;
        gacc(G, T.lc2b + 16 * h + i, v[i]);
      }
      put16(tWk, t, 16 * h, 32, v);
    }
    const uint32_t acc0 = first ? 0u : 1u;
    round([&] {
      const uint32_t dx = idesc_bf16_mn(128, 64, 0, 1), dw = idesc_bf16_mn(128, 64, 1, 1);
      for (int s = 0; s < 2; ++s) umma_bf16(tm + kColWork, kdesc(sWk, 32, s), mndesc(sW2, 64, s), dx, s > 0);
      for (int s = 0; s < 8; ++s) umma_bf16(tm + kColG2, mndesc(sWk, 32, s), mndesc(sA2, 64, s), dw, s > 0 || acc0);
    });
    // dA2 = (dA3 LC2) * [A2 > 0]
#pragma unroll 1
    for (int h = 0; h < 4; ++h) {
      float v[16];
      tmem_ld16(tm + lane + kColWork + 16 * h, v);
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        const int j = 16 * h + i;
        v[i] = (m2[j >> 5] >> (j & 31)) & 1u ? v[i] : 0.0f;
        gacc(G, T.lc1b + j, v[i]);
      }
      put16(tWk, t, 16 * h, 64, v);
    }
    round([&] {
      const uint32_t dx = idesc_bf16_mn(128, 128, 0, 1), dw = idesc_bf16_mn(128, 128, 1, 1);
      for (int s = 0; s < 4; ++s) umma_bf16(tm + kColWork, kdesc(sWk, 64, s), mndesc(sW1, 128, s), dx, s > 0);
      for (int s = 0; s < 8; ++s) umma_bf16(tm + kColG1, mndesc(sWk, 64, s), mndesc(sA1, 128, s), dw, s > 0 || acc0);
    });
    // dA1 = (dA2 LC1) * [A1 > 0]
#pragma unroll 1
    for (int h = 0; h < 8; ++h) {
      float v[16];
      tmem_ld16(tm + lane + kColWork + 16 * h, v);
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        const int j = 16 * h + i;
        v[i] = (m1[j >> 5] >> (j & 31)) & 1u ? v[i] : 0.0f;
        gacc(G, T.lc0b + j, v[i]);
      }
      put16(tWk, t, 16 * h, 128, v);
    }
    round([&] {
      const uint32_t dx = idesc_bf16_mn(128, 128, 0, 1), dw = idesc_bf16_mn(128, 128, 1, 1);
      for (int s = 0; s < 8; ++s) umma_bf16(tm + kColWork, kdesc(sWk, 128, s), mndesc(sW0, 128, s), dx, s > 0);
      for (int s = 0; s < 8; ++s) umma_bf16(tm + kColG0, mndesc(sWk, 128, s), mndesc(sH0, 128, s), dw, s > 0 || acc0);
    });
    // dH0 = dA1 LC0
#pragma unroll 1
    for (int h = 0; h < 8; ++h) {
      float v[16];
      tmem_ld16(tm + lane + kColWork + 16 * h, v);
      if (valid) {
        float4* o = reinterpret_cast<float4*>(a.dh0 + (size_t)row * 128 + 16 * h);
#pragma unroll
        for (int q = 0; q < 4; ++q) o[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
      }
    }
    first = false;
  }
  // the CTA's weight gradients: TMEM lane = output unit
  if (!first && ok) {
#pragma unroll 1
    for (int h = 0; h < 8; ++h) {
      float v[16];
      tmem_ld16(tm + lane + kColG0 + 16 * h, v);
#pragma unroll
      for (int i = 0; i < 16; ++i) atomicAdd(G + T.lc0w + t * 128 + 16 * h + i, v[i]);
    }
    if (warp < 2) {
#pragma unroll 1
      for (int h = 0; h < 8; ++h) {
        float v[16];
        tmem_ld16(tm + lane + kColG1 + 16 * h, v);
#pragma unroll
        for (int i = 0; i < 16; ++i) atomicAdd(G + T.lc1w + t * 128 + 16 * h + i, v[i]);
      }
    }
    if (warp == 0) {
#pragma unroll 1
      for (int h = 0; h < 4; ++h) {
        float v[16];
        tmem_ld16(tm + lane + kColG2 + 16 * h, v);
#pragma unroll
        for (int i = 0; i < 16; ++i) atomicAdd(G + T.lc2w + t * 64 + 16 * h + i, v[i]);
      }
    }
  }
  if (!ok && t == 0) atomicExch(a.err, 1);
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tm), "r"(512));
  }
}

// The BF16 training step's three launches after the weight image: the trunks'
// forward (head input per row), the tensor-core head, the trunks' backward.
int launch_head_tc(const float* w, float* grad, uint8_t* img, const float* h0, float* dh0, const float* aux,
                   const float* label, int n, float inv_batch, float* loss, int* err, cudaStream_t s) {
  static DeviceCache attr;
  int rc = attr.once([] {
    MR_CUDA(cudaFuncSetAttribute(k_train_head_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, kHeadTrainSmem));
    return (int)MR_OK;
  });
  if (rc) return rc;
  k_pack_head<<<(kHeadImgBytes / 2 + 255) / 256, 256, 0, s>>>(w, img);
  MR_CUDA(cudaGetLastError());
  HeadTrainArgs a;
  a.img = img;
  a.w = w;
  a.grad = grad;
  a.h0 = h0;
  a.dh0 = dh0;
  a.aux = aux;
  a.label = label;
  a.n = n;
  a.inv_batch = inv_batch;
  a.loss = loss;
  a.err = err;
  const int tiles = (n + 127) / 128;
  k_train_head_tc<<<std::min(tiles, sm_count()), 128, kHeadTrainSmem, s>>>(a);
  MR_CUDA(cudaGetLastError());
  return MR_OK;
}
size_t head_image_bytes() { return kHeadImgBytes; }

}  // namespace mr

using namespace mr;

extern "C" int mr_tc_selftest_mn(int32_t n, int32_t k, int32_t a_mn, int32_t b_mn, const uint16_t* host_a,
                                 const uint16_t* host_b, float* host_d) {
  clear_error();
  if (!host_a || !host_b || !host_d) return set_error(MR_ERR_ARG, "mr_tc_selftest_mn: NULL argument");
  if ((a_mn | b_mn) & ~1) return set_error(MR_ERR_ARG, "mr_tc_selftest_mn: flags must be 0 or 1");
  const bool built = (n == 64 && k == 32) || (n == 128 && k == 64) || (n == 128 && k == 128) || (n == 64 && k == 128);
  if (!built) return set_error(MR_ERR_ARG, "mr_tc_selftest_mn: shape %dx%d not built", n, k);
  uint16_t *a = nullptr, *b = nullptr;
  float* d = nullptr;
  int* err = nullptr;
  cudaError_t ce = cudaMalloc(&a, 128 * k * 2);
  if (ce == cudaSuccess) ce = cudaMalloc(&b, n * k * 2);
  if (ce == cudaSuccess) ce = cudaMalloc(&d, 128 * n * 4);
  if (ce == cudaSuccess) ce = cudaMalloc(&err, 4);
  if (ce == cudaSuccess) ce = cudaMemset(err, 0, 4);
  if (ce == cudaSuccess) ce = cudaMemcpy(a, host_a, 128 * k * 2, cudaMemcpyHostToDevice);
  if (ce == cudaSuccess) ce = cudaMemcpy(b, host_b, n * k * 2, cudaMemcpyHostToDevice);
  if (ce != cudaSuccess) {
    cudaFree(a);
    cudaFree(b);
    cudaFree(d);
    cudaFree(err);
    return cuda_error(ce, "mr_tc_selftest_mn buffers");
  }
  int rc = MR_OK;
  const int sm = 131072 + 16;
#define MR_SELFTEST(NN, KK)                                                                         \
  if (n == NN && k == KK) {                                                                         \
    cudaFuncSetAttribute(k_tc_selftest_mn<NN, KK>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm); \
    k_tc_selftest_mn<NN, KK><<<1, 128, sm>>>(a, b, d, a_mn, b_mn, err);                              \
  } else
  MR_SELFTEST(64, 32) MR_SELFTEST(128, 64) MR_SELFTEST(128, 128) MR_SELFTEST(64, 128)
  rc = set_error(MR_ERR_ARG, "mr_tc_selftest_mn: shape %dx%d not built", n, k);
#undef MR_SELFTEST
  if (rc == MR_OK) {
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) rc = cuda_error(e, "tc selftest mn");
  }
  int he = 0;
  if (rc == MR_OK) cudaMemcpy(&he, err, 4, cudaMemcpyDeviceToHost);
  if (rc == MR_OK && he) rc = set_error(MR_ERR_TIMEOUT, "tc selftest mn: mbarrier wait timed out");
  if (rc == MR_OK) cudaMemcpy(host_d, d, 128 * n * 4, cudaMemcpyDeviceToHost);
  cudaFree(a);
  cudaFree(b);
  cudaFree(d);
  cudaFree(err);
  return rc;
}
