// Seeded procedural cloud densities (the synthetic inputs of the benchmark
// and the training generator): Perlin gradient noise ("improved noise",
// Perlin 2002: quintic fade, 12 edge gradients, permutation table from a
// seeded Fisher-Yates shuffle), summed as fractional Brownian motion,
// normalised to [0, 1], thresholded and shaped by a radial falloff:
//   n(p)  = 0.5 + 0.5 * sum_o gain^o noise(p * f0 * lac^o) / sum_o gain^o
//   d(p)  = max(0, n - thr) / (1 - thr) * max(0, 1 - (2|p - 0.5|)^2)
// evaluated at texel centres p = (i + 0.5) / res, index (x*res+y)*res+z.
#include "mr_internal.h"

namespace mr {

__device__ __forceinline__ float fade(float t) { return t * t * t * (t * (t * 6.0f - 15.0f) + 10.0f); }
__device__ __forceinline__ float grad(int h, float x, float y, float z) {
  h &= 15;
  float u = h < 8 ? x : y;
  float v = h < 4 ? y : (h == 12 || h == 14 ? x : z);
  return ((h & 1) ? -u : u) + ((h & 2) ? -v : v);
}
__device__ float perlin(const int* __restrict__ P, float x, float y, float z) {
  float fx = floorf(x), fy = floorf(y), fz = floorf(z);
  int X = (int)fx & 255, Y = (int)fy & 255, Z = (int)fz & 255;
  x -= fx; y -= fy; z -= fz;
  float u = fade(x), v = fade(y), w = fade(z);
  int A = P[X] + Y, AA = P[A] + Z, AB = P[A + 1] + Z;
  int B = P[X + 1] + Y, BA = P[B] + Z, BB = P[B + 1] + Z;
  return lerpf(lerpf(lerpf(grad(P[AA], x, y, z), grad(P[BA], x - 1, y, z), u),
                     lerpf(grad(P[AB], x, y - 1, z), grad(P[BB], x - 1, y - 1, z), u), v),
               lerpf(lerpf(grad(P[AA + 1], x, y, z - 1), grad(P[BA + 1], x - 1, y, z - 1), u),
                     lerpf(grad(P[AB + 1], x, y - 1, z - 1), grad(P[BB + 1], x - 1, y - 1, z - 1), u), v),
               w);
}

struct CloudArgs {
  int res, octaves;
  float f0, lac, gain, thr;
};

__global__ void k_cloud(const int* __restrict__ perm, CloudArgs a, float* __restrict__ out) {
  __shared__ int P[512];
  for (int i = threadIdx.x; i < 512; i += blockDim.x) P[i] = perm[i & 255];
  __syncthreads();
  size_t n = (size_t)a.res * a.res * a.res;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    int z = (int)(i % a.res), y = (int)((i / a.res) % a.res), x = (int)(i / ((size_t)a.res * a.res));
    float px = ((float)x + 0.5f) / a.res, py = ((float)y + 0.5f) / a.res, pz = ((float)z + 0.5f) / a.res;
    float sum = 0.0f, norm = 0.0f, amp = 1.0f, f = a.f0;
    for (int o = 0; o < a.octaves; ++o) {
      sum += amp * perlin(P, px * f, py * f, pz * f);
      norm += amp;
      amp *= a.gain;
      f *= a.lac;
    }
    float nv = 0.5f + 0.5f * sum / norm;
    float dx = px - 0.5f, dy = py - 0.5f, dz = pz - 0.5f;
    float r2 = 4.0f * (dx * dx + dy * dy + dz * dz);
    float fall = fmaxf(0.0f, 1.0f - r2);
    out[i] = fmaxf(0.0f, nv - a.thr) / (1.0f - a.thr) * fall;
  }
}

// Permutation of 0..255 by Fisher-Yates with Philox(seed; i, 0, 0, TAG_MISC+1).
void cloud_permutation(uint32_t seed, int* perm) {
  for (int i = 0; i < 256; ++i) perm[i] = i;
  for (int i = 255; i > 0; --i) {
    uint32_t o[4];
    philox4x32_10((uint32_t)i, 0u, 0u, TAG_MISC + 1, seed, 0u, o);
    int j = (int)(o[0] % (uint32_t)(i + 1));
    int t = perm[i]; perm[i] = perm[j]; perm[j] = t;
  }
}

}  // namespace mr

using namespace mr;

extern "C" int mr_generate_cloud(int32_t res, uint32_t seed, int32_t octaves, float base_freq, float lacunarity,
                                 float gain, float threshold, float* dev_out, void* stream) {
  clear_error();
  if (!dev_out || res < 1 || res > 2048 || octaves < 1 || octaves > 16 || !(threshold < 1.0f))
    return set_error(MR_ERR_ARG, "mr_generate_cloud: invalid argument");
  int perm[256];
  cloud_permutation(seed, perm);
  int* d_perm = nullptr;
  cudaStream_t s = (cudaStream_t)stream;
  MR_CUDA(cudaMallocAsync(&d_perm, sizeof(perm), s));
  MR_CUDA(cudaMemcpyAsync(d_perm, perm, sizeof(perm), cudaMemcpyHostToDevice, s));
  CloudArgs a{res, octaves, base_freq, lacunarity, gain, threshold};
  k_cloud<<<sm_count() * 8, 256, 0, s>>>(d_perm, a, dev_out);
  MR_CUDA(cudaGetLastError());
  MR_CUDA(cudaFreeAsync(d_perm, s));
  return MR_OK;
}

extern "C" int mr_cloud_permutation(uint32_t seed, int32_t* host_out256) {
  clear_error();
  if (!host_out256) return set_error(MR_ERR_ARG, "mr_cloud_permutation: NULL");
  cloud_permutation(seed, host_out256);
  return MR_OK;
}
