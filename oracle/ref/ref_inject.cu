// Descriptor-injection harness for the reference network - TEST
// INFRASTRUCTURE ONLY.
//
// Linked with the reference's core/radiancePredict.cu (via ref_net_tu.cu) and
// core/vector.cu, but NOT with core/renderResources.cu: the three volume
// readers that RadiancePredict calls (MipDensityDynamic, ShadowTerm_TRTex and
// the _HGLut fetch, core/radiancePredict.cu:335-358) are defined here and
// return values taken from a caller-given descriptor, so the reference's own
// network code runs on exactly the inputs this project's network gets.
//   X_Val[i]     = log(1 + alpha*rho_i/64)  -> rho_i = raw[0][i] with alpha = 64
//   X_Val_Sub[i] = raw[1][i]
//   X_Val_Hg[i]  = log(HG0*HG1 + 1)          -> HG0 = raw[2][i], HG1 = 1   (i >= 1)
// X_Val_Hg[0] is computed by the reference from the frames (HG(X.L, g)).
#include "radiancePredict.cuh"

__device__ const float* g_raw;  // n x 576 raw reader values
__device__ int* g_calls;        // 3 counters per thread
__device__ int g_n;

__device__ __forceinline__ int inj_tid() { return blockIdx.x * blockDim.x + threadIdx.x; }
__device__ __forceinline__ int inj_rec() { int t = inj_tid(); return t < g_n ? t : g_n - 1; }

__device__ float MipDensityDynamic(int mip, float3 pos) {
  int t = inj_tid();
  int i = g_calls[3 * t + 0]++;
  return g_raw[576 * inj_rec() + i];
}
__device__ float MipTrDynamic(int mip, float3 pos) { return 0.0f; }
__device__ float MipVarianceDynamic(int mip, float3 pos) { return 0.0f; }
__device__ float3 ShadowTerm_TRTex(float3 ori, float3 lightDir, float3 dir, float3 lightColor, float g, int mip) {
  int t = inj_tid();
  int i = g_calls[3 * t + 1]++;
  return float3{g_raw[576 * inj_rec() + 192 + i], 0.0f, 0.0f};
}
// The HG table reads come in pairs (HG0, HG1) for stencil indices 1..191.
__device__ float inj_hglut(float u, float v) {
  int t = inj_tid();
  int c = g_calls[3 * t + 2]++;
  if (c & 1) return 1.0f;
  return g_raw[576 * inj_rec() + 384 + 1 + (c >> 1)];
}

// Texture-reference globals declared by core/renderResources.cuh.
texture<float, cudaTextureType2D, cudaReadModeElementType> _HGLut;
texture<float, cudaTextureType3D, cudaReadModeElementType> _DensityVolume;
texture<float4, cudaTextureType2D> _HDRI;

__global__ void k_inject(int n, const float* frame, float3 L, float g, float3 scatterrate, float* out) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  int kk = k < n ? k : n - 1;
  const float* f = frame + 12 * kk;
  curandState st;
  float3 r = RadiancePredict(&st, true, float3{0, 0, 0}, L, float3{f[0], f[1], f[2]}, float3{f[3], f[4], f[5]},
                             float3{f[6], f[7], f[8]}, float3{f[9], f[10], f[11]}, float3{0, 0, 0},
                             float3{0, 0, 0}, 64.0f, g, scatterrate);
  if (k < n) { out[3 * k] = r.x; out[3 * k + 1] = r.y; out[3 * k + 2] = r.z; }
}

extern "C" int ref_inject_predict(int n, const float* raw, const float* frame, const float* light, float g,
                                  const float* scatterrate, float* out) {
  float *d_raw, *d_fr, *d_out;
  int* d_calls;
  int nt = (n + 31) / 32 * 32;
  if (cudaMalloc(&d_raw, 576 * (size_t)n * sizeof(float)) != cudaSuccess) return 1;
  if (cudaMalloc(&d_fr, 12 * (size_t)n * sizeof(float)) != cudaSuccess) return 1;
  if (cudaMalloc(&d_out, 3 * (size_t)n * sizeof(float)) != cudaSuccess) return 1;
  if (cudaMalloc(&d_calls, 3 * (size_t)nt * sizeof(int)) != cudaSuccess) return 1;
  cudaMemcpy(d_raw, raw, 576 * (size_t)n * sizeof(float), cudaMemcpyHostToDevice);
  cudaMemcpy(d_fr, frame, 12 * (size_t)n * sizeof(float), cudaMemcpyHostToDevice);
  cudaMemset(d_calls, 0, 3 * (size_t)nt * sizeof(int));
  cudaMemcpyToSymbol(g_raw, &d_raw, sizeof(d_raw));
  cudaMemcpyToSymbol(g_calls, &d_calls, sizeof(d_calls));
  cudaMemcpyToSymbol(g_n, &n, sizeof(int));
  k_inject<<<nt / 32, 32>>>(n, d_fr, float3{light[0], light[1], light[2]}, g,
                            float3{scatterrate[0], scatterrate[1], scatterrate[2]}, d_out);
  int rc = cudaDeviceSynchronize() == cudaSuccess ? 0 : 2;
  cudaMemcpy(out, d_out, 3 * (size_t)n * sizeof(float), cudaMemcpyDeviceToHost);
  cudaFree(d_raw);
  cudaFree(d_fr);
  cudaFree(d_out);
  cudaFree(d_calls);
  return rc;
}
