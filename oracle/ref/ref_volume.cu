// Harness around the reference's VolumeRender (core/volume.cu) - TEST
// INFRASTRUCTURE ONLY.
//
// Linked (with cuda12_texref_shim.cuh force-included) with the reference's
// core/volume.cu, core/camera.cu, core/omp.cpp, core/vector.cu,
// core/renderResources.cu and core/radiancePredict.cu, taken where they lie
// in the reference checkout, into oracle/_ref/libref_volume.so. Everything
// below runs the reference's own kernels and member functions:
//  - Fill_TR (core/volume.cu:1320-1345) over caller-given mip levels, with the
//    launch shape of Update_TR (core/volume.cu:1395-1403);
//  - Fill_Hg (core/volume.cu:1082-1160) with the launch shape of UpdateHGLut,
//    plus the curand offset each texel draws (InitRand + Rand,
//    core/render.cuh:82-91, in the same thread layout);
//  - Denoise<bool> (core/volume.cu:210-264) on caller-given buffers;
//  - VolumeRender::Update, GetSamples and the interactive Render overload;
//  - SaveBMP (core/camera.cu:10-61);
//  - load_hdr_float4 (core/hdr_loader.h:249), SetHDRI / SetEnvExp and the
//    offline Render (core/volume.cu:410-467) with the environment map.
// This TU includes only the reference's headers; the device globals and
// kernels of core/volume.cu and core/render.cuh are declared extern here.
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <vector>

#include "volume.hpp"
#include "camera.hpp"
#include "renderResources.cuh"
#include "hdr_loader.h"

extern texture<float, cudaTextureType3D, cudaReadModeElementType> texRef;
extern surface<void, cudaSurfaceType3D> surfRef;
extern surface<void, cudaSurfaceType2D> hgSurfRef;
extern __device__ int randNum;
extern __device__ int frameNum;
extern __device__ int flip;
extern __device__ float exposure;
__device__ void InitRand(curandState* seed);
__device__ float Rand(curandState* seed);
__global__ void Fill_TR(int res, float alpha, float3 lightDir);
__global__ void Fill_Hg(float g);
template <bool denoise>
__global__ void Denoise(float3* target, Histogram* histo_buffer, unsigned int* target2, int2 size, int toneType);

namespace {

int fail(cudaError_t e, const char* what) {
  fprintf(stderr, "ref volume harness: %s: %s\n", what, cudaGetErrorString(e));
  return (int)e;
}
#define CK(x) do { cudaError_t e_ = (x); if (e_ != cudaSuccess) return fail(e_, #x); } while (0)

float3 F3(const float* v) { return float3{v[0], v[1], v[2]}; }

// the offset Fill_Hg's thread (i, j) draws: its first curand_uniform
__global__ void k_hg_offsets(float* bn) {
  unsigned int i = blockIdx.x * blockDim.x + threadIdx.x;
  unsigned int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= LUT_SIZE || j >= LUT_SIZE) return;
  curandState seed;
  InitRand(&seed);
  bn[i + j * LUT_SIZE] = Rand(&seed);
}

cudaArray_t g_env_arr = nullptr;

}  // namespace

extern "C" {

void* refv_create(int res) { return new VolumeRender(res); }
void refv_destroy(void* h) { delete (VolumeRender*)h; }

// SetDatas with the caller's x-major grid, then the reference's Update():
// density texture, majorant, mip and variance pyramids. Returns max_density.
int refv_set_density_update(void* h, const float* data, float* max_density) {
  VolumeRender* v = (VolumeRender*)h;
  int r = v->resolution;
  v->SetDatas([=](int x, int y, int z, float, float, float) { return data[((size_t)x * r + y) * r + z]; });
  v->Update();
  CK(cudaDeviceSynchronize());
  *max_density = v->max_density;
  return 0;
}

// Scalars the reference keeps in __device__ globals (SetTrScale,
// SetScatterRate, SetEnvExp) and a constant environment bound to _HDRI as a
// 1 x 1 texture (what SetHDRI binds, core/volume.cu:1449-1455).
int refv_set_scalars(void* h, float tr_scale, const float* scatter3, float env_exp, const float* env_rgb) {
  VolumeRender* v = (VolumeRender*)h;
  v->SetTrScale(tr_scale);
  v->SetScatterRate(F3(scatter3));
  v->SetEnvExp(env_exp);
  v->SetCheckboard(false);
  cudaChannelFormatDesc d = cudaCreateChannelDesc<float4>();
  if (!g_env_arr) CK(cudaMallocArray(&g_env_arr, &d, 1, 1));
  float4 e = make_float4(env_rgb[0], env_rgb[1], env_rgb[2], 1.0f);
  CK(cudaMemcpy2DToArray(g_env_arr, 0, 0, &e, sizeof(e), sizeof(e), 1, cudaMemcpyHostToDevice));
  _HDRI.normalized = true;
  _HDRI.filterMode = cudaFilterModeLinear;
  _HDRI.addressMode[0] = _HDRI.addressMode[1] = _HDRI.addressMode[2] = cudaAddressModeWrap;
  CK(cudaBindTextureToArray(_HDRI, g_env_arr, d));
  CK(cudaDeviceSynchronize());
  return 0;
}

// Fill_TR for the 8 TR levels: level k (res 128 >> k) from mip level k+1 of
// `mips` (the 9 concatenated levels 256^3 .. 1^3, x-major) with alpha /
// 1.73^(k+1), as Update_TR runs it on the GPU. tr_out: the 8 levels, x-major.
int refv_fill_tr(const float* mips, float alpha, const float* light, float* tr_out) {
  cudaChannelFormatDesc ch = cudaCreateChannelDesc<float>();
  size_t moff = (size_t)256 * 256 * 256, toff = 0;
  for (int k = 0; k < 8; ++k) {
    int sr = 128 >> k;  // mip k+1
    int r = 128 >> k;   // TR level k
    cudaArray_t src = nullptr, dst = nullptr;
    CK(cudaMalloc3DArray(&src, &ch, make_cudaExtent(sr, sr, sr)));
    CK(cudaMalloc3DArray(&dst, &ch, make_cudaExtent(r, r, r), cudaArraySurfaceLoadStore));
    cudaMemcpy3DParms cp = {};
    cp.srcPtr = make_cudaPitchedPtr((void*)(mips + moff), sr * sizeof(float), sr, sr);
    cp.dstArray = src;
    cp.extent = make_cudaExtent(sr, sr, sr);
    cp.kind = cudaMemcpyHostToDevice;
    CK(cudaMemcpy3D(&cp));
    texRef.normalized = true;
    texRef.filterMode = cudaFilterModeLinear;
    texRef.addressMode[0] = texRef.addressMode[1] = texRef.addressMode[2] = cudaAddressModeBorder;
    CK(cudaBindTextureToArray(texRef, src));
    CK(cudaBindSurfaceToArray(surfRef, dst));
    float alpha_k = alpha / pow(1.73f, k + 1.0f);
    dim3 block(4, 4, 4), grid((r + 3) / 4, (r + 3) / 4, (r + 3) / 4);
    Fill_TR<<<grid, block>>>(r, alpha_k, F3(light));
    CK(cudaGetLastError());
    CK(cudaDeviceSynchronize());
    cudaMemcpy3DParms cb = {};
    cb.srcArray = dst;
    cb.dstPtr = make_cudaPitchedPtr((void*)(tr_out + toff), r * sizeof(float), r, r);
    cb.extent = make_cudaExtent(r, r, r);
    cb.kind = cudaMemcpyDeviceToHost;
    CK(cudaMemcpy3D(&cb));
    cudaDestroyTextureObject(texRef.obj);
    cudaDestroySurfaceObject(surfRef.obj);
    cudaFreeArray(src);
    cudaFreeArray(dst);
    moff += (size_t)sr * sr * sr;
    toff += (size_t)r * r * r;
  }
  return 0;
}

// Fill_Hg(g) with randNum = randnum: lut_out 512 x 512 (index i + 512 j) and
// the offset each texel drew, bn_out 512 x 512.
int refv_fill_hg(float g, int randnum, float* lut_out, float* bn_out) {
  cudaChannelFormatDesc ch = cudaCreateChannelDesc<float>();
  cudaArray_t arr = nullptr;
  CK(cudaMallocArray(&arr, &ch, LUT_SIZE, LUT_SIZE, cudaArraySurfaceLoadStore));
  CK(cudaMemcpyToSymbol(randNum, &randnum, sizeof(int)));
  CK(cudaBindSurfaceToArray(hgSurfRef, arr));
  Fill_Hg<<<dim3(LUT_SIZE / 8, LUT_SIZE / 8), dim3(8, 8)>>>(g);
  CK(cudaGetLastError());
  float* d_bn = nullptr;
  CK(cudaMalloc(&d_bn, LUT_SIZE * LUT_SIZE * sizeof(float)));
  k_hg_offsets<<<dim3(LUT_SIZE / 8, LUT_SIZE / 8), dim3(8, 8)>>>(d_bn);
  CK(cudaGetLastError());
  CK(cudaDeviceSynchronize());
  CK(cudaMemcpy2DFromArray(lut_out, LUT_SIZE * sizeof(float), arr, 0, 0, LUT_SIZE * sizeof(float), LUT_SIZE,
                           cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(bn_out, d_bn, LUT_SIZE * LUT_SIZE * sizeof(float), cudaMemcpyDeviceToHost));
  cudaFree(d_bn);
  cudaDestroySurfaceObject(hgSurfRef.obj);
  cudaFreeArray(arr);
  return 0;
}

// Denoise<denoise> on caller buffers: accum w*h*3, hist w*h*33 (the
// Histogram layout), frame (frameNum), flip, tone (0 none, 1 gamma, 2 ACES),
// exposure; out w*h packed 0xAARRGGBB. kernel_ms (may be null) receives the
// kernel's device time from CUDA events around its launch.
int refv_denoise(const float* accum, const float* hist, int w, int h, int frame, int flip_, int tone, int denoise,
                 float exp_, uint32_t* out, float* kernel_ms) {
  int n = w * h;
  float3* d_acc = nullptr;
  Histogram* d_hist = nullptr;
  unsigned int* d_out = nullptr;
  CK(cudaMalloc(&d_acc, n * sizeof(float3)));
  CK(cudaMalloc(&d_hist, n * sizeof(Histogram)));
  CK(cudaMalloc(&d_out, n * sizeof(unsigned int)));
  CK(cudaMemcpy(d_acc, accum, n * sizeof(float3), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(d_hist, hist, n * sizeof(Histogram), cudaMemcpyHostToDevice));
  CK(cudaMemcpyToSymbol(frameNum, &frame, sizeof(int)));
  CK(cudaMemcpyToSymbol(flip, &flip_, sizeof(int)));
  CK(cudaMemcpyToSymbol(exposure, &exp_, sizeof(float)));
  int group = 32, groups = (n + group - 1) / group;
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  CK(cudaEventRecord(e0));
  if (denoise)
    Denoise<true><<<groups, group>>>(d_acc, d_hist, d_out, int2{w, h}, tone);
  else
    Denoise<false><<<groups, group>>>(d_acc, d_hist, d_out, int2{w, h}, tone);
  CK(cudaGetLastError());
  CK(cudaEventRecord(e1));
  CK(cudaDeviceSynchronize());
  if (kernel_ms) CK(cudaEventElapsedTime(kernel_ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  CK(cudaMemcpy(out, d_out, n * sizeof(unsigned int), cudaMemcpyDeviceToHost));
  cudaFree(d_acc);
  cudaFree(d_hist);
  cudaFree(d_out);
  return 0;
}

// VolumeRender::GetSamples (core/volume.cu:550-626) for n points with one
// light, alpha, g and scatter; randNum = randnum seeds the curand streams.
int refv_get_samples(void* h, int n, const float* pos, const float* dir, const float* light, float alpha, float g,
                     float scatter, int bounces, int spp, int randnum, float* out) {
  VolumeRender* v = (VolumeRender*)h;
  CK(cudaMemcpyToSymbol(randNum, &randnum, sizeof(int)));
  std::vector<float> a(n, alpha), gs(n, g), sc(n, scatter);
  std::vector<float3> o(n), d(n), l(n, F3(light));
  for (int k = 0; k < n; ++k) {
    o[k] = F3(pos + 3 * k);
    d[k] = F3(dir + 3 * k);
  }
  std::vector<float3> r = v->GetSamples(a, o, d, l, gs, sc, float3{1, 1, 1}, bounces, spp);
  CK(cudaDeviceSynchronize());
  for (int k = 0; k < n; ++k) {
    out[3 * k] = r[k].x;
    out[3 * k + 1] = r[k].y;
    out[3 * k + 2] = r[k].z;
  }
  return 0;
}

// `frames` calls of the interactive Render overload (core/volume.cu:469-547)
// in delta-tracking mode with randseed 0, 1, ...: accum w*h*3, hist w*h*33,
// bgra w*h after the last frame (square frames: the reference's indexing
// assumes width = height).
int refv_interactive(void* h, int w, int hh, const float* ori, const float* up, const float* right, const float* light,
                     const float* lc, float alpha, int bounces, float g, int frames, int tone, int denoise,
                     float* accum_out, float* hist_out, uint32_t* bgra_out) {
  VolumeRender* v = (VolumeRender*)h;
  int n = w * hh;
  float3* d_acc = nullptr;
  Histogram* d_hist = nullptr;
  unsigned int* d_out = nullptr;
  CK(cudaMalloc(&d_acc, n * sizeof(float3)));
  CK(cudaMalloc(&d_hist, n * sizeof(Histogram)));
  CK(cudaMalloc(&d_out, n * sizeof(unsigned int)));
  CK(cudaMemset(d_acc, 0, n * sizeof(float3)));
  CK(cudaMemset(d_hist, 0, n * sizeof(Histogram)));
  for (int f = 0; f < frames; ++f)
    v->Render(d_acc, d_hist, d_out, int2{w, hh}, F3(ori), F3(up), F3(right), F3(light), F3(lc), alpha, bounces, g, f,
              VolumeRender::RenderType::PT, tone, denoise != 0);
  CK(cudaDeviceSynchronize());
  CK(cudaMemcpy(accum_out, d_acc, n * sizeof(float3), cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(hist_out, d_hist, n * sizeof(Histogram), cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(bgra_out, d_out, n * sizeof(unsigned int), cudaMemcpyDeviceToHost));
  cudaFree(d_acc);
  cudaFree(d_hist);
  cudaFree(d_out);
  return 0;
}

// SaveBMP (core/camera.cu:10-61) of a w x h RGBA8 image (it swaps R and B
// in place and appends ".bmp" to the path). Its swap loop visits pixel
// j + i * w for i < w, j < h, which stays inside the image only when w = h
// (the reference's cameras are square); the copy handed to it is padded to
// max(w, h)^2 pixels so that other shapes stay in bounds.
int refv_save_bmp(const uint8_t* rgba, int w, int h, const char* path) {
  size_t m = (size_t)(w > h ? w : h);
  std::vector<unsigned char> img(m * m * 4, 0);
  std::copy(rgba, rgba + (size_t)w * h * 4, img.begin());
  return SaveBMP(img.data(), w, h, path);
}

// load_hdr_float4 (core/hdr_loader.h:249): *w, *h and, if out is not null
// and cap allows, w*h*4 floats.
int refv_load_hdr(const char* path, float* out, size_t cap, int* w, int* h) {
  float* px = nullptr;
  unsigned int rx = 0, ry = 0;
  if (!load_hdr_float4(&px, &rx, &ry, path)) return 1;
  *w = (int)rx;
  *h = (int)ry;
  if (out && cap >= (size_t)rx * ry * 4) std::copy(px, px + (size_t)rx * ry * 4, out);
  free(px);
  return 0;
}

// VolumeRender::SetHDRI(path) and SetEnvExp(exp).
int refv_set_hdri(void* h, const char* path, float env_exp) {
  VolumeRender* v = (VolumeRender*)h;
  v->SetHDRI(path);
  v->SetEnvExp(env_exp);
  CK(cudaDeviceSynchronize());
  return 0;
}

// The offline VolumeRender::Render (core/volume.cu:410-467), delta tracking:
// the mean of spp passes, w x hh x 3 (square frames: its indexing assumes
// w = hh).
int refv_render_pt(void* h, int w, int hh, const float* ori, const float* up, const float* right, const float* light,
                   const float* lc, float alpha, int bounces, float g, int spp, float* out) {
  VolumeRender* v = (VolumeRender*)h;
  std::vector<float3> r = v->Render(int2{w, hh}, F3(ori), F3(up), F3(right), F3(light), VolumeRender::RenderType::PT,
                                    g, alpha, F3(lc), bounces, spp);
  CK(cudaDeviceSynchronize());
  for (size_t k = 0; k < r.size(); ++k) {
    out[3 * k] = r[k].x;
    out[3 * k + 1] = r[k].y;
    out[3 * k + 2] = r[k].z;
  }
  return 0;
}

// Camera::ACES and Camera::Gamma (core/camera.cu:66-160), the host tone maps
// RenderToFile applies: n colours in, n colours out.
int refv_tone_host(int n, const float* rgb, int tone, float* out) {
  for (int k = 0; k < n; ++k) {
    float3 c = F3(rgb + 3 * k);
    float3 r = tone == 2 ? Camera::ACES(c) : (tone == 1 ? Camera::Gamma(c) : Camera::None(c));
    out[3 * k] = r.x;
    out[3 * k + 1] = r.y;
    out[3 * k + 2] = r.z;
  }
  return 0;
}

}  // extern "C"
