// Harness around the reference's own device code - TEST INFRASTRUCTURE ONLY.
//
// Compiled (with cuda12_texref_shim.cuh force-included) together with the
// reference's core/vector.cu, core/renderResources.cu and
// core/radiancePredict.cu, taken where they lie in the reference checkout,
// into oracle/_ref/libref_mrpnn.so. The kernels below call the reference's
// CalculateRadiance, NNPredict<MRPNN> and RadiancePredict unchanged; only the
// launch loop of VolumeRender::Render (core/volume.cu:147-179, 410-467) is
// restated here, with its (8,4) block shape so that the reference's curand
// seeding (InitRand, core/render.cuh:82-87) sees the same thread ids.
#include "render.cuh"

#include <cstdio>
#include <vector>

namespace {

struct Tex3 {
  cudaArray_t arr = nullptr;
  cudaTextureObject_t obj = 0;
};
std::vector<Tex3> g_tex;
cudaArray_t g_lut_arr = nullptr, g_env_arr = nullptr;
cudaTextureObject_t g_lut = 0, g_env = 0;

int fail(cudaError_t e, const char* what) {
  fprintf(stderr, "ref harness: %s: %s\n", what, cudaGetErrorString(e));
  return (int)e;
}
#define CK(x) do { cudaError_t e_ = (x); if (e_ != cudaSuccess) return fail(e_, #x); } while (0)

// 3-D float texture of res^3 (x-major host data) with the reference's
// settings: normalized coordinates, linear filter, given address mode.
int make_tex3(const float* host, int res, cudaTextureAddressMode mode, cudaTextureObject_t* out) {
  Tex3 t;
  cudaChannelFormatDesc ch = cudaCreateChannelDesc<float>();
  cudaExtent ext = make_cudaExtent(res, res, res);
  CK(cudaMalloc3DArray(&t.arr, &ch, ext));
  cudaMemcpy3DParms cp = {};
  cp.srcPtr = make_cudaPitchedPtr((void*)host, res * sizeof(float), res, res);
  cp.dstArray = t.arr;
  cp.extent = ext;
  cp.kind = cudaMemcpyHostToDevice;
  CK(cudaMemcpy3D(&cp));
  cudaResourceDesc rd = {};
  rd.resType = cudaResourceTypeArray;
  rd.res.array.array = t.arr;
  cudaTextureDesc td = {};
  td.addressMode[0] = td.addressMode[1] = td.addressMode[2] = mode;
  td.filterMode = cudaFilterModeLinear;
  td.readMode = cudaReadModeElementType;
  td.normalizedCoords = 1;
  CK(cudaCreateTextureObject(&t.obj, &rd, &td, nullptr));
  g_tex.push_back(t);
  *out = t.obj;
  return 0;
}

int make_tex2(const void* host, int w, int h, cudaChannelFormatDesc ch, size_t elem, cudaTextureAddressMode mode,
              cudaArray_t* arr, cudaTextureObject_t* out) {
  CK(cudaMallocArray(arr, &ch, w, h));
  CK(cudaMemcpy2DToArray(*arr, 0, 0, host, w * elem, w * elem, h, cudaMemcpyHostToDevice));
  cudaResourceDesc rd = {};
  rd.resType = cudaResourceTypeArray;
  rd.res.array.array = *arr;
  cudaTextureDesc td = {};
  td.addressMode[0] = td.addressMode[1] = mode;
  td.filterMode = cudaFilterModeLinear;
  td.readMode = cudaReadModeElementType;
  td.normalizedCoords = 1;
  CK(cudaCreateTextureObject(out, &rd, &td, nullptr));
  return 0;
}

template <class R>
int set_ref(R& symbol, cudaTextureObject_t obj) {
  legacy_texref<float> h;
  h.obj = obj;
  CK(cudaMemcpyToSymbol(symbol, &h, sizeof(h)));
  return 0;
}

__global__ void k_pass_pt(float3* out, int2 size, float3 ori, float3 up, float3 right, float3 lightDir,
                          float3 lightColor, float alpha, int multiScatter, float g) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  int idx = i * size.x + j;
  curandState seed;
  InitRand(&seed);
  float u = 1 - (j + Rand(&seed)) / size.x;
  float v = 1 - (i + Rand(&seed)) / size.y;
  float3 forward = normalize(-ori);
  float3 dir = normalize(forward + (right * (u * 2 - 1)) + (up * (v * 2 - 1)));
  float4 r = CalculateRadiance(ori, dir, lightDir, lightColor, alpha, multiScatter, g, 1);
  float3 res = max(float3{0, 0, 0}, make_float3(r));
  if (i >= size.x || j >= size.y) return;
  out[idx] = res;
}

__global__ void k_pass_nn(float3* out, int2 size, float3 ori, float3 up, float3 right, float3 lightDir,
                          float3 lightColor, float alpha, float g) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  int idx = i * size.x + j;
  curandState seed;
  InitRand(&seed);
  float u = 1 - (j + Rand(&seed)) / size.x;
  float v = 1 - (i + Rand(&seed)) / size.y;
  float3 forward = normalize(-ori);
  float3 dir = normalize(forward + (right * (u * 2 - 1)) + (up * (v * 2 - 1)));
  float4 r = NNPredict<Type::MRPNN>(ori, dir, lightDir, lightColor, alpha, g);
  float3 res = max(float3{0, 0, 0}, make_float3(r));
  if (i >= size.x || j >= size.y) return;
  out[idx] = res;
}

// NNPredict<Type::marching_MRPNN> (core/render.cuh:524-633), which the
// reference's own host code never instantiates: one pass, same camera model.
__global__ void k_pass_march(float3* out, int2 size, float3 ori, float3 up, float3 right, float3 lightDir,
                             float3 lightColor, float alpha, float g) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  int idx = i * size.x + j;
  curandState seed;
  InitRand(&seed);
  float u = 1 - (j + Rand(&seed)) / size.x;
  float v = 1 - (i + Rand(&seed)) / size.y;
  float3 forward = normalize(-ori);
  float3 dir = normalize(forward + (right * (u * 2 - 1)) + (up * (v * 2 - 1)));
  float4 r = NNPredict<Type::marching_MRPNN>(ori, dir, lightDir, lightColor, alpha, g);
  float3 res = max(float3{0, 0, 0}, make_float3(r));
  if (i >= size.x || j >= size.y) return;
  out[idx] = res;
}

__global__ void k_accum(const float3* in, int n, double* sum, double* sumsq) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  float3 v = in[k];
  sum[3 * k] += v.x; sum[3 * k + 1] += v.y; sum[3 * k + 2] += v.z;
  sumsq[3 * k] += (double)v.x * v.x; sumsq[3 * k + 1] += (double)v.y * v.y; sumsq[3 * k + 2] += (double)v.z * v.z;
}

// RadiancePredict with explicit frames; every lane of a warp calls it (the
// reference's layer code shuffles across the full warp).
__global__ void k_predict_frames(int n, const float* pos, const float* frame, float3 L, float alpha, float g,
                                 float3 scatterrate, float* out) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  int kk = k < n ? k : n - 1;
  const float* f = frame + 12 * kk;
  curandState st;
  float3 p = float3{pos[3 * kk], pos[3 * kk + 1], pos[3 * kk + 2]};
  float3 r = RadiancePredict(&st, true, p, L, float3{f[0], f[1], f[2]}, float3{f[3], f[4], f[5]},
                             float3{f[6], f[7], f[8]}, float3{f[9], f[10], f[11]}, float3{0, 0, 0},
                             float3{0, 0, 0}, alpha, g, scatterrate);
  if (k < n) { out[3 * k] = r.x; out[3 * k + 1] = r.y; out[3 * k + 2] = r.z; }
}

__global__ void k_stencil(float* out) {
  int i = threadIdx.x;
  if (i >= 160) return;
  float3 p = SphereRandom3(i, 1.0f, float3{1, 0, 0}, float3{0, 1, 0}, float3{0, 0, 1}, 0.0f);
  out[3 * i] = p.x; out[3 * i + 1] = p.y; out[3 * i + 2] = p.z;
}

float3 F3(const float* v) { return float3{v[0], v[1], v[2]}; }

}  // namespace

extern "C" {

// Bind the volume tables: density res^3, mips (9 concatenated levels
// 256^3..1^3), tr (8 levels 128^3..1^3), lut 512x512, constant environment.
int ref_setup(const float* density, int res, float max_density, const float* mips, const float* tr,
              const float* lut, const float* env, const float* albedo, float tr_scale_) {
  cudaTextureObject_t o;
  if (make_tex3(density, res, cudaAddressModeBorder, &o)) return 1;
  if (set_ref(_DensityVolume, o)) return 1;
  size_t off = 0;
  for (int k = 0; k < 9; ++k) {
    int r = 256 >> k;
    if (make_tex3(mips + off, r, cudaAddressModeBorder, &o)) return 1;
    off += (size_t)r * r * r;
    int rc = 0;
    switch (k) {
      case 0: rc = set_ref(_Mips0, o); break; case 1: rc = set_ref(_Mips1, o); break;
      case 2: rc = set_ref(_Mips2, o); break; case 3: rc = set_ref(_Mips3, o); break;
      case 4: rc = set_ref(_Mips4, o); break; case 5: rc = set_ref(_Mips5, o); break;
      case 6: rc = set_ref(_Mips6, o); break; case 7: rc = set_ref(_Mips7, o); break;
      default: rc = set_ref(_Mips8, o); break;
    }
    if (rc) return 1;
  }
  off = 0;
  for (int k = 0; k < 8; ++k) {
    int r = 128 >> k;
    if (make_tex3(tr + off, r, cudaAddressModeClamp, &o)) return 1;
    off += (size_t)r * r * r;
    int rc = 0;
    switch (k) {
      case 0: rc = set_ref(_TR_Mips0, o); break; case 1: rc = set_ref(_TR_Mips1, o); break;
      case 2: rc = set_ref(_TR_Mips2, o); break; case 3: rc = set_ref(_TR_Mips3, o); break;
      case 4: rc = set_ref(_TR_Mips4, o); break; case 5: rc = set_ref(_TR_Mips5, o); break;
      case 6: rc = set_ref(_TR_Mips6, o); break; default: rc = set_ref(_TR_Mips7, o); break;
    }
    if (rc) return 1;
  }
  if (make_tex2(lut, 512, 512, cudaCreateChannelDesc<float>(), sizeof(float), cudaAddressModeClamp, &g_lut_arr,
                &g_lut))
    return 1;
  if (set_ref(_HGLut, g_lut)) return 1;
  float4 e = make_float4(env[0], env[1], env[2], 1.0f);
  if (make_tex2(&e, 1, 1, cudaCreateChannelDesc<float4>(), sizeof(float4), cudaAddressModeWrap, &g_env_arr, &g_env))
    return 1;
  if (set_ref(_HDRI, g_env)) return 1;
  float one = 1.0f, ior = -1.0f;
  float3 sr = F3(albedo);
  CK(cudaMemcpyToSymbol(maxDensity, &max_density, sizeof(float)));
  CK(cudaMemcpyToSymbol(Resolution, &res, sizeof(int)));
  CK(cudaMemcpyToSymbol(tr_scale, &tr_scale_, sizeof(float)));
  CK(cudaMemcpyToSymbol(enviroment_exp, &one, sizeof(float)));
  CK(cudaMemcpyToSymbol(IOR, &ior, sizeof(float)));
  CK(cudaMemcpyToSymbol(scatter_rate, &sr, sizeof(float3)));
  return 0;
}

// SetSurfaceIOR (the marching form's surface; <= 0: none).
int ref_set_ior(float ior) {
  CK(cudaMemcpyToSymbol(IOR, &ior, sizeof(float)));
  return 0;
}

// mode 0: offline PT render (VolumeRender::Render with rt = PT); 1: NNPredict<MRPNN>;
// 2: NNPredict<marching_MRPNN>. spp passes, per-pixel
// fp64 sums and sums of squares of the per-pass radiance (host buffers).
int ref_render(int mode, int w, int h, const float* ori, const float* up, const float* right, const float* light,
               const float* light_color, float alpha, int multi_scatter, float g, int spp, double* sum,
               double* sumsq) {
  int n = w * h;
  float3* d_out = nullptr;
  double *d_sum = nullptr, *d_sq = nullptr;
  CK(cudaMalloc(&d_out, n * sizeof(float3)));
  CK(cudaMalloc(&d_sum, 3 * n * sizeof(double)));
  CK(cudaMalloc(&d_sq, 3 * n * sizeof(double)));
  CK(cudaMemset(d_sum, 0, 3 * n * sizeof(double)));
  CK(cudaMemset(d_sq, 0, 3 * n * sizeof(double)));
  dim3 block(8, 4), grid((w + 7) / 8, (h + 3) / 4);
  for (int i = 0; i < spp; ++i) {
    CK(cudaMemcpyToSymbol(frameNum, &i, sizeof(int)));
    CK(cudaMemcpyToSymbol(randNum, &i, sizeof(int)));
    if (mode == 0)
      k_pass_pt<<<grid, block>>>(d_out, int2{w, h}, F3(ori), F3(up), F3(right), F3(light), F3(light_color), alpha,
                                 multi_scatter, g);
    else if (mode == 1)
      k_pass_nn<<<grid, block>>>(d_out, int2{w, h}, F3(ori), F3(up), F3(right), F3(light), F3(light_color), alpha, g);
    else
      k_pass_march<<<grid, block>>>(d_out, int2{w, h}, F3(ori), F3(up), F3(right), F3(light), F3(light_color), alpha,
                                    g);
    k_accum<<<(n + 127) / 128, 128>>>(d_out, n, d_sum, d_sq);
    CK(cudaGetLastError());
  }
  CK(cudaDeviceSynchronize());
  CK(cudaMemcpy(sum, d_sum, 3 * n * sizeof(double), cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(sumsq, d_sq, 3 * n * sizeof(double), cudaMemcpyDeviceToHost));
  cudaFree(d_out);
  cudaFree(d_sum);
  cudaFree(d_sq);
  return 0;
}

// RadiancePredict (gather through the bound tables + network) for n points
// with explicit frames: pos n x 3, frame n x 12, out n x 3 (host buffers).
int ref_predict_frames(int n, const float* pos, const float* frame, const float* light, float alpha, float g,
                       const float* scatterrate, float* out) {
  float *d_pos, *d_fr, *d_out;
  CK(cudaMalloc(&d_pos, 3 * n * sizeof(float)));
  CK(cudaMalloc(&d_fr, 12 * n * sizeof(float)));
  CK(cudaMalloc(&d_out, 3 * n * sizeof(float)));
  CK(cudaMemcpy(d_pos, pos, 3 * n * sizeof(float), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(d_fr, frame, 12 * n * sizeof(float), cudaMemcpyHostToDevice));
  k_predict_frames<<<(n + 31) / 32, 32>>>(n, d_pos, d_fr, F3(light), alpha, g, F3(scatterrate), d_out);
  CK(cudaGetLastError());
  CK(cudaDeviceSynchronize());
  CK(cudaMemcpy(out, d_out, 3 * n * sizeof(float), cudaMemcpyDeviceToHost));
  cudaFree(d_pos);
  cudaFree(d_fr);
  cudaFree(d_out);
  return 0;
}

// The reference's 160 stencil points (SphereRandom3 with the identity frame).
int ref_read_stencil(float* out480) {
  float* d;
  CK(cudaMalloc(&d, 480 * sizeof(float)));
  k_stencil<<<1, 160>>>(d);
  CK(cudaDeviceSynchronize());
  CK(cudaMemcpy(out480, d, 480 * sizeof(float), cudaMemcpyDeviceToHost));
  cudaFree(d);
  return 0;
}

void ref_teardown() {
  for (auto& t : g_tex) { cudaDestroyTextureObject(t.obj); cudaFreeArray(t.arr); }
  g_tex.clear();
  if (g_lut) cudaDestroyTextureObject(g_lut);
  if (g_env) cudaDestroyTextureObject(g_env);
  if (g_lut_arr) cudaFreeArray(g_lut_arr);
  if (g_env_arr) cudaFreeArray(g_env_arr);
  g_lut = g_env = 0;
  g_lut_arr = g_env_arr = nullptr;
}

}  // extern "C"
