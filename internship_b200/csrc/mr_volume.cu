// Volume build on the GPU: global majorant, density mip pyramid with its
// 2x2x2 variance pyramid, light-transmittance (TR) pyramid and the
// cone-averaged Henyey-Greenstein table. Replaces VolumeRender::Update /
// Update_TR / UpdateHGLut (core/volume.cu:1161-1424) and the host OpenMP loops
// they ran; all tables live as raw fp32 arrays in HBM (index (x*r+y)*r+z).
#include <cmath>

#include "mr_internal.h"

namespace mr {

// ---- majorant -------------------------------------------------------------------
// max over the grid (floored at 1e-5 like core/volume.cu:1219-1224); values are
// compared as non-negative floats through their int bit patterns.
__global__ void k_max_density(const float* __restrict__ d, size_t n, float* out) {
  float m = 0.00001f;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    m = fmaxf(m, __ldg(d + i));
  for (int o = 16; o; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  __shared__ float sm[32];
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) sm[wid] = m;
  __syncthreads();
  if (wid == 0) {
    m = lane < (int)(blockDim.x >> 5) ? sm[lane] : 0.00001f;
    for (int o = 16; o; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (lane == 0) atomicMax((int*)out, __float_as_int(m));
  }
}

// mip0 = trilinear resample of the density (negatives clamped to 0, zero
// border) at the 256^3 texel centres (core/volume.cu:675-703, 1228-1247).
__global__ void k_mip0(const float* __restrict__ d, int res, float* __restrict__ m0) {
  unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 256u * 256u * 256u) return;
  int z = i & 255, y = (i >> 8) & 255, x = i >> 16;
  float px = ((float)x + 0.5f) / 256.0f * res - 0.5f;
  float py = ((float)y + 0.5f) / 256.0f * res - 0.5f;
  float pz = ((float)z + 0.5f) / 256.0f * res - 0.5f;
  float fx = floorf(px), fy = floorf(py), fz = floorf(pz);
  int xi = (int)fx, yi = (int)fy, zi = (int)fz;
  float wx = px - fx, wy = py - fy, wz = pz - fz;
  auto tap = [&](int a, int b, int c) -> float {
    if ((unsigned)a >= (unsigned)res || (unsigned)b >= (unsigned)res || (unsigned)c >= (unsigned)res) return 0.0f;
    return fmaxf(0.0f, __ldg(d + ((size_t)a * res + b) * res + c));
  };
  float c000 = tap(xi, yi, zi), c001 = tap(xi, yi, zi + 1), c010 = tap(xi, yi + 1, zi), c011 = tap(xi, yi + 1, zi + 1);
  float c100 = tap(xi + 1, yi, zi), c101 = tap(xi + 1, yi, zi + 1), c110 = tap(xi + 1, yi + 1, zi), c111 = tap(xi + 1, yi + 1, zi + 1);
  m0[i] = lerpf(lerpf(lerpf(c000, c001, wz), lerpf(c010, c011, wz), wy),
                lerpf(lerpf(c100, c101, wz), lerpf(c110, c111, wz), wy), wx);
}

// mip k+1 = 2x2x2 mean of mip k, var k+1 = max(0, E[x^2]-E[x]^2)
// (intended semantics of core/volume.cu:1249-1287 and :775-827).
__global__ void k_mip_down(const float* __restrict__ src, int r, float* __restrict__ dm, float* __restrict__ dv) {
  int nr = r >> 1;
  unsigned n = (unsigned)nr * nr * nr;
  unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int z = i % nr, y = (i / nr) % nr, x = i / (nr * nr);
  float s = 0.0f, s2 = 0.0f;
#pragma unroll
  for (int dx = 0; dx < 2; ++dx)
#pragma unroll
    for (int dy = 0; dy < 2; ++dy)
#pragma unroll
      for (int dz = 0; dz < 2; ++dz) {
        float v = __ldg(src + ((size_t)(2 * x + dx) * r + (2 * y + dy)) * r + (2 * z + dz));
        s += v;
        s2 = __fadd_rn(s2, __fmul_rn(v, v));
      }
  float mean = s / 8.0f;
  float variance = __fsub_rn(s2 / 8.0f, __fmul_rn(mean, mean));
  dm[i] = mean;
  dv[i] = fmaxf(0.0f, variance);
}

// Fill_TR (core/volume.cu:1320-1345): per voxel of TR level k (res r =
// 128>>k), 128 steps towards the light through mip k+1, alpha/1.73^(k+1).
__global__ void k_tr_level(const float* __restrict__ src, int r, float a, F3 L, float* __restrict__ dst) {
  unsigned n = (unsigned)r * r * r;
  unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int z = i % r, y = (i / r) % r, x = i / (r * r);
  F3 uv = f3(((float)x + 0.5f) / (float)r, ((float)y + 0.5f) / (float)r, ((float)z + 0.5f) / (float)r);
  F3 o = uv - 0.5f;
  float dis = ray_box_distance(o, L);
  float step = dis / 128.0f;
  F3 lp = o;
  float sum = 0.0f;
  for (int s = 0; s < 128; ++s) {
    lp = lp + L * step;
    sum = sum + tri_border(src, r, lp + 0.5f);
  }
  dst[i] = expf(-sum * a * step);
}

// Scrambled radical inverse of a in base B: digit d of a becomes digit
// perm(d), perm packed four bits per digit in P (digit d at bits 4d..4d+3),
// and the infinite tail of perm(0) digits is added in closed form,
// perm(0) / (B - 1) times the last digit weight; clamped below 1
// (ScrambledRadicalInverse, core/volume.cu:1060-1076).
template <uint32_t B, uint64_t P>
__device__ __forceinline__ float scrambled_radical_inverse(uint32_t a) {
  const float inv_base = 1.0f / (float)B;
  uint32_t rev = 0;
  float inv_bn = 1.0f;
  while (a) {
    uint32_t next = a / B;
    uint32_t digit = a - next * B;
    rev = rev * B + (uint32_t)((P >> (4u * digit)) & 15u);
    inv_bn *= inv_base;
    a = next;
  }
  return fminf(inv_bn * ((float)rev + inv_base * (float)(P & 15u) / (1.0f - inv_base)), 0.99999994f);
}
// Digit permutations of the four Halton dimensions the HG table draws
// (dimensions 0, 1, 2 and 4: bases 2, 3, 5 and 11). They are the entries of
// the reference's permutation table for those bases (core/volume.cu:956-958:
// {0,1}, {2,1,0}, {4,1,2,3,0}, {8,3,5,4,7,2,6,9,1,10,0}); the table's sample
// points, and so its values, depend on them.
constexpr uint64_t kPermB2 = 0x10ull, kPermB3 = 0x12ull, kPermB5 = 0x3214ull, kPermB11 = 0xa196274538ull;
__device__ __forceinline__ float fracf_(float f) { return f - (float)(long long)f; }

// Fill_Hg (core/volume.cu:1082-1160): lut[i + j*512] = mean of HG over a ball
// of radius tan(angle_j) centred at unit distance along cos_i, estimated with
// 1024 scrambled Halton points (bases 2,3,5,11) mixing HG-sampled chords and
// uniform ball points. Per-texel Cranley-Patterson offset from Philox
// (TAG_LUT) where the reference draws it from curand.
__global__ void k_hglut(float g, uint32_t seed, float* __restrict__ lut) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= kLut || j >= kLut) return;
  float costheta = (((float)i + 0.5f) / 512.0f) * 2.0f - 1.0f;
  float aa = ((float)j + 0.5f) / 512.0f;
  float angle = aa * 3.1415926535f * 60.0f / 180.0f;
  uint32_t o[4];
  philox4x32_10((uint32_t)(i + j * 512), 0u, 0u, TAG_LUT, seed, 0u, o);
  float bn = u01(o[0]);
  float hg = 0.0f;
  float R = tanf(angle);
  F3 view = f3(1, 0, 0);
  F3 D = f3(costheta, sqrtf(1.0f - costheta * costheta), 0.0f);
  float mis = 0.0f;
  {
    float p = R * R - 1 + D.x * D.x;
    if (p > 0) {
      float sdotl = g > 0 ? D.x : -D.x;
      float w = sqrtf(p);
      float d0 = fmaxf(0.0f, sdotl - w) / R;
      float d1 = (sdotl + w) / R;
      float d = d1 * d1 * d1 - d0 * d0 * d0;
      mis = (d1 > d0) ? d : 0.0f;
    }
    mis = fminf(fmaxf(mis, 1e-8f), 1.0f);
    float a = fabsf(g);
    a = a < 0.6f ? 0.0f : (a < 0.7f ? (a - 0.6f) * 9.0f : (powf((a - 0.7f) / 0.3f, 0.05f) * 0.1f + 0.9f));
    mis = 1.0f - 1.0f / (1.0f + a * mis / (1.0f - a));
  }
  for (int k = 0; k < 1024; ++k) {
    float r0 = fracf_(scrambled_radical_inverse<2, kPermB2>(k) + bn);
    float r1 = fracf_(scrambled_radical_inverse<3, kPermB3>(k) + bn);
    if (fracf_(scrambled_radical_inverse<11, kPermB11>(k) + bn) < mis) {
      F3 l = hg_sample_dir(r0, r1, view, g);
      float sdotl = dot(D, l);
      float p = R * R - 1 + sdotl * sdotl;
      if (p <= 0) continue;
      float w = sqrtf(p);
      float d0 = sdotl - w;
      float d1 = (sdotl + w) / R;
      d0 = fmaxf(0.0f, d0) / R;
      float d = d1 * d1 * d1 - d0 * d0 * d0;
      hg += fmaxf(0.0f, d / 4);
    } else {
      float r2 = fracf_(scrambled_radical_inverse<5, kPermB5>(k) + bn);
      float theta = r0 * 2.0f * 3.1415926535f;
      float phi = acosf(2.0f * r1 - 1.0f);
      float rr = cbrtf(r2);
      float sphi = sinf(phi), cphi = cosf(phi);
      float x = R * rr * sphi * cosf(theta);
      float y = R * rr * sphi * sinf(theta);
      float z = R * rr * cphi;
      F3 rp = f3(x, y, z) + D;
      hg += hg_phase(dot(normalize(rp), view), g);
    }
  }
  lut[i + j * 512] = hg / 1024.0f;
}

static int grid_for(size_t n, int block) { return (int)((n + block - 1) / block); }

// L is normalised by the caller and is also the key the callers compare with
// (normalising it again could change it by an ulp and defeat the cache).
int launch_update_tr(Volume* v, F3 L, float alpha, cudaStream_t s) {
  v->timer.mark(ST_TR, s);
  for (int k = 0; k < 8; ++k) {
    int r = 128 >> k;
    float a = alpha / powf(1.73f, (float)k + 1.0f);
    size_t n = (size_t)r * r * r;
    k_tr_level<<<grid_for(n, 128), 128, 0, s>>>(v->mips + mip_offset(k + 1), r, a, L, v->tr + tr_offset(k));
  }
  v->timer.mark(ST_TR, s);
  MR_CUDA(cudaGetLastError());
  v->tr_valid = true;
  v->tex_tr_stale = true;
  v->gth_tr_stale = true;
  v->tr_light = L;
  v->tr_alpha = alpha;
  return MR_OK;
}

int launch_update_lut(Volume* v, float g, uint32_t seed, cudaStream_t s) {
  v->timer.mark(ST_LUT, s);
  k_hglut<<<dim3(kLut / 16, kLut / 16), dim3(16, 16), 0, s>>>(g, seed, v->lut);
  v->timer.mark(ST_LUT, s);
  MR_CUDA(cudaGetLastError());
  v->lut_valid = true;
  v->tex_lut_stale = true;
  v->gth_lut_stale = true;
  v->lut_g = g;
  v->lut_seed = seed;
  return MR_OK;
}

// ---- texture-unit copies (MR_SAMPLER_TEXTURE) --------------------------------------
// cudaArray extent (width, height, depth) = (z, y, x) of the x-major tables;
// sampled as tex3D(obj, uv.z, uv.y, uv.x) like the reference's texture refs.
static int make_tex3(cudaArray_t* arr, cudaTextureObject_t* tex, int r, cudaTextureAddressMode mode) {
  cudaChannelFormatDesc ch = cudaCreateChannelDesc<float>();
  MR_CUDA(cudaMalloc3DArray(arr, &ch, make_cudaExtent(r, r, r)));
  cudaResourceDesc rd = {};
  rd.resType = cudaResourceTypeArray;
  rd.res.array.array = *arr;
  cudaTextureDesc td = {};
  td.addressMode[0] = td.addressMode[1] = td.addressMode[2] = mode;
  td.filterMode = cudaFilterModeLinear;
  td.readMode = cudaReadModeElementType;
  td.normalizedCoords = 1;
  MR_CUDA(cudaCreateTextureObject(tex, &rd, &td, nullptr));
  return MR_OK;
}
int copy_to_array(cudaArray_t arr, const float* src, int r, cudaStream_t s) {
  cudaMemcpy3DParms cp = {};
  cp.srcPtr = make_cudaPitchedPtr((void*)src, r * sizeof(float), r, r);
  cp.dstArray = arr;
  cp.extent = make_cudaExtent(r, r, r);
  cp.kind = cudaMemcpyDeviceToDevice;
  MR_CUDA(cudaMemcpy3DAsync(&cp, s));
  return MR_OK;
}

int refresh_textures(Volume* v, cudaStream_t s) {
  if (!v->lut_arr) {
    for (int k = 0; k < 9; ++k) {
      int rc = make_tex3(&v->mip_arr[k], &v->mip_tex[k], 256 >> k, cudaAddressModeBorder);
      if (rc) return rc;
    }
    for (int k = 0; k < 8; ++k) {
      int rc = make_tex3(&v->tr_arr[k], &v->tr_tex[k], 128 >> k, cudaAddressModeClamp);
      if (rc) return rc;
    }
    cudaChannelFormatDesc ch = cudaCreateChannelDesc<float>();
    MR_CUDA(cudaMallocArray(&v->lut_arr, &ch, kLut, kLut));
    cudaResourceDesc rd = {};
    rd.resType = cudaResourceTypeArray;
    rd.res.array.array = v->lut_arr;
    cudaTextureDesc td = {};
    td.addressMode[0] = td.addressMode[1] = cudaAddressModeClamp;
    td.filterMode = cudaFilterModeLinear;
    td.readMode = cudaReadModeElementType;
    td.normalizedCoords = 1;
    MR_CUDA(cudaCreateTextureObject(&v->lut_tex, &rd, &td, nullptr));
    v->tex_mips_stale = v->tex_tr_stale = v->tex_lut_stale = true;
  }
  if (v->tex_mips_stale) {
    for (int k = 0; k < 9; ++k) {
      int rc = copy_to_array(v->mip_arr[k], v->mips + mip_offset(k), 256 >> k, s);
      if (rc) return rc;
    }
    v->tex_mips_stale = false;
  }
  if (v->tex_tr_stale) {
    for (int k = 0; k < 8; ++k) {
      int rc = copy_to_array(v->tr_arr[k], v->tr + tr_offset(k), 128 >> k, s);
      if (rc) return rc;
    }
    v->tex_tr_stale = false;
  }
  if (v->tex_lut_stale) {
    MR_CUDA(cudaMemcpy2DToArrayAsync(v->lut_arr, 0, 0, v->lut, kLut * sizeof(float), kLut * sizeof(float), kLut,
                                     cudaMemcpyDeviceToDevice, s));
    v->tex_lut_stale = false;
  }
  return MR_OK;
}

// ---- layered copies for the exact sampler's texture gathers ------------------------
// Layered cudaArray of r layers (x) of r x r texels (width z, height y), read
// with unnormalised coordinates and point sampling: tld4 returns the four
// texels of a 2 x 2 (z, y) footprint unchanged, and the y / z borders come
// from the address mode (border 0 for the density levels, clamp for the
// transmittance levels), as in the fp32 software filter.
int make_gather_tex(cudaArray_t* arr, cudaTextureObject_t* tex, int r, cudaTextureAddressMode mode) {
  cudaChannelFormatDesc ch = cudaCreateChannelDesc<float>();
  MR_CUDA(cudaMalloc3DArray(arr, &ch, make_cudaExtent(r, r, r), cudaArrayLayered));
  cudaResourceDesc rd = {};
  rd.resType = cudaResourceTypeArray;
  rd.res.array.array = *arr;
  cudaTextureDesc td = {};
  td.addressMode[0] = td.addressMode[1] = td.addressMode[2] = mode;
  td.filterMode = cudaFilterModePoint;
  td.readMode = cudaReadModeElementType;
  td.normalizedCoords = 0;
  MR_CUDA(cudaCreateTextureObject(tex, &rd, &td, nullptr));
  return MR_OK;
}

int refresh_gather_textures(Volume* v, cudaStream_t s) {
  if (!v->gth_lut_arr) {
    for (int k = 0; k < 9; ++k) {
      int rc = make_gather_tex(&v->gth_mip_arr[k], &v->gth_mip_tex[k], 256 >> k, cudaAddressModeBorder);
      if (rc) return rc;
    }
    for (int k = 0; k < 8; ++k) {
      int rc = make_gather_tex(&v->gth_tr_arr[k], &v->gth_tr_tex[k], 128 >> k, cudaAddressModeClamp);
      if (rc) return rc;
    }
    cudaChannelFormatDesc ch = cudaCreateChannelDesc<float>();
    MR_CUDA(cudaMallocArray(&v->gth_lut_arr, &ch, kLut, kLut));
    cudaResourceDesc rd = {};
    rd.resType = cudaResourceTypeArray;
    rd.res.array.array = v->gth_lut_arr;
    cudaTextureDesc td = {};
    td.addressMode[0] = td.addressMode[1] = cudaAddressModeClamp;
    td.filterMode = cudaFilterModePoint;
    td.readMode = cudaReadModeElementType;
    td.normalizedCoords = 0;
    MR_CUDA(cudaCreateTextureObject(&v->gth_lut_tex, &rd, &td, nullptr));
    v->gth_mips_stale = v->gth_tr_stale = v->gth_lut_stale = true;
  }
  if (v->gth_mips_stale) {
    for (int k = 0; k < 9; ++k) {
      int rc = copy_to_array(v->gth_mip_arr[k], v->mips + mip_offset(k), 256 >> k, s);
      if (rc) return rc;
    }
    v->gth_mips_stale = false;
  }
  if (v->gth_tr_stale) {
    for (int k = 0; k < 8; ++k) {
      int rc = copy_to_array(v->gth_tr_arr[k], v->tr + tr_offset(k), 128 >> k, s);
      if (rc) return rc;
    }
    v->gth_tr_stale = false;
  }
  if (v->gth_lut_stale) {
    MR_CUDA(cudaMemcpy2DToArrayAsync(v->gth_lut_arr, 0, 0, v->lut, kLut * sizeof(float), kLut * sizeof(float), kLut,
                                     cudaMemcpyDeviceToDevice, s));
    v->gth_lut_stale = false;
  }
  return MR_OK;
}

int density_gather_texture(Volume* v, cudaStream_t s, cudaTextureObject_t* out) {
  if (!v->gth_den_arr) {
    int rc = make_gather_tex(&v->gth_den_arr, &v->gth_den_tex, v->res, cudaAddressModeBorder);
    if (rc) return rc;
    v->gth_den_stale = true;
  }
  if (v->gth_den_stale) {
    int rc = copy_to_array(v->gth_den_arr, v->density, v->res, s);
    if (rc) return rc;
    v->gth_den_stale = false;
  }
  *out = v->gth_den_tex;
  return MR_OK;
}

void destroy_textures(Volume* v) {
  if (v->gth_den_tex) cudaDestroyTextureObject(v->gth_den_tex);
  if (v->gth_den_arr) cudaFreeArray(v->gth_den_arr);
  for (int k = 0; k < 9; ++k) {
    if (v->gth_mip_tex[k]) cudaDestroyTextureObject(v->gth_mip_tex[k]);
    if (v->gth_mip_arr[k]) cudaFreeArray(v->gth_mip_arr[k]);
  }
  for (int k = 0; k < 8; ++k) {
    if (v->gth_tr_tex[k]) cudaDestroyTextureObject(v->gth_tr_tex[k]);
    if (v->gth_tr_arr[k]) cudaFreeArray(v->gth_tr_arr[k]);
  }
  if (v->gth_lut_tex) cudaDestroyTextureObject(v->gth_lut_tex);
  if (v->gth_lut_arr) cudaFreeArray(v->gth_lut_arr);
  for (int k = 0; k < 9; ++k) {
    if (v->mip_tex[k]) cudaDestroyTextureObject(v->mip_tex[k]);
    if (v->mip_arr[k]) cudaFreeArray(v->mip_arr[k]);
  }
  for (int k = 0; k < 8; ++k) {
    if (v->tr_tex[k]) cudaDestroyTextureObject(v->tr_tex[k]);
    if (v->tr_arr[k]) cudaFreeArray(v->tr_arr[k]);
  }
  if (v->lut_tex) cudaDestroyTextureObject(v->lut_tex);
  if (v->lut_arr) cudaFreeArray(v->lut_arr);
}

int ensure_scratch(Volume* v, size_t bytes, cudaStream_t s) {
  if (v->scratch_bytes >= bytes) return MR_OK;
  if (v->scratch) MR_CUDA(cudaFreeAsync(v->scratch, s));
  v->scratch = nullptr;
  v->scratch_bytes = 0;
  cudaError_t e = cudaMallocAsync(&v->scratch, bytes, s);
  if (e != cudaSuccess) return set_error(MR_ERR_NOMEM, "scratch allocation of %zu bytes failed: %s", bytes, cudaGetErrorString(e));
  v->scratch_bytes = bytes;
  return MR_OK;
}

}  // namespace mr

using namespace mr;

extern "C" {

int mr_volume_create(int32_t resolution, mr_volume** out) {
  clear_error();
  if (!out) return set_error(MR_ERR_ARG, "mr_volume_create: out is NULL");
  *out = nullptr;
  if (resolution < 2 || resolution > 2048) return set_error(MR_ERR_ARG, "resolution %d outside [2, 2048]", resolution);
  mr_volume* h = new mr_volume();
  Volume* v = &h->v;
  v->res = resolution;
  cudaGetDevice(&v->device);
  size_t n = (size_t)resolution * resolution * resolution;
  cudaError_t e = cudaSuccess;
  if (e == cudaSuccess) e = cudaMalloc(&v->density, n * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&v->mips, kMipTotal * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&v->var, kMipTotal * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&v->tr, kTrTotal * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&v->lut, kLut * kLut * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&v->d_max, sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&v->d_counters, kCounters * sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMemset(v->d_counters, 0, kCounters * sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMemset(v->density, 0, n * sizeof(float));
  if (e != cudaSuccess) {
    mr_volume_destroy(h);
    return set_error(MR_ERR_NOMEM, "mr_volume_create(%d): %s", resolution, cudaGetErrorString(e));
  }
  *out = h;
  return MR_OK;
}

int mr_volume_destroy(mr_volume* h) {
  if (!h) return MR_OK;
  Volume* v = &h->v;
  cudaFree(v->density);
  cudaFree(v->mips);
  cudaFree(v->var);
  cudaFree(v->tr);
  cudaFree(v->lut);
  cudaFree(v->d_max);
  cudaFree(v->d_counters);
  if (v->scratch) cudaFree(v->scratch);
  if (v->inter) cudaFree(v->inter);
  if (v->mom) cudaFree(v->mom);
  if (v->env_dev) cudaFree(v->env_dev);
  if (v->copy_stream) {
    cudaStreamSynchronize(v->copy_stream);  // host copies still reading the frames
    for (int i = 0; i < 2; ++i) {
      cudaEventDestroy(v->rendered[i]);
      cudaEventDestroy(v->copied[i]);
    }
    cudaStreamDestroy(v->copy_stream);
  }
  for (int i = 0; i < 2; ++i)
    if (v->frame[i]) cudaFree(v->frame[i]);
  if (v->side_stream) {
    cudaStreamSynchronize(v->side_stream);
    cudaEventDestroy(v->side_fork);
    cudaEventDestroy(v->side_join);
    cudaStreamDestroy(v->side_stream);
  }
  destroy_textures(v);
  delete h;
  return MR_OK;
}

int mr_volume_set_data(mr_volume* h, const float* host_data, size_t count) {
  clear_error();
  if (!h || !host_data) return set_error(MR_ERR_ARG, "mr_volume_set_data: NULL argument");
  Volume* v = &h->v;
  size_t n = (size_t)v->res * v->res * v->res;
  if (count != n) return set_error(MR_ERR_ARG, "mr_volume_set_data: count %zu != res^3 = %zu", count, n);
  MR_CUDA(cudaMemcpy(v->density, host_data, n * sizeof(float), cudaMemcpyHostToDevice));
  v->data_set = true;
  v->gth_den_stale = true;
  v->mips_valid = v->tr_valid = false;
  return MR_OK;
}

int mr_volume_set_data_device(mr_volume* h, const float* dev_data, size_t count, void* stream) {
  clear_error();
  if (!h || !dev_data) return set_error(MR_ERR_ARG, "mr_volume_set_data_device: NULL argument");
  Volume* v = &h->v;
  size_t n = (size_t)v->res * v->res * v->res;
  if (count != n) return set_error(MR_ERR_ARG, "mr_volume_set_data_device: count %zu != res^3 = %zu", count, n);
  MR_CUDA(cudaMemcpyAsync(v->density, dev_data, n * sizeof(float), cudaMemcpyDeviceToDevice, (cudaStream_t)stream));
  v->data_set = true;
  v->gth_den_stale = true;
  v->mips_valid = v->tr_valid = false;
  return MR_OK;
}

int mr_volume_update(mr_volume* h, void* stream) {
  clear_error();
  if (!h) return set_error(MR_ERR_ARG, "mr_volume_update: NULL volume");
  Volume* v = &h->v;
  cudaStream_t s = (cudaStream_t)stream;
  size_t n = (size_t)v->res * v->res * v->res;
  float init = 0.00001f;
  MR_CUDA(cudaMemcpyAsync(v->d_max, &init, sizeof(float), cudaMemcpyHostToDevice, s));
  int blocks = sm_count() * 4;
  k_max_density<<<blocks, 512, 0, s>>>(v->density, n, v->d_max);
  k_mip0<<<grid_for(256u * 256u * 256u, 256), 256, 0, s>>>(v->density, v->res, v->mips);
  MR_CUDA(cudaMemsetAsync(v->var, 0, sizeof(float) * 256 * 256 * 256, s));
  for (int k = 0; k < 8; ++k) {
    int r = 256 >> k;
    size_t nn = (size_t)(r / 2) * (r / 2) * (r / 2);
    k_mip_down<<<grid_for(nn, 256), 256, 0, s>>>(v->mips + mip_offset(k), r, v->mips + mip_offset(k + 1),
                                                 v->var + mip_offset(k + 1));
  }
  MR_CUDA(cudaGetLastError());
  float md = 0;
  MR_CUDA(cudaMemcpyAsync(&md, v->d_max, sizeof(float), cudaMemcpyDeviceToHost, s));
  MR_CUDA(cudaStreamSynchronize(s));
  v->max_density = md;
  v->mips_valid = true;
  v->tex_mips_stale = true;
  v->gth_mips_stale = true;
  v->tr_valid = false;
  return MR_OK;
}

int mr_volume_update_tr(mr_volume* h, mr_float3 light_dir, float alpha, void* stream) {
  clear_error();
  if (!h) return set_error(MR_ERR_ARG, "mr_volume_update_tr: NULL volume");
  Volume* v = &h->v;
  if (!v->mips_valid) return set_error(MR_ERR_STATE, "mr_volume_update_tr before mr_volume_update");
  F3 L = normalize(to_f3(light_dir));
  if (!(dot(L, L) > 0.5f)) return set_error(MR_ERR_ARG, "light direction must be non-zero");
  if (v->tr_valid && L.x == v->tr_light.x && L.y == v->tr_light.y && L.z == v->tr_light.z && alpha == v->tr_alpha)
    return MR_OK;
  return launch_update_tr(v, L, alpha, (cudaStream_t)stream);
}

int mr_volume_update_hglut(mr_volume* h, float g, uint32_t seed, void* stream) {
  clear_error();
  if (!h) return set_error(MR_ERR_ARG, "mr_volume_update_hglut: NULL volume");
  if (!(g > -1.0f && g < 1.0f)) return set_error(MR_ERR_ARG, "g = %f outside (-1, 1)", g);
  Volume* v = &h->v;
  if (v->lut_valid && v->lut_g == g && v->lut_seed == seed) return MR_OK;
  return launch_update_lut(v, g, seed, (cudaStream_t)stream);
}

// SetHDRI (core/volume.cu:1426-1458) from pixels: w x h RGBA fp32, row 0 =
// straight up (v = acos(d.y) / pi), column u = atan2(-d.z, d.x) / 2 pi + 1/2.
int mr_volume_set_hdri(mr_volume* h, const float* host_rgba, int32_t w, int32_t hh) {
  clear_error();
  if (!h || !host_rgba) return set_error(MR_ERR_ARG, "mr_volume_set_hdri: NULL argument");
  if (w <= 0 || hh <= 0 || (long long)w * hh > (1ll << 26)) return set_error(MR_ERR_ARG, "bad HDRI size %d x %d", w, hh);
  Volume* v = &h->v;
  const size_t n = (size_t)w * hh * 4;
  for (size_t i = 0; i < n; ++i)
    if (!std::isfinite(host_rgba[i])) return set_error(MR_ERR_ARG, "HDRI value %zu is not finite", i);
  float4* d = nullptr;
  cudaError_t e = cudaMalloc(&d, n * sizeof(float));
  if (e != cudaSuccess) return set_error(MR_ERR_NOMEM, "HDRI: %s", cudaGetErrorString(e));
  e = cudaMemcpy(d, host_rgba, n * sizeof(float), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    cudaFree(d);
    return cuda_error(e, "cudaMemcpy(HDRI)");
  }
  // renders still queued may read the old map: wait for the device first
  if (v->env_dev) {
    cudaDeviceSynchronize();
    cudaFree(v->env_dev);
  }
  v->env_dev = d;
  v->env_host.assign(host_rgba, host_rgba + n);
  v->env_w = w;
  v->env_h = hh;
  return MR_OK;
}

int mr_volume_clear_hdri(mr_volume* h) {
  clear_error();
  if (!h) return set_error(MR_ERR_ARG, "mr_volume_clear_hdri: NULL argument");
  Volume* v = &h->v;
  if (v->env_dev) {
    cudaDeviceSynchronize();
    cudaFree(v->env_dev);
  }
  v->env_dev = nullptr;
  v->env_host.clear();
  v->env_w = v->env_h = 0;
  return MR_OK;
}

int mr_volume_max_density(const mr_volume* h, float* out) {
  if (!h || !out) return set_error(MR_ERR_ARG, "mr_volume_max_density: NULL argument");
  *out = h->v.max_density;
  return MR_OK;
}

int mr_volume_resolution(const mr_volume* h, int32_t* out) {
  if (!h || !out) return set_error(MR_ERR_ARG, "mr_volume_resolution: NULL argument");
  *out = h->v.res;
  return MR_OK;
}

int mr_volume_read(const mr_volume* h, int32_t what, int32_t level, float* host_out, size_t count) {
  clear_error();
  if (!h || !host_out) return set_error(MR_ERR_ARG, "mr_volume_read: NULL argument");
  const Volume* v = &h->v;
  const float* src = nullptr;
  size_t n = 0;
  switch (what) {
    case MR_READ_DENSITY: src = v->density; n = (size_t)v->res * v->res * v->res; break;
    case MR_READ_MIP:
    case MR_READ_VARIANCE:
      if (level < 0 || level > 8) return set_error(MR_ERR_ARG, "mip level %d outside [0, 8]", level);
      src = (what == MR_READ_MIP ? v->mips : v->var) + mip_offset(level);
      n = (size_t)(256 >> level) * (256 >> level) * (256 >> level);
      break;
    case MR_READ_TR:
      if (level < 0 || level > 7) return set_error(MR_ERR_ARG, "TR level %d outside [0, 7]", level);
      src = v->tr + tr_offset(level);
      n = (size_t)(128 >> level) * (128 >> level) * (128 >> level);
      break;
    case MR_READ_HGLUT: src = v->lut; n = (size_t)kLut * kLut; break;
    default: return set_error(MR_ERR_ARG, "mr_volume_read: unknown table %d", what);
  }
  if (count != n) return set_error(MR_ERR_ARG, "mr_volume_read: count %zu != %zu", count, n);
  MR_CUDA(cudaDeviceSynchronize());
  MR_CUDA(cudaMemcpy(host_out, src, n * sizeof(float), cudaMemcpyDeviceToHost));
  return MR_OK;
}

int mr_volume_set_timing(mr_volume* h, int32_t enable) {
  clear_error();
  if (!h) return set_error(MR_ERR_ARG, "mr_volume_set_timing: NULL volume");
  h->v.timer.on = enable != 0;
  return MR_OK;
}

int mr_volume_stage_times(mr_volume* h, double* host_ms, int32_t* host_launches, int32_t n) {
  clear_error();
  if (!h || !host_ms || !host_launches || n < 1) return set_error(MR_ERR_ARG, "mr_volume_stage_times: bad argument");
  MR_CUDA(cudaDeviceSynchronize());
  for (int st = 0; st < n && st < ST_COUNT; ++st) {
    auto& ev = h->v.timer.ev[st];
    double ms = 0.0;
    int pairs = (int)ev.size() / 2;
    for (int i = 0; i < pairs; ++i) {
      float t = 0.0f;
      cudaEventElapsedTime(&t, ev[2 * i], ev[2 * i + 1]);
      ms += t;
    }
    for (auto e : ev) cudaEventDestroy(e);
    ev.clear();
    host_ms[st] = ms;
    host_launches[st] = pairs;
  }
  return MR_OK;
}

int mr_volume_counters(const mr_volume* h, uint64_t* host_out4) {
  clear_error();
  if (!h || !host_out4) return set_error(MR_ERR_ARG, "mr_volume_counters: NULL argument");
  unsigned long long c[kCounters];
  MR_CUDA(cudaMemcpy(c, h->v.d_counters, sizeof(c), cudaMemcpyDeviceToHost));
  for (int i = 0; i < 4; ++i) host_out4[i] = c[i];
  return MR_OK;
}

}  // extern "C"
