// Compatibility shim that lets the reference's device code compile with
// CUDA 12 (test infrastructure only).
//
// CUDA 12 removed the legacy texture- and surface-reference APIs the
// reference uses (`texture<T, dim, mode>` / `surface<void, dim>` globals read
// with tex2D/tex3D and written with surf2Dwrite/surf3Dwrite, bound with
// cudaBindTextureToArray / cudaBindSurfaceToArray, e.g.
// core/renderResources.cuh:20-58, core/volume.cu:1081,1318-1345) and the
// float overload of saturate(). This header, force-included ahead of the
// reference's own headers, turns every `texture<...>` declaration into a
// __device__ holder of a cudaTextureObject_t (plus the host-side sampler
// fields the reference sets before binding) and every `surface<...>` into a
// holder of a cudaSurfaceObject_t. The bind calls create the object from the
// array with the holder's settings and copy it into the device holder, so
// the reference's own host code (VolumeRender::Update, Update_TR,
// UpdateHGLut) binds its tables as it did with the legacy API. Harnesses may
// also fill the holders directly.
#pragma once
#include <cuda_runtime.h>
#include <math_functions.h>
#include <device_functions.h>
#include <curand_kernel.h>
#include <cuda_texture_types.h>
#include <texture_fetch_functions.h>
#include <surface_functions.h>

template <class T, int dim = 1, enum cudaTextureReadMode mode = cudaReadModeElementType>
struct legacy_texref {
  cudaTextureObject_t obj;
  // sampler settings of the legacy reference (host side only)
  int normalized;
  cudaTextureFilterMode filterMode;
  cudaTextureAddressMode addressMode[3];
};
template <class T, int dim = 1>
struct legacy_surfref {
  cudaSurfaceObject_t obj;
};

template <class T, class R>
__device__ T tex3D(const R& r, float x, float y, float z) { return tex3D<T>(r.obj, x, y, z); }
#ifdef MR_REF_INJECT
// Injection build (ref_inject.cu): 2-D table reads return injected values.
__device__ float inj_hglut(float u, float v);
template <class T, class R>
__device__ T tex2D(const R& r, float x, float y) { return (T)inj_hglut(x, y); }
#else
template <class T, class R>
__device__ T tex2D(const R& r, float x, float y) { return tex2D<T>(r.obj, x, y); }
#endif
template <class T, int dim>
__device__ void surf2Dwrite(T v, const legacy_surfref<void, dim>& r, int x, int y) { surf2Dwrite<T>(v, r.obj, x, y); }
template <class T, int dim>
__device__ void surf3Dwrite(T v, const legacy_surfref<void, dim>& r, int x, int y, int z) {
  surf3Dwrite<T>(v, r.obj, x, y, z);
}
__device__ inline float saturate(float x) { return __saturatef(x); }

// cudaBindTextureToArray(texref, array[, desc]): a texture object over the
// array with the holder's sampler settings, copied into the device holder.
template <class T, int dim, enum cudaTextureReadMode mode, class... Rest>
cudaError_t cudaBindTextureToArray(legacy_texref<T, dim, mode>& r, cudaArray_const_t arr, Rest...) {
  cudaResourceDesc rd = {};
  rd.resType = cudaResourceTypeArray;
  rd.res.array.array = (cudaArray_t)arr;
  cudaTextureDesc td = {};
  for (int i = 0; i < 3; ++i) td.addressMode[i] = r.addressMode[i];
  td.filterMode = r.filterMode;
  td.readMode = mode;
  td.normalizedCoords = r.normalized;
  legacy_texref<T, dim, mode> h = r;
  cudaError_t e = cudaCreateTextureObject(&h.obj, &rd, &td, nullptr);
  if (e != cudaSuccess) return e;
  r.obj = h.obj;
  return cudaMemcpyToSymbol(r, &h, sizeof(h));
}
// cudaBindSurfaceToArray(surfref, array): a surface object over the array.
template <int dim, class... Rest>
cudaError_t cudaBindSurfaceToArray(legacy_surfref<void, dim>& r, cudaArray_const_t arr, Rest...) {
  cudaResourceDesc rd = {};
  rd.resType = cudaResourceTypeArray;
  rd.res.array.array = (cudaArray_t)arr;
  legacy_surfref<void, dim> h = r;
  cudaError_t e = cudaCreateSurfaceObject(&h.obj, &rd);
  if (e != cudaSuccess) return e;
  r.obj = h.obj;
  return cudaMemcpyToSymbol(r, &h, sizeof(h));
}

#define texture __device__ legacy_texref
#define surface __device__ legacy_surfref
