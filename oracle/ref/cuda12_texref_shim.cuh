// Compatibility shim that lets the reference's device code compile with
// CUDA 12 (test infrastructure only).
//
// CUDA 12 removed the legacy texture-reference API the reference uses
// (`texture<T, dim, mode>` globals read with tex2D/tex3D, e.g.
// core/renderResources.cuh:20-58) and the float overload of saturate().
// This header, force-included ahead of the reference's own headers, turns
// every `texture<...>` declaration into a __device__ holder of a
// cudaTextureObject_t, and routes tex2D/tex3D on such a holder to the
// texture-object intrinsics. The harness fills the holders with texture
// objects created with the reference's sampler settings.
#pragma once
#include <cuda_runtime.h>
#include <math_functions.h>
#include <device_functions.h>
#include <curand_kernel.h>
#include <cuda_texture_types.h>
#include <texture_fetch_functions.h>

template <class T, int dim = 1, enum cudaTextureReadMode mode = cudaReadModeElementType>
struct legacy_texref {
  cudaTextureObject_t obj;
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
__device__ inline float saturate(float x) { return __saturatef(x); }
#define texture __device__ legacy_texref
