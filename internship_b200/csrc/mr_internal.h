// Host-side internals shared by the library's translation units.
#pragma once
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/mrpnn_b200.h"
#include "../../include/mrpnn_weights.h"
#include "mr_device.cuh"

namespace mr {

// Counters kept per volume on the device ([0] density fetches, [1] paths,
// [2] loop-cap hits, [3] active neural pixels, [4..7] scratch).
constexpr int kCounters = 8;

// Optional per-stage CUDA-event timing (mr_volume_set_timing).
enum Stage {
  ST_PT = 0, ST_NN_TRACE = 1, ST_NN_PREDICT = 2, ST_TR = 3, ST_LUT = 4, ST_MIPS = 5, ST_NN_MLP = 6,
  ST_NN_TRUNK = 7,  // the fp32 network's main-trunk kernel alone (inside ST_NN_MLP)
  ST_COUNT = 8
};
struct StageTimer {
  bool on = false;
  std::vector<cudaEvent_t> ev[ST_COUNT];  // begin/end pairs
  void mark(int st, cudaStream_t s) {
    if (!on) return;
    cudaEvent_t e;
    if (cudaEventCreate(&e) != cudaSuccess) return;
    cudaEventRecord(e, s);
    ev[st].push_back(e);
  }
};

struct Volume {
  int res = 0;
  int device = 0;
  float* density = nullptr;  // res^3
  float* mips = nullptr;     // kMipTotal
  float* var = nullptr;      // kMipTotal
  float* tr = nullptr;       // kTrTotal
  float* lut = nullptr;      // 512 x 512
  float* d_max = nullptr;    // device majorant (one float)
  unsigned long long* d_counters = nullptr;
  float max_density = 0.00001f;
  bool data_set = false;
  bool mips_valid = false;
  bool tr_valid = false;
  F3 tr_light{0, 0, 0};
  float tr_alpha = 0;
  bool lut_valid = false;
  float lut_g = 0;
  uint32_t lut_seed = 0;
  StageTimer timer;
  // Texture-unit copies of the tables for MR_SAMPLER_TEXTURE, created on first
  // use and refreshed when the linear tables change.
  cudaArray_t mip_arr[9] = {}, tr_arr[8] = {}, lut_arr = nullptr;
  cudaTextureObject_t mip_tex[9] = {}, tr_tex[8] = {}, lut_tex = 0;
  bool tex_mips_stale = true, tex_tr_stale = true, tex_lut_stale = true;
  // Layered copies of the same tables (layer = x) read by the exact sampler
  // through texture gathers, which return a 2 x 2 texel footprint unfiltered;
  // created on first use, refreshed when the linear tables change.
  cudaArray_t gth_mip_arr[9] = {}, gth_tr_arr[8] = {}, gth_lut_arr = nullptr;
  cudaTextureObject_t gth_mip_tex[9] = {}, gth_tr_tex[8] = {}, gth_lut_tex = 0;
  bool gth_mips_stale = true, gth_tr_stale = true, gth_lut_stale = true;
  // layered copy of the density grid for the trackers' texture gathers
  cudaArray_t gth_den_arr = nullptr;
  cudaTextureObject_t gth_den_tex = 0;
  bool gth_den_stale = true;
  // Per-render scratch owned by the volume (grown on demand).
  void* scratch = nullptr;
  size_t scratch_bytes = 0;
  // Interactive neural mode: radiance and first-hit distance of the frame.
  void* inter = nullptr;
  size_t inter_bytes = 0;
  // Environment map (SetHDRI): w x h RGBA fp32, row 0 = straight up, on the
  // device for the trackers' escaped rays and on the host for the neural
  // render's light selection.
  float4* env_dev = nullptr;
  std::vector<float> env_host;
  int env_w = 0, env_h = 0;
  // SetSurfaceIOR: index of refraction of the marching form's surface
  // (negative: no surface, the reference's default -1).
  float surface_ior = -1.0f;
  // Interactive delta tracking: FP64 per-pixel sums of the radiance (3), of
  // the histogram luminance l and of l^2, SoA (sum k of pixel p at
  // mom[k * mom_npx + p]), for the histogram buffer mom_hist they belong to.
  double* mom = nullptr;
  size_t mom_bytes = 0, mom_npx = 0;
  const void* mom_hist = nullptr;
  // Pipelined host delivery (mr_render_host_async): two device frames used in
  // turn, a copy stream, and per frame the events "rendered" (on the caller's
  // stream) and "copied" (on the copy stream).
  float* frame[2] = {};
  size_t frame_bytes = 0;
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t rendered[2] = {}, copied[2] = {};
  long long frame_seq = 0;  // frames issued so far; frame t uses frame[t % 2]
  // Side stream of a neural render (the per-point table beside the trace),
  // forked from and joined back to the caller's stream by events.
  cudaStream_t side_stream = nullptr;
  cudaEvent_t side_fork = nullptr, side_join = nullptr;
};

struct Network {
  float* w = nullptr;        // MR_WEIGHT_TOTAL fp32, blob layout
  float* stencil = nullptr;  // 160 x 3
  void* packed = nullptr;    // tensor-core operand images (bf16/fp8), see mr_mlp_tc.cu
  size_t packed_bytes = 0;
  std::vector<float> h_rowwise;  // fp32 per-row weights passed as kernel parameters (mr_mlp_tc.cu)
  std::vector<float> h_winv8;    // inverse per-layer scales of the E4M3 weight image
  std::vector<float> h_se;       // per-block squeeze-excitation records of the tensor-core trunk (mr_mlp_tc.cu)
  float* simt_img = nullptr;     // weight image of the fp32 network kernels (simt_weight_image)
  std::vector<float> h_tail;     // LXW .. LX12B, kernel parameters of the fp32 head's tail (mr_mlp_simt.cu)
  std::vector<float> h_light;    // kernel parameters of the fp32 light-direction trunk (mr_mlp_simt.cu)
  float h_stencil[MR_STENCIL_POINTS * 3];
};

// Output of one job of a batched neural render: its image, light colour and
// per-channel albedo (the network kernels' compose step reads them per row).
struct BatchOut {
  float* out;
  F3 light_color, scatter;
};

// A value that belongs to one device (an SM count, an occupancy, whether a
// kernel attribute was set there), computed the first time a thread asks for
// it with that device current and kept for the process. Safe to use from
// several threads and devices at once.
constexpr int kMaxDevices = 64;
struct DeviceCache {
  std::mutex mu;
  int value[kMaxDevices] = {};
  bool ready[kMaxDevices] = {};
  // f() -> int, evaluated under the lock on the first call per device.
  template <class F>
  int get(F&& f) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return f();
    std::lock_guard<std::mutex> lock(mu);
    if (!ready[dev]) {
      value[dev] = f();
      ready[dev] = true;
    }
    return value[dev];
  }
  // f() -> mr_status, run once per device; only a success is kept, so a
  // failed first attempt is retried by the next call.
  template <class F>
  int once(F&& f) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= kMaxDevices) return f();
    std::lock_guard<std::mutex> lock(mu);
    if (ready[dev]) return 0;
    int rc = f();
    if (rc == 0) ready[dev] = true;
    return rc;
  }
};

// Error reporting: thread-local message, returns the code.
int set_error(int code, const char* fmt, ...);
int cuda_error(cudaError_t e, const char* what);
void clear_error();

#define MR_CUDA(call)                                   \
  do {                                                  \
    cudaError_t e_ = (call);                            \
    if (e_ != cudaSuccess) return ::mr::cuda_error(e_, #call); \
  } while (0)

inline F3 to_f3(const mr_float3& a) { return F3{a.x, a.y, a.z}; }

// Grows v->scratch to at least `bytes` (stream-ordered free of the old block).
int ensure_scratch(Volume* v, size_t bytes, cudaStream_t s);

// Kernels launched from several translation units.
int launch_update_tr(Volume* v, F3 L, float alpha, cudaStream_t s);
int launch_update_lut(Volume* v, float g, uint32_t seed, cudaStream_t s);
int refresh_textures(Volume* v, cudaStream_t s);
int refresh_gather_textures(Volume* v, cudaStream_t s);
// Texture object of the density grid's layered copy (created on first use,
// refreshed after mr_volume_set_data*).
int density_gather_texture(Volume* v, cudaStream_t s, cudaTextureObject_t* out);
// r^3 x-major fp32 table <-> cudaArray (3-D or layered, extent z, y, x)
int copy_to_array(cudaArray_t arr, const float* src, int r, cudaStream_t s);
int make_gather_tex(cudaArray_t* arr, cudaTextureObject_t* tex, int r, cudaTextureAddressMode mode);
void destroy_textures(Volume* v);
int sm_count();
// Points a scene's escaped-ray lookup at the volume's environment map (if any).
struct PathScene;
void attach_env(PathScene& sc, const Volume* v);
// The neural render's light for this pass when the volume has an environment
// map (the env / light choice of core/volume.cu:417-432): q's light_dir and
// light_color are replaced in place.
void select_env_light(const Volume* v, mr_render_params* q);

}  // namespace mr

struct mr_volume { mr::Volume v; };
struct mr_network { mr::Network n; };
