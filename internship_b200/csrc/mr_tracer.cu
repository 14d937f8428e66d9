// Delta-tracking path tracer (render type PT): a persistent kernel whose
// threads claim (pixel, sample) work items from a global queue with
// warp-aggregated atomics and start a new path as soon as theirs ends, so that
// lanes stay busy however long individual paths run. Replaces the
// one-launch-per-spp RenderCamera<false> loop of core/volume.cu:147-179,415-459.
#include "mr_internal.h"
#include "mr_track.cuh"

namespace mr {

struct DTArgs {
  Medium m;
  PathScene sc;
  CameraModel cam;
  uint32_t seed, sample_offset;
  int spp;
  unsigned long long total;         // W*H*spp
  unsigned long long* queue;        // work counter (zeroed before launch)
  unsigned long long* counters;     // [0] fetches, [1] paths, [2] loop caps
  float* sum32;                     // W*H*3 (nullable)
  double* sum64;                    // W*H*3 (nullable)
  double* sumsq64;                  // W*H*3 (nullable)
};

__global__ void __launch_bounds__(128) k_delta_track(DTArgs a) {
  TrackStats st{0, 0};
  unsigned paths = 0;
  const unsigned long long P = (unsigned long long)a.cam.width * a.cam.height;
  for (;;) {
    unsigned long long w = claim_work(a.queue);
    if (w >= a.total) break;
    // sample-major order: concurrently traced paths are neighbouring pixels.
    unsigned s = (unsigned)(w / P);
    unsigned pix = (unsigned)(w - (unsigned long long)s * P);
    int row = pix / a.cam.width, col = pix - row * a.cam.width;
    Rng rng;
    rng.init(a.seed, pix, a.sample_offset + s, TAG_PT);
    float jx = rng.next(), jy = rng.next();
    F3 dir = camera_dir(a.cam, row, col, jx, jy);
    float t;
    F3 L = path_radiance(a.m, a.sc, rng, a.cam.ori, dir, &t, st);
    L = vmax(L, f3(0, 0, 0));
    ++paths;
    size_t o = (size_t)pix * 3;
    if (a.sum32) {
      atomicAdd(a.sum32 + o, L.x);
      atomicAdd(a.sum32 + o + 1, L.y);
      atomicAdd(a.sum32 + o + 2, L.z);
    }
    if (a.sum64) {
      atomicAdd(a.sum64 + o, (double)L.x);
      atomicAdd(a.sum64 + o + 1, (double)L.y);
      atomicAdd(a.sum64 + o + 2, (double)L.z);
    }
    if (a.sumsq64) {
      atomicAdd(a.sumsq64 + o, (double)L.x * L.x);
      atomicAdd(a.sumsq64 + o + 1, (double)L.y * L.y);
      atomicAdd(a.sumsq64 + o + 2, (double)L.z * L.z);
    }
  }
  // one atomic per warp for the statistics
  unsigned f = st.fetches, c = st.caps, p = paths;
  for (int o = 16; o; o >>= 1) {
    f += __shfl_xor_sync(0xffffffffu, f, o);
    c += __shfl_xor_sync(0xffffffffu, c, o);
    p += __shfl_xor_sync(0xffffffffu, p, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(a.counters + 0, (unsigned long long)f);
    atomicAdd(a.counters + 1, (unsigned long long)p);
    if (c) atomicAdd(a.counters + 2, (unsigned long long)c);
  }
}

__global__ void k_scale(float* x, size_t n, float s) {
  size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i < n) x[i] *= s;
}

// SM count of the current device.
int sm_count() {
  static DeviceCache cache;
  return cache.get([] {
    int dev = 0, n = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    return n > 0 ? n : 1;
  });
}

// Resident grid of the delta tracker on the current device.
static int dt_grid() {
  static DeviceCache cache;
  return cache.get([] {
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_delta_track, 128, 0);
    if (per_sm <= 0) per_sm = 1;
    return per_sm * sm_count();
  });
}

CameraModel make_camera(const mr_render_params* p) {
  CameraModel c;
  c.ori = to_f3(p->ori);
  c.fwd = normalize(-c.ori);
  c.up = to_f3(p->up);
  c.right = to_f3(p->right);
  c.width = p->width;
  c.height = p->height;
  return c;
}

PathScene make_path_scene(const mr_render_params* p) {
  PathScene sc;
  sc.L = normalize(to_f3(p->light_dir));
  sc.light_color = to_f3(p->light_color);
  sc.scatter = to_f3(p->scatter_rate);
  sc.env = to_f3(p->env_color);
  sc.alpha = p->alpha;
  sc.g = p->g;
  sc.max_bounces = p->max_bounces;
  return sc;
}

int check_params(const mr_render_params* p) {
  if (!p) return set_error(MR_ERR_ARG, "render params are NULL");
  if (p->width <= 0 || p->height <= 0 || (long long)p->width * p->height > (1ll << 28))
    return set_error(MR_ERR_ARG, "image size %dx%d invalid", p->width, p->height);
  if (p->spp <= 0) return set_error(MR_ERR_ARG, "spp must be positive (got %d)", p->spp);
  if (p->max_bounces < 0) return set_error(MR_ERR_ARG, "max_bounces must be >= 0");
  if (!(p->alpha > 0.0f)) return set_error(MR_ERR_ARG, "alpha must be > 0");
  if (!(p->g > -1.0f && p->g < 1.0f)) return set_error(MR_ERR_ARG, "g = %f outside (-1, 1)", p->g);
  F3 L = to_f3(p->light_dir);
  if (!(dot(L, L) > 0.0f)) return set_error(MR_ERR_ARG, "light direction must be non-zero");
  F3 o = to_f3(p->ori);
  if (!(dot(o, o) > 0.0f)) return set_error(MR_ERR_ARG, "camera position must not be the volume centre");
  return MR_OK;
}

// Launch the tracer; exactly one of sum32 / sum64 is non-null.
int launch_delta_track(Volume* v, const mr_render_params* p, float* sum32, double* sum64, double* sumsq64,
                       cudaStream_t s) {
  if (!v->data_set) return set_error(MR_ERR_STATE, "render before mr_volume_set_data");
  if (!v->mips_valid) return set_error(MR_ERR_STATE, "render before mr_volume_update");
  DTArgs a;
  a.m = Medium{v->density, v->res, v->max_density, p->tr_scale, 0};
  {
    int rc = density_gather_texture(v, s, &a.m.tex);
    if (rc) return rc;
  }
  a.sc = make_path_scene(p);
  a.cam = make_camera(p);
  a.seed = p->seed;
  a.sample_offset = p->sample_offset;
  a.spp = p->spp;
  a.total = (unsigned long long)p->width * p->height * p->spp;
  a.queue = v->d_counters + 4;
  a.counters = v->d_counters;
  a.sum32 = sum32;
  a.sum64 = sum64;
  a.sumsq64 = sumsq64;
  MR_CUDA(cudaMemsetAsync(v->d_counters, 0, kCounters * sizeof(unsigned long long), s));
  v->timer.mark(ST_PT, s);
  k_delta_track<<<dt_grid(), 128, 0, s>>>(a);
  v->timer.mark(ST_PT, s);
  MR_CUDA(cudaGetLastError());
  return MR_OK;
}

int render_pt(Volume* v, const mr_render_params* p, float* dev_rgb, cudaStream_t s) {
  size_t n = (size_t)p->width * p->height * 3;
  MR_CUDA(cudaMemsetAsync(dev_rgb, 0, n * sizeof(float), s));
  int rc = launch_delta_track(v, p, dev_rgb, nullptr, nullptr, s);
  if (rc) return rc;
  k_scale<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(dev_rgb, n, 1.0f / (float)p->spp);
  MR_CUDA(cudaGetLastError());
  return MR_OK;
}

}  // namespace mr

using namespace mr;

extern "C" int mr_render_accumulate_f64(mr_volume* h, const mr_render_params* p, double* dev_sum,
                                        double* dev_sumsq, void* stream) {
  clear_error();
  if (!h || !dev_sum) return set_error(MR_ERR_ARG, "mr_render_accumulate_f64: NULL argument");
  int rc = check_params(p);
  if (rc) return rc;
  return launch_delta_track(&h->v, p, nullptr, dev_sum, dev_sumsq, (cudaStream_t)stream);
}
