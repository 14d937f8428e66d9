// Delta-tracking path tracer (render type PT): a persistent kernel whose
// threads claim (pixel, sample) work items from a global queue with
// warp-aggregated atomics and start a new path as soon as theirs ends, so that
// lanes stay busy however long individual paths run. Replaces the
// one-launch-per-spp RenderCamera<false> loop of core/volume.cu:147-179,415-459.
#include <algorithm>
#include <cmath>

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

// Per-pixel sums of one finished path's radiance (clamped at 0).
__device__ __forceinline__ void add_path(const DTArgs& a, unsigned pix, F3 L) {
  L = vmax(L, f3(0, 0, 0));
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

// CalculateRadiance regenerated per bounce: each iteration of the loop is one
// bounce (free flight to the next vertex, then NEE towards the light) of
// every lane's path, and a lane whose path ended takes its next work item at
// the top of the next iteration instead of idling until the warp's longest
// path ends. Path lengths are heavy-tailed (up to max_bounces vertices in an
// optically thick medium against none for a ray that misses the volume), so
// whole-path lockstep leaves most lanes idle. A path draws the same random
// numbers in the same order as path_radiance, so its radiance is the same.
__global__ void __launch_bounds__(128) k_delta_track(DTArgs a) {
  TrackStats st{0, 0};
  unsigned paths = 0;
  const unsigned long long P = (unsigned long long)a.cam.width * a.cam.height;
  Rng rng;
  F3 pos = f3(0, 0, 0), rd = f3(0, 0, 0), rate = f3(0, 0, 0), res = f3(0, 0, 0);
  unsigned pix = 0;
  int bounce = 0;
  bool live = false, done = false;
  for (;;) {
    // lanes without a path claim work items until one enters the volume
    while (!live) {
      unsigned long long w = claim_work(a.queue);
      if (w >= a.total) { done = true; break; }
      // sample-major order: concurrently traced paths are neighbouring pixels.
      unsigned s = (unsigned)(w / P);
      pix = (unsigned)(w - (unsigned long long)s * P);
      int row = pix / a.cam.width, col = pix - row * a.cam.width;
      rng.init(a.seed, pix, a.sample_offset + s, TAG_PT);
      float jx = rng.next(), jy = rng.next();
      F3 dir = normalize(camera_dir(a.cam, row, col, jx, jy));
      float dis = ray_box_offset(a.cam.ori, dir);
      ++paths;
      if (dis < 0) { add_path(a, pix, sky(a.sc, dir)); continue; }
      if (a.sc.max_bounces <= 0) { add_path(a, pix, f3(0, 0, 0)); continue; }
      pos = a.cam.ori + dir * dis;
      rd = dir;
      rate = f3(1, 1, 1);
      res = f3(0, 0, 0);
      bounce = 0;
      live = true;
    }
    if (done) break;
    // one bounce (the body of CalculateRadiance's loop, core/render.cuh:219-254)
    F3 np, nd;
    float maxd = ray_box_distance(pos, rd);
    if (!next_vertex(a.m, rng, a.sc.alpha, a.sc.g, pos, rd, maxd, np, nd, st)) {
      res = res + sky(a.sc, rd) * rate;
      add_path(a, pix, res);
      live = false;
      continue;
    }
    pos = np;
    rate = rate * a.sc.scatter;
    maxd = ray_box_distance(pos, a.sc.L);
    float ph = hg_phase(dot(rd, a.sc.L), a.sc.g);
    res = res + (a.sc.light_color * rate) * (transmittance(a.m, rng, pos, a.sc.L, maxd, a.sc.alpha, st) * ph);
    rd = nd;
    if (++bounce >= a.sc.max_bounces) {
      add_path(a, pix, res);
      live = false;
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
  sc.env_map = nullptr;
  sc.env_w = sc.env_h = 0;
  return sc;
}

void attach_env(PathScene& sc, const Volume* v) {
  sc.env_map = v->env_dev;
  sc.env_w = v->env_w;
  sc.env_h = v->env_h;
}

// Image_host::Sample (core/volume.hpp:22-42): bilinear with clamped texel
// indices at pos = uv * size - 1/2.
static F3 env_sample_host(const Volume* v, float u, float vv) {
  const int w = v->env_w, h = v->env_h;
  auto at = [&](int x, int y) {
    x = std::min(std::max(x, 0), w - 1);
    y = std::min(std::max(y, 0), h - 1);
    const float* q = &v->env_host[((size_t)y * w + x) * 4];
    return f3(q[0], q[1], q[2]);
  };
  const float px = u * (float)w - 0.5f, py = vv * (float)h - 0.5f;
  const int x = (int)std::floor(px), y = (int)std::floor(py);
  const float wx = px - (float)x, wy = py - (float)y;
  auto lerp3 = [](F3 a, F3 b, float t) { return a * (1.0f - t) + b * t; };
  return lerp3(lerp3(at(x, y), at(x + 1, y), wx), lerp3(at(x, y + 1), at(x + 1, y + 1), wx), wy);
}

// One light per neural pass (core/volume.cu:417-432): with probability
// rate = 4e / (4e + max(light colour)), e the environment scale, the light
// comes from the map: direction = the uniform sphere point of the R2
// sequence (Roberts2, core/vector.cu:174-178) at the pass index, colour =
// map(direction) * env * 4 / rate; otherwise the directional light with
// colour / (1 - rate). The coin is Philox (seed; pass, 0, 0, TAG_ENV) where
// the reference calls rand().
void select_env_light(const Volume* v, mr_render_params* q) {
  if (!v->env_dev || v->env_host.empty()) return;
  const F3 env = to_f3(q->env_color), lc = to_f3(q->light_color);
  const float e = std::max(env.x, std::max(env.y, env.z));
  const float m = std::max(lc.x, std::max(lc.y, lc.z));
  if (!(e > 0.0f)) return;
  const float rate = e * 4.0f / (e * 4.0f + m);
  uint32_t o[4];
  philox4x32_10(q->sample_offset, 0u, 0u, TAG_ENV, q->seed, 0u, o);
  if (u01(o[0]) < rate) {
    const float g = 1.32471795724474602596f;
    const float ax = 1.0f / g, ay = 1.0f / (g * g);
    const float n = (float)q->sample_offset;
    float rx = ax * n + 0.5f, ry = ay * n + 0.5f;
    rx -= std::floor(rx);
    ry -= std::floor(ry);
    const F3 d = uniform_sphere(rx, ry);
    const float u = std::atan2(-d.z, d.x) * (float)(0.5 / 3.1415926) + 0.5f;
    const float vv = std::acos(std::max(std::min(d.y, 1.0f), -1.0f)) * (float)(1.0 / 3.1415926);
    const F3 c = env_sample_host(v, u, vv);
    const float k = 4.0f / rate;
    q->light_dir = mr_float3{d.x, d.y, d.z};
    q->light_color = mr_float3{c.x * env.x * k, c.y * env.y * k, c.z * env.z * k};
  } else {
    const float k = 1.0f / (1.0f - rate);
    q->light_color = mr_float3{lc.x * k, lc.y * k, lc.z * k};
  }
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
  attach_env(a.sc, v);
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
