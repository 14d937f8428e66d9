// C ABI glue: error state, version, network objects, render dispatch and the
// watchdog wait.
#include <chrono>
#include <cstring>
#include <cmath>
#include <thread>

#include "mr_internal.h"
#include "mr_net_layout.cuh"

namespace mr {

static thread_local std::string t_error;

int set_error(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  t_error = buf;
  return code;
}
int cuda_error(cudaError_t e, const char* what) {
  return set_error(MR_ERR_CUDA, "%s failed: %s", what, cudaGetErrorString(e));
}
void clear_error() { t_error.clear(); }

int render_pt(Volume* v, const mr_render_params* p, float* dev_rgb, cudaStream_t s);
int render_neural(Volume* v, const Network* net, const mr_render_params* p, float* dev_rgb, cudaStream_t s);
int render_marching(Volume* v, const Network* net, const mr_render_params* p, float* dev_rgb, cudaStream_t s);
int check_params(const mr_render_params* p);
int pack_network(Network* n);
void free_packed(Network* n);

// Default stencil: the reference's 160 directions (core/vector.cu:77-172),
// the points the reference network's weights were trained on.
#include "mr_ref_stencil.inc"
static void builtin_stencil(float* out) { std::memcpy(out, kRefStencil, sizeof(kRefStencil)); }

// Spiral stencil (opt-in, mr_spiral_stencil): 160 directions in the
// reference's shell layout (shells of 8, 8, 16, 16, 16 unit points, the
// first point of shell 0 at the centre, then three shells of 32 points inside
// the unit ball). Shells 0-4 are golden-angle spirals about rotated axes,
// shells 5-7 spirals with radii cbrt of a stratified sequence.
static void spiral_stencil(float* out) {
  const double ga = 2.39996322972865332;  // golden angle
  int k = 0;
  auto put = [&](double x, double y, double z) { out[3 * k] = (float)x; out[3 * k + 1] = (float)y; out[3 * k + 2] = (float)z; ++k; };
  // axis rotations per shell (fixed Euler angles)
  const double eul[8][3] = {{0, 0, 0}, {0.0, 1.5707963, 0.0}, {1.5707963, 0, 0}, {0.61, 1.13, 0.37},
                            {2.05, 0.41, 1.77}, {0.93, 2.21, 0.18}, {1.49, 0.73, 2.61}, {2.71, 1.87, 0.95}};
  const int sizes[8] = {8, 8, 16, 16, 16, 32, 32, 32};
  for (int sh = 0; sh < 8; ++sh) {
    double a = eul[sh][0], b = eul[sh][1], c = eul[sh][2];
    double ca = std::cos(a), sa = std::sin(a), cb = std::cos(b), sb = std::sin(b), cc = std::cos(c), sc = std::sin(c);
    double R[3][3] = {{ca * cb, ca * sb * sc - sa * cc, ca * sb * cc + sa * sc},
                      {sa * cb, sa * sb * sc + ca * cc, sa * sb * cc - ca * sc},
                      {-sb, cb * sc, cb * cc}};
    int n = sizes[sh];
    int start = (sh == 0) ? 1 : 0;
    if (sh == 0) put(0, 0, 0);
    int m = n - start;
    for (int i = 0; i < m; ++i) {
      double h = (m == 1) ? 0.0 : 1.0 - 2.0 * i / (m - 1);
      double r = std::sqrt(std::max(0.0, 1.0 - h * h));
      double th = ga * i;
      double p[3] = {h, r * std::cos(th), r * std::sin(th)};
      double rad = 1.0;
      if (sh >= 5) rad = std::cbrt((i + 0.5) / m * 0.85 + 0.15);
      double q[3];
      for (int d = 0; d < 3; ++d) q[d] = (R[d][0] * p[0] + R[d][1] * p[1] + R[d][2] * p[2]) * rad;
      put(q[0], q[1], q[2]);
    }
  }
}

}  // namespace mr

using namespace mr;

extern "C" {

int mr_volume_set_surface_ior(mr_volume* h, float ior) {
  clear_error();
  if (!h) return set_error(MR_ERR_ARG, "mr_volume_set_surface_ior: NULL argument");
  if (!std::isfinite(ior)) return set_error(MR_ERR_ARG, "IOR is not finite");
  h->v.surface_ior = ior;
  return MR_OK;
}

const char* mr_version(void) { return "mrpnn-b200 0.1.0 (sm_100a)"; }
const char* mr_last_error(void) { return t_error.c_str(); }

int mr_builtin_stencil(float* host_out, size_t count) {
  clear_error();
  if (!host_out || count != MR_STENCIL_POINTS * 3) return set_error(MR_ERR_ARG, "stencil needs 480 floats");
  builtin_stencil(host_out);
  return MR_OK;
}

int mr_spiral_stencil(float* host_out, size_t count) {
  clear_error();
  if (!host_out || count != MR_STENCIL_POINTS * 3) return set_error(MR_ERR_ARG, "stencil needs 480 floats");
  spiral_stencil(host_out);
  return MR_OK;
}

// Xavier-uniform weights (limit sqrt(6/(fan_in+fan_out))), zero biases, from
// Philox(seed; array index, element block, 0, TAG_MISC).
int mr_weights_xavier(uint32_t seed, float* host_out, size_t count) {
  clear_error();
  if (!host_out || count != MR_WEIGHT_TOTAL) return set_error(MR_ERR_ARG, "weights need %d floats", MR_WEIGHT_TOTAL);
  struct Shape { int in, out; };
  auto shape = [](const char* name, int n) -> Shape {
    std::string s(name);
    if (s == "LSEFin1W") return {75, 16};
    if (s == "LSEFin2W") return {16, 6};
    if (s == "LGGSW") return {3, 8};
    if (s == "LC1W") return {128, 64};
    if (s == "LC2W") return {64, 32};
    if (s == "LXW") return {32, 16};
    if (s == "LX12W") return {16, 1};
    if (s.size() > 4 && s.substr(s.size() - 2) == "2W" && n == 24) return {8, 3};  // SE second layer
    int k = (int)std::lround(std::sqrt((double)n));
    return {k, k};
  };
  int idx = 0;
  size_t off = 0;
#define MR_XAV(name, n)                                                                     \
  {                                                                                         \
    const char* nm = #name;                                                                 \
    bool bias = nm[std::strlen(nm) - 1] == 'B';                                             \
    Shape sh = shape(nm, (n));                                                              \
    float lim = bias ? 0.0f : (float)std::sqrt(6.0 / (double)(sh.in + sh.out));             \
    for (int e = 0; e < (n); ++e) {                                                         \
      uint32_t o[4];                                                                        \
      philox4x32_10((uint32_t)idx, (uint32_t)(e >> 2), 0u, TAG_MISC, seed, 0u, o);          \
      float u = u01(o[e & 3]);                                                              \
      host_out[off + e] = bias ? 0.0f : (2.0f * u - 1.0f) * lim;                            \
    }                                                                                       \
    off += (n);                                                                             \
    ++idx;                                                                                  \
  }
  MR_WEIGHT_LIST(MR_XAV)
#undef MR_XAV
  return MR_OK;
}

int mr_network_create(const float* host_weights, size_t count, const float* stencil_xyz, mr_network** out) {
  clear_error();
  if (!out) return set_error(MR_ERR_ARG, "mr_network_create: out is NULL");
  *out = nullptr;
  if (!host_weights) return set_error(MR_ERR_ARG, "mr_network_create: weights are NULL");
  if (count != MR_WEIGHT_TOTAL)
    return set_error(MR_ERR_ARG, "weight blob has %zu floats, expected %d", count, MR_WEIGHT_TOTAL);
  for (size_t i = 0; i < count; ++i)
    if (!std::isfinite(host_weights[i])) return set_error(MR_ERR_ARG, "weight %zu is not finite", i);
  mr_network* h = new mr_network();
  Network* n = &h->n;
  if (stencil_xyz) std::memcpy(n->h_stencil, stencil_xyz, sizeof(n->h_stencil));
  else builtin_stencil(n->h_stencil);
  cudaError_t e = cudaMalloc(&n->w, MR_WEIGHT_TOTAL * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&n->stencil, sizeof(n->h_stencil));
  if (e == cudaSuccess) e = cudaMemcpy(n->w, host_weights, MR_WEIGHT_TOTAL * sizeof(float), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(n->stencil, n->h_stencil, sizeof(n->h_stencil), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    mr_network_destroy(h);
    return set_error(MR_ERR_NOMEM, "mr_network_create: %s", cudaGetErrorString(e));
  }
  int rc = pack_network(n);
  if (rc) { mr_network_destroy(h); return rc; }
  *out = h;
  return MR_OK;
}

int mr_network_destroy(mr_network* h) {
  if (!h) return MR_OK;
  cudaFree(h->n.w);
  cudaFree(h->n.stencil);
  free_packed(&h->n);
  delete h;
  return MR_OK;
}

int mr_render(mr_volume* h, const mr_network* net, const mr_render_params* p, float* dev_rgb, void* stream) {
  clear_error();
  if (!h || !dev_rgb) return set_error(MR_ERR_ARG, "mr_render: NULL argument");
  int rc = check_params(p);
  if (rc) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  switch (p->render_type) {
    case MR_RT_PT: return render_pt(&h->v, p, dev_rgb, s);
    case MR_RT_MRPNN: return render_neural(&h->v, net ? &net->n : nullptr, p, dev_rgb, s);
    case MR_RT_MARCHING_MRPNN: return render_marching(&h->v, net ? &net->n : nullptr, p, dev_rgb, s);
    case MR_RT_RPNN: return set_error(MR_ERR_UNSUPPORTED, "RPNN is not supported (its weights are not published)");
    default: return set_error(MR_ERR_ARG, "unknown render type %d", p->render_type);
  }
}

int mr_render_host(mr_volume* h, const mr_network* net, const mr_render_params* p, float* host_rgb) {
  clear_error();
  if (!h || !host_rgb) return set_error(MR_ERR_ARG, "mr_render_host: NULL argument");
  int rc = check_params(p);
  if (rc) return rc;
  size_t n = (size_t)p->width * p->height * 3;
  float* d = nullptr;
  MR_CUDA(cudaMalloc(&d, n * sizeof(float)));
  rc = mr_render(h, net, p, d, nullptr);
  if (rc == MR_OK) {
    cudaError_t e = cudaMemcpy(host_rgb, d, n * sizeof(float), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) rc = cuda_error(e, "cudaMemcpy(result)");
  }
  cudaFree(d);
  return rc;
}

int mr_render_host_async(mr_volume* h, const mr_network* net, const mr_render_params* p, float* host_rgb,
                         void* stream, int64_t* ticket) {
  clear_error();
  if (!h || !host_rgb) return set_error(MR_ERR_ARG, "mr_render_host_async: NULL argument");
  int rc = check_params(p);
  if (rc) return rc;
  Volume* v = &h->v;
  cudaStream_t s = (cudaStream_t)stream;
  const size_t bytes = (size_t)p->width * p->height * 3 * sizeof(float);
  if (!v->copy_stream) {
    MR_CUDA(cudaStreamCreateWithFlags(&v->copy_stream, cudaStreamNonBlocking));
    for (int i = 0; i < 2; ++i) {
      MR_CUDA(cudaEventCreateWithFlags(&v->rendered[i], cudaEventDisableTiming));
      MR_CUDA(cudaEventCreateWithFlags(&v->copied[i], cudaEventDisableTiming));
    }
  }
  if (v->frame_bytes < bytes) {
    MR_CUDA(cudaStreamSynchronize(v->copy_stream));  // earlier copies still read the old frames
    for (int i = 0; i < 2; ++i) {
      if (v->frame[i]) MR_CUDA(cudaFree(v->frame[i]));
      v->frame[i] = nullptr;
    }
    v->frame_bytes = 0;
    for (int i = 0; i < 2; ++i) {
      cudaError_t e = cudaMalloc(&v->frame[i], bytes);
      if (e != cudaSuccess) return set_error(MR_ERR_NOMEM, "frame buffer of %zu bytes: %s", bytes, cudaGetErrorString(e));
    }
    v->frame_bytes = bytes;
  }
  const int slot = (int)(v->frame_seq & 1);
  // the frame two calls back must be on the host before this render overwrites it
  MR_CUDA(cudaStreamWaitEvent(s, v->copied[slot], 0));
  rc = mr_render(h, net, p, v->frame[slot], stream);
  if (rc) return rc;
  MR_CUDA(cudaEventRecord(v->rendered[slot], s));
  MR_CUDA(cudaStreamWaitEvent(v->copy_stream, v->rendered[slot], 0));
  MR_CUDA(cudaMemcpyAsync(host_rgb, v->frame[slot], bytes, cudaMemcpyDeviceToHost, v->copy_stream));
  MR_CUDA(cudaEventRecord(v->copied[slot], v->copy_stream));
  if (ticket) *ticket = v->frame_seq;
  ++v->frame_seq;
  return MR_OK;
}

int mr_render_host_wait(mr_volume* h, int64_t ticket, int32_t timeout_ms) {
  clear_error();
  if (!h) return set_error(MR_ERR_ARG, "mr_render_host_wait: NULL argument");
  Volume* v = &h->v;
  if (ticket >= v->frame_seq) return set_error(MR_ERR_ARG, "frame %lld has not been issued", (long long)ticket);
  if (!v->copy_stream || v->frame_seq == 0) return MR_OK;
  // copies run in issue order on the copy stream: the last copy recorded for
  // the ticket's frame buffer is that frame's or a later one
  cudaEvent_t e = ticket < 0 ? v->copied[(v->frame_seq - 1) & 1] : v->copied[ticket & 1];
  auto t0 = std::chrono::steady_clock::now();
  for (;;) {
    cudaError_t q = cudaEventQuery(e);
    if (q == cudaSuccess) return MR_OK;
    if (q != cudaErrorNotReady) return cuda_error(q, "cudaEventQuery(frame copy)");
    auto ms = std::chrono::duration_cast<std::chrono::milliseconds>(std::chrono::steady_clock::now() - t0).count();
    if (timeout_ms >= 0 && ms > timeout_ms)
      return set_error(MR_ERR_TIMEOUT, "frame copy still running after %d ms", timeout_ms);
    std::this_thread::sleep_for(std::chrono::microseconds(50));
  }
}

int mr_sync(void* stream, int32_t timeout_ms) {
  clear_error();
  auto t0 = std::chrono::steady_clock::now();
  for (;;) {
    cudaError_t e = cudaStreamQuery((cudaStream_t)stream);
    if (e == cudaSuccess) return MR_OK;
    if (e != cudaErrorNotReady) return cuda_error(e, "cudaStreamQuery");
    auto ms = std::chrono::duration_cast<std::chrono::milliseconds>(std::chrono::steady_clock::now() - t0).count();
    if (timeout_ms >= 0 && ms > timeout_ms)
      return set_error(MR_ERR_TIMEOUT, "stream still busy after %d ms", timeout_ms);
    std::this_thread::sleep_for(std::chrono::microseconds(200));
  }
}

}  // extern "C"
