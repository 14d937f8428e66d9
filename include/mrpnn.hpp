// mrpnn.hpp - C++ host interface of the B200 renderer, header-only over the
// C ABI of mrpnn_b200.h. Class and method names, argument order, defaults and
// meaning follow the reference's host API so that its callers port by
// swapping the include:
//   VolumeRender  core/volume.hpp:45-146 (SetData/SetDatas/Update/Update_TR/
//                 UpdateHGLut/SetScatterRate/SetTrScale/SetExposure/Render)
//   Camera        core/camera.hpp:10-41, core/camera.cu:163-252
//                 (SetPosition, Render, RenderToFile writing <path>.bmp)
//   SaveBMP       core/camera.cu:10-61 (32-bit BGRA, top-down)
// Vector arguments accept any type with .x/.y/.z (CUDA's float3 included).
// Errors are reported like the reference (printed to stderr, execution
// continues); define MRPNN_THROW_ON_ERROR to throw std::runtime_error instead.
// Link with libmrpnn_b200.so.
#ifndef MRPNN_HPP
#define MRPNN_HPP

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <functional>
#include <stdexcept>
#include <string>
#include <vector>

#include "mrpnn_b200.h"
#include "mrpnn_weights.h"

namespace mrpnn {

inline bool check(int rc, const char* what) {
  if (rc == MR_OK) return true;
#ifdef MRPNN_THROW_ON_ERROR
  throw std::runtime_error(std::string(what) + ": " + mr_last_error());
#else
  std::fprintf(stderr, "mrpnn: %s: %s\n", what, mr_last_error());
  return false;
#endif
}

template <class V>
inline mr_float3 f3(const V& v) { return mr_float3{(float)v.x, (float)v.y, (float)v.z}; }
inline mr_float3 f3(float x, float y, float z) { return mr_float3{x, y, z}; }

inline mr_float3 operator*(mr_float3 a, float s) { return f3(a.x * s, a.y * s, a.z * s); }
inline float dot(mr_float3 a, mr_float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline mr_float3 cross(mr_float3 a, mr_float3 b) {
  return f3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
inline mr_float3 normalize(mr_float3 a) { return a * (1.0f / std::sqrt(dot(a, a))); }

using FillFunc = std::function<float(int, int, int, float, float, float)>;  // omp.hpp:8

class VolumeRender {
 public:
  enum class RenderType { PT = MR_RT_PT, RPNN = MR_RT_RPNN, MRPNN = MR_RT_MRPNN };  // volume.hpp:88-90

  int resolution = 0;
  float max_density = 0.0f;

  explicit VolumeRender(int res) : resolution(res), data_((size_t)res * res * res, 0.0f) {
    check(mr_volume_create(res, &vol_), "VolumeRender(resolution)");
  }
  ~VolumeRender() {
    if (net_) mr_network_destroy(net_);
    if (vol_) mr_volume_destroy(vol_);
  }
  VolumeRender(const VolumeRender&) = delete;
  VolumeRender& operator=(const VolumeRender&) = delete;

  // SetData / SetDatas (volume.cu:938-944): host copy, uploaded by Update().
  void SetData(int x, int y, int z, float v) { data_[((size_t)x * resolution + y) * resolution + z] = v; }
  void SetDatas(const FillFunc& f) {
    const int r = resolution;
#pragma omp parallel for schedule(static)
    for (int x = 0; x < r; ++x)
      for (int y = 0; y < r; ++y)
        for (int z = 0; z < r; ++z)
          data_[((size_t)x * r + y) * r + z] = f(x, y, z, (x + 0.5f) / r, (y + 0.5f) / r, (z + 0.5f) / r);
  }
  void SetDatas(const float* values) { std::copy(values, values + data_.size(), data_.begin()); }
  // Update (volume.cu:1203-1316): upload, majorant, mip and variance pyramids.
  void Update() {
    if (!check(mr_volume_set_data(vol_, data_.data(), data_.size()), "SetDatas")) return;
    if (!check(mr_volume_update(vol_, nullptr), "Update")) return;
    check(mr_volume_max_density(vol_, &max_density), "Update");
  }
  template <class V>
  void Update_TR(const V& lightDir, float alpha = 64.0f) {
    check(mr_volume_update_tr(vol_, f3(lightDir), alpha, nullptr), "Update_TR");
  }
  void UpdateHGLut(float g) { check(mr_volume_update_hglut(vol_, g, seed_, nullptr), "UpdateHGLut"); }

  void SetScatterRate(float s) { scatter_ = f3(s, s, s); }
  template <class V>
  void SetScatterRate(const V& s) { scatter_ = f3(s); }
  void SetTrScale(float s) { tr_scale_ = s; }
  void SetExposure(float e) { exposure_ = e; }
  float GetExposure() const { return exposure_; }
  void SetEnvColor(mr_float3 c) { env_ = c; }
  void SetCheckboard(bool c) { checkerboard_ = c; }
  void SetSeed(uint32_t s) { seed_ = s; }
  void SetPrecision(mr_precision p) { precision_ = p; }
  void SetSampler(mr_sampler s) { sampler_ = s; }

  // The NNWeight.cuh arrays as one blob in declaration order (mrpnn_weights.h);
  // stencil: 160 x 3 directions, empty = the library's built-in stencil.
  bool SetWeights(const std::vector<float>& blob, const std::vector<float>& stencil = {}) {
    if (net_) mr_network_destroy(net_);
    net_ = nullptr;
    return check(mr_network_create(blob.data(), blob.size(), stencil.empty() ? nullptr : stencil.data(), &net_),
                 "SetWeights");
  }

  // Render(int2 size, ...) (volume.cu:410-467): mean radiance over spp
  // samples (PT) or spp neural passes (MRPNN); row-major, top row first.
  template <class I2, class V>
  std::vector<mr_float3> Render(const I2& size, const V& ori, const V& up, const V& right, const V& lightDir,
                                RenderType rt = RenderType::PT, float g = 0.857f, float alpha = 1.0f,
                                mr_float3 lightColor = {1, 1, 1}, int multiScatter = 512, int spp = 1024) {
    mr_render_params p = params(size.x, size.y, f3(ori), f3(up), f3(right), f3(lightDir), rt, g, alpha, lightColor,
                                multiScatter, spp);
    const size_t n = (size_t)size.x * size.y;
    std::vector<mr_float3> out(n, f3(0, 0, 0));
    if (rt == RenderType::PT) {
      check(mr_render_host(vol_, net_, &p, reinterpret_cast<float*>(out.data())), "Render");
      return out;
    }
    // neural: spp passes averaged (progressive accumulation of the reference)
    std::vector<float> pass(3 * n);
    const int passes = std::max(1, spp);
    for (int k = 0; k < passes; ++k) {
      p.sample_offset = (uint32_t)k;
      if (!check(mr_render_host(vol_, net_, &p, pass.data()), "Render")) break;
      float* o = reinterpret_cast<float*>(out.data());
      for (size_t i = 0; i < 3 * n; ++i) o[i] += (pass[i] - o[i]) / (float)(k + 1);
    }
    return out;
  }

  // Interactive Render (volume.cu:469-547) into caller device buffers:
  // accum W*H*3 floats, hist W*H histograms, bgra W*H pixels.
  template <class I2, class V>
  void Render(float* accum, mr_histogram* hist, uint32_t* bgra, const I2& size, const V& ori, const V& up,
              const V& right, const V& lightDir, mr_float3 lightColor, float alpha, int multiScatter, float g,
              int randseed, RenderType rt = RenderType::PT, int toneType = 2, bool denoise = false) {
    mr_render_params p = params(size.x, size.y, f3(ori), f3(up), f3(right), f3(lightDir), rt, g, alpha, lightColor,
                                multiScatter, 1);
    mr_interactive it{};
    it.prev_ori = has_prev_ ? prev_ori_ : p.ori;
    it.prev_up = has_prev_ ? prev_up_ : p.up;
    it.prev_right = has_prev_ ? prev_right_ : p.right;
    it.frame_index = randseed;
    it.checkerboard = checkerboard_ ? 1 : 0;
    it.tone = toneType;
    it.denoise = denoise ? 1 : 0;
    it.exposure = exposure_;
    check(mr_render_interactive(vol_, net_, &p, &it, accum, hist, bgra, nullptr), "Render");
    prev_ori_ = p.ori;
    prev_up_ = p.up;
    prev_right_ = p.right;
    has_prev_ = true;
  }

  mr_volume* handle() const { return vol_; }
  mr_network* network() const { return net_; }

 private:
  mr_render_params params(int w, int h, mr_float3 ori, mr_float3 up, mr_float3 right, mr_float3 L, RenderType rt,
                          float g, float alpha, mr_float3 lc, int bounces, int spp) const {
    mr_render_params p{};
    p.width = w;
    p.height = h;
    p.ori = ori;
    p.up = up;
    p.right = right;
    p.light_dir = L;
    p.light_color = lc;
    p.alpha = alpha;
    p.g = g;
    p.scatter_rate = scatter_;
    p.tr_scale = tr_scale_;
    p.env_color = env_;
    p.max_bounces = bounces;
    p.spp = std::max(1, spp);
    p.seed = seed_;
    p.sample_offset = 0;
    p.render_type = (int32_t)rt;
    p.precision = precision_;
    p.sampler = sampler_;
    return p;
  }

  mr_volume* vol_ = nullptr;
  mr_network* net_ = nullptr;
  std::vector<float> data_;
  mr_float3 scatter_{1, 1, 1}, env_{0, 0, 0};
  float tr_scale_ = 1.0f, exposure_ = 1.0f;
  bool checkerboard_ = false;
  uint32_t seed_ = 0;
  mr_precision precision_ = MR_PREC_FP32;
  mr_sampler sampler_ = MR_SAMPLER_EXACT;
  bool has_prev_ = false;
  mr_float3 prev_ori_{}, prev_up_{}, prev_right_{};
};

using ToneMapFunction = std::function<mr_float3(mr_float3)>;  // camera.hpp:6

// SaveBMP (camera.cu:10-61): RGBA bytes row-major, written as 32-bit BGRA
// with a negative height (top-down) to <filename>.bmp.
inline int SaveBMP(const unsigned char* rgba, int w, int h, const char* filename) {
  unsigned char hd[54] = {0x42, 0x4d, 0, 0, 0, 0, 0, 0, 0, 0, 0x36, 0, 0, 0, 0x28, 0, 0, 0, 0,
                          0,    0,    0, 0, 0, 0, 0, 0x01, 0, 0x20, 0, 0, 0, 0, 0, 0, 0, 0x10, 0,
                          0,    0,    0, 0, 0, 0, 0, 0, 0, 0, 0,    0, 0, 0, 0, 0};
  const uint32_t size = (uint32_t)w * (uint32_t)h * 4u + 54u;
  const int32_t hh = -h;
  for (int i = 0; i < 4; ++i) {
    hd[2 + i] = (unsigned char)(size >> (8 * i));
    hd[18 + i] = (unsigned char)((uint32_t)w >> (8 * i));
    hd[22 + i] = (unsigned char)((uint32_t)hh >> (8 * i));
  }
  std::FILE* fp = std::fopen((std::string(filename) + ".bmp").c_str(), "wb");
  if (!fp) return -1;
  std::fwrite(hd, 1, 54, fp);
  std::vector<unsigned char> row((size_t)w * 4);
  for (int y = 0; y < h; ++y) {
    const unsigned char* src = rgba + (size_t)y * w * 4;
    for (int x = 0; x < w; ++x) {
      row[4 * x] = src[4 * x + 2];
      row[4 * x + 1] = src[4 * x + 1];
      row[4 * x + 2] = src[4 * x];
      row[4 * x + 3] = src[4 * x + 3];
    }
    std::fwrite(row.data(), 1, row.size(), fp);
  }
  std::fclose(fp);
  return 0;
}

class Camera {
 public:
  int resolution;
  std::string name;

  // Camera(volume, name, position, resolution) (camera.cu:163-171): looks at
  // the origin, 90 degree field of view (unit right / up).
  template <class V = mr_float3>
  Camera(VolumeRender& volume, std::string name_ = "test camera", const V& position = V{0.75f, 0.75f, 0.75f},
         int res = 512)
      : resolution(res), name(std::move(name_)), volume_(&volume) {
    SetPosition(position);
  }

  // SetPosition (camera.cu:173-189), with the reference's pole cases.
  template <class V>
  void SetPosition(const V& position) {
    ori_ = f3(position);
    forward_ = normalize(ori_ * -1.0f);
    right_ = normalize(cross(f3(0, 1, 0), forward_));
    up_ = cross(forward_, right_);
    if (ori_.x == 0 && ori_.z == 0) {
      right_ = f3(1, 0, 0);
      up_ = ori_.y > 0 ? f3(0, 0, 1) : f3(0, 0, -1);
    }
  }
  mr_float3 GetPosition() const { return ori_; }
  void SetVolume(VolumeRender& v) { volume_ = &v; }

  static mr_float3 None(mr_float3 c) { return c; }
  static mr_float3 Gamma(mr_float3 c) {
    return f3(std::pow(std::max(c.x, 0.0f), 1.0f / 2.2f), std::pow(std::max(c.y, 0.0f), 1.0f / 2.2f),
              std::pow(std::max(c.z, 0.0f), 1.0f / 2.2f));
  }
  // ACES RRT + ODT fit (camera.cu:74-160): the ACES colour-space matrices,
  // desaturation, the fitted tonescale, dim surround, gamma 2.2.
  static mr_float3 ACES(mr_float3 c) {
    auto mul = [](const float* m, mr_float3 x) {
      return f3(m[0] * x.x + m[1] * x.y + m[2] * x.z, m[3] * x.x + m[4] * x.y + m[5] * x.z,
                m[6] * x.x + m[7] * x.y + m[8] * x.z);
    };
    static const float srgb_ap0[9] = {0.4397010f, 0.3829780f, 0.1773350f, 0.0897923f, 0.8134230f,
                                      0.0967616f, 0.0175440f, 0.1115440f, 0.8707040f};
    static const float ap0_ap1[9] = {1.4514393161f, -0.2365107469f, -0.2149285693f, -0.0765537734f, 1.1762296998f,
                                     -0.0996759264f, 0.0083161484f, -0.0060324498f, 0.9977163014f};
    static const float ap1_xyz[9] = {0.6624541811f, 0.1340042065f, 0.1561876870f, 0.2722287168f, 0.6740817658f,
                                     0.0536895174f, -0.0055746495f, 0.0040607335f, 1.0103391003f};
    static const float xyz_ap1[9] = {1.6410233797f, -0.3248032942f, -0.2364246952f, -0.6636628587f, 1.6153315917f,
                                     0.0167563477f, 0.0117218943f, -0.0082844420f, 0.9883948585f};
    static const float d60_d65[9] = {0.98722400f, -0.00611327f, 0.0159533f, -0.00759836f, 1.00186000f,
                                     0.0053302f, 0.00307257f, -0.00509595f, 1.0816800f};
    static const float xyz_709[9] = {3.2409699419f, -1.5373831776f, -0.4986107603f, -0.9692436363f, 1.8759675015f,
                                     0.0415550574f, 0.0556300797f, -0.2039769589f, 1.0569715142f};
    const mr_float3 ap1_y = f3(0.272229f, 0.674082f, 0.0536895f);
    mr_float3 x = mul(ap0_ap1, mul(srgb_ap0, c));
    float y = dot(x, ap1_y);
    x = f3(y * (1.0f - 0.96f) + x.x * 0.96f, y * (1.0f - 0.96f) + x.y * 0.96f, y * (1.0f - 0.96f) + x.z * 0.96f);
    auto ts = [](float t) { return (t * (t * 278.5085f + 10.7772f)) / (t * (t * 293.6045f + 88.7122f) + 80.6889f); };
    x = f3(ts(x.x), ts(x.y), ts(x.z));
    mr_float3 XYZ = mul(ap1_xyz, x);
    const float div = std::max(XYZ.x + XYZ.y + XYZ.z, 1e-4f);
    const float cx = XYZ.x / div, cy = XYZ.y / div;
    const float Y = std::pow(std::min(std::max(XYZ.y, 0.0f), 65504.0f), 0.9811f);
    const float m = Y / std::max(cy, 1e-4f);
    x = mul(xyz_ap1, f3(cx * m, Y, (1.0f - cx - cy) * m));
    y = dot(x, ap1_y);
    x = f3(y * (1.0f - 0.93f) + x.x * 0.93f, y * (1.0f - 0.93f) + x.y * 0.93f, y * (1.0f - 0.93f) + x.z * 0.93f);
    return Gamma(mul(xyz_709, mul(d60_d65, mul(ap1_xyz, x))));
  }

  // RenderToFile (camera.cu:226-252): render, tone map, write <path>.bmp.
  template <class V>
  void RenderToFile(const std::string& path, const V& lightDir, mr_float3 lightColor = {1, 1, 1}, float alpha = 1.0f,
                    int multiScatter = 1, float g = 0.0f, int sampleNum = 1, ToneMapFunction tone = ACES,
                    VolumeRender::RenderType rt = VolumeRender::RenderType::PT, float exp = 1.0f) {
    struct I2 { int x, y; } size{resolution, resolution};
    const auto img = volume_->Render(size, ori_, up_, right_, f3(lightDir), rt, g, alpha, lightColor, multiScatter,
                                     sampleNum);
    std::vector<unsigned char> rgba((size_t)resolution * resolution * 4);
    for (size_t i = 0; i < img.size(); ++i) {
      const mr_float3 c = tone(img[i] * exp);
      rgba[4 * i] = (unsigned char)(255.0f * std::min(std::max(c.x, 0.0f), 1.0f));
      rgba[4 * i + 1] = (unsigned char)(255.0f * std::min(std::max(c.y, 0.0f), 1.0f));
      rgba[4 * i + 2] = (unsigned char)(255.0f * std::min(std::max(c.z, 0.0f), 1.0f));
      rgba[4 * i + 3] = 255;
    }
    SaveBMP(rgba.data(), resolution, resolution, path.c_str());
  }

  mr_float3 up() const { return up_; }
  mr_float3 right() const { return right_; }

 private:
  mr_float3 ori_{}, forward_{}, right_{}, up_{};
  VolumeRender* volume_;
};

}  // namespace mrpnn

#endif  // MRPNN_HPP
