// Exercises the C++ host interface (include/mrpnn.hpp) the way the
// reference's main.cu drives VolumeRender and Camera: a solid sphere filled
// through SetDatas, Update, a delta-tracking render, a neural render and
// Camera::RenderToFile.
//   shim_demo <out_pt.f32> <out_nn.f32> <bmp_path_without_extension>
#include <cstdio>
#include <vector>

#include "mrpnn.hpp"

struct Vec { float x, y, z; };
struct Size { int x, y; };

int main(int argc, char** argv) {
  if (argc < 4) {
    std::fprintf(stderr, "usage: shim_demo out_pt out_nn bmp\n");
    return 2;
  }
  mrpnn::VolumeRender volume(64);
  volume.SetDatas([](int, int, int, float u, float v, float w) {
    const float dx = u - 0.5f, dy = v - 0.5f, dz = w - 0.5f;
    return dx * dx + dy * dy + dz * dz < 0.25f * 0.25f ? 1.0f : 0.0f;
  });
  volume.Update();
  volume.SetScatterRate(0.99f);
  const Vec ori{0.0f, 0.0f, 2.0f}, up{0.0f, 0.4f, 0.0f}, right{0.4f, 0.0f, 0.0f}, L{0.3f, 0.8f, 0.52f};
  const Size size{48, 32};
  auto pt = volume.Render(size, ori, up, right, L, mrpnn::VolumeRender::RenderType::PT, 0.857f, 16.0f,
                          mr_float3{1, 1, 1}, 64, 16);
  std::vector<float> w(MR_WEIGHT_TOTAL);
  mr_weights_xavier(1, w.data(), w.size());
  volume.SetWeights(w);
  auto nn = volume.Render(size, ori, up, right, L, mrpnn::VolumeRender::RenderType::MRPNN, 0.857f, 16.0f,
                          mr_float3{1, 1, 1}, 64, 2);
  mrpnn::Camera cam(volume, "demo", Vec{0.75f, 0.75f, 0.75f}, 40);
  cam.RenderToFile(argv[3], L, mr_float3{1, 1, 1}, 16.0f, 32, 0.857f, 8, mrpnn::Camera::ACES);
  for (int k = 0; k < 2; ++k) {
    std::FILE* fp = std::fopen(argv[1 + k], "wb");
    if (!fp) return 1;
    const auto& img = k == 0 ? pt : nn;
    std::fwrite(img.data(), sizeof(mr_float3), img.size(), fp);
    std::fclose(fp);
  }
  std::printf("max_density %g\n", volume.max_density);
  return 0;
}
