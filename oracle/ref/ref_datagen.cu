// Harness around the reference's training-point sampler - TEST
// INFRASTRUCTURE ONLY.
//
// Compiles the reference's dataGen.cu in place (its main renamed, its GUI
// header replaced by oracle/ref/stub/GUI.hpp) into oracle/_ref/libref_volume.so
// and exposes GetDesiredCountSample / MeanFreePathSample (dataGen.cu:148-216).
// Those host functions read VolumeRender::DensityAtPosition(0, p), the 256^3
// mip level 0, which the reference's own Update() leaves unfilled (its mip
// loop reads the level it writes): the harness hands them the intended level
// 0 through the class's data members, made reachable here by compiling
// volume.hpp with `class` read as `struct` (same members, same layout).
#include <algorithm>
#include <chrono>
#include <cstdint>
#include <cstring>
#include <fstream>
#include <functional>
#include <iomanip>
#include <iostream>
#include <random>
#include <sstream>
#include <string>
#include <vector>

#include <cuda_runtime.h>
#include <vector_types.h>

#define class struct
#include "volume.hpp"
#undef class

#define main refdatagen_main
#include "dataGen.cu"
#undef main

extern "C" {

// GetDesiredCountSample(v, Samples, n, alpha, alpha) on a volume whose mip
// level 0 is `mip0` (256^3, x-major) and whose majorant is max_density:
// n points (pos n x 3, view n x 3); g is dataGen's fixed 0.857.
int refv_datagen_samples(void* h, const float* mip0, float max_density, float alpha, int n, float* pos,
                         float* view) {
  VolumeRender* v = (VolumeRender*)h;
  std::memcpy(v->mips[0], mip0, sizeof(float) * 256 * 256 * 256);
  v->max_density = max_density;
  std::vector<SamplePoint> s;
  GetDesiredCountSample(*v, s, n, alpha, alpha);
  const int m = (int)s.size() < n ? (int)s.size() : n;
  for (int k = 0; k < m; ++k) {
    pos[3 * k] = s[k].Position.x;
    pos[3 * k + 1] = s[k].Position.y;
    pos[3 * k + 2] = s[k].Position.z;
    view[3 * k] = s[k].ViewDir.x;
    view[3 * k + 1] = s[k].ViewDir.y;
    view[3 * k + 2] = s[k].ViewDir.z;
  }
  return m;
}

}  // extern "C"
