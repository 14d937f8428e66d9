"""Generate tests/golden/ref_math.npz from the reference's own math code.

Compiles the reference's core/vector.cu (its __host__ __device__ functions)
together with a small host driver written here, runs it on a fixed grid of
inputs and stores the outputs. Needs nvcc and the reference checkout
(located by oracle/build.py, MRPNN_REFERENCE overrides it); the committed .npz
is what the tests read.

Functions pinned: HenyeyGreenstein, SampleHeneyGreenstein,
SampleHenyeyGreenstein, UniformSampleSphere, RayBoxOffset, RayBoxDistance,
GetSamples23_ (core/vector.cu:41-75, 190-237, 299-400).
"""
import os
import subprocess
import sys
import tempfile

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__)))))
from oracle.build import REF_SRC as REF  # noqa: E402
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "ref_math.npz")

DRIVER = r'''
#include "vector.cuh"
#include <cstdio>
#include <cstdlib>
int main(int argc, char** argv) {
  FILE* fi = fopen(argv[1], "rb");
  FILE* fo = fopen(argv[2], "wb");
  int n; fread(&n, 4, 1, fi);
  float* a = (float*)malloc(sizeof(float) * n * 8);
  fread(a, sizeof(float), n * 8, fi);
  for (int k = 0; k < n; ++k) {
    float* x = a + 8 * k;   // c, g, s, e0, e1, px, py, pz  (dir reuses e0/e1 via sphere)
    float hg = HenyeyGreenstein(x[0], x[1]);
    float cs = SampleHeneyGreenstein(x[2], x[1]);
    float3 v = UniformSampleSphere(float2{x[3], x[4]});
    float3 d = SampleHenyeyGreenstein(x[2], x[3], v, x[1]);
    float3 p = float3{x[5], x[6], x[7]};
    float off = RayBoxOffset(p, v);
    float dis = RayBoxDistance(p, v);
    float rec[10] = {hg, cs, v.x, v.y, v.z, d.x, d.y, d.z, off, dis};
    fwrite(rec, sizeof(float), 10, fo);
  }
  for (int i = 0; i < 193; ++i) {
    Offset_Layer_ o = GetSamples23_(i);
    float rec[4] = {o.Offset, o.Layer, (float)o.type, (float)o.localindex};
    fwrite(rec, sizeof(float), 4, fo);
  }
  fclose(fo);
  return 0;
}
'''


def main():
    core = os.path.join(REF, "core")
    if not os.path.isdir(core):
        sys.exit("reference checkout not found: " + core)
    rng = np.random.default_rng(20261203)
    n = 4096
    a = np.zeros((n, 8), np.float32)
    a[:, 0] = rng.uniform(-1, 1, n)
    a[:, 1] = rng.choice([0.0, 0.3, 0.7, 0.857, 0.9, -0.5], n)
    a[:, 2] = rng.uniform(0, 1, n)
    a[:, 3] = rng.uniform(0, 1, n)
    a[:, 4] = rng.uniform(0, 1, n)
    a[:, 5:8] = rng.uniform(-1.2, 1.2, (n, 3))
    with tempfile.TemporaryDirectory() as td:
        drv = os.path.join(td, "driver.cu")
        open(drv, "w").write(DRIVER)
        exe = os.path.join(td, "driver")
        subprocess.check_call(["nvcc", "-std=c++17", "-w", "-I", core, drv,
                               os.path.join(core, "vector.cu"), "-o", exe])
        fin, fout = os.path.join(td, "in.bin"), os.path.join(td, "out.bin")
        with open(fin, "wb") as f:
            f.write(np.int32(n).tobytes())
            f.write(a.tobytes())
        subprocess.check_call([exe, fin, fout])
        raw = np.fromfile(fout, np.float32)
    per = raw[:n * 10].reshape(n, 10)
    sten = raw[n * 10:].reshape(193, 4)
    np.savez_compressed(OUT, inputs=a, outputs=per, stencil=sten)
    print("wrote", OUT)


if __name__ == "__main__":
    main()
