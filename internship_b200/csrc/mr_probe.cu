// Memory-path probe: streams a device buffer through the SMs with 16-byte
// loads that bypass L1 (ld.global.cg), `passes` times, so that a buffer that
// fits in L2 measures the L2 -> SM read bandwidth and a buffer far larger than
// L2 measures HBM. The roofline denominators of the L2-resident kernels (the
// descriptor gather, delta tracking on small grids) come from it.
#include "mr_internal.h"

namespace mr {

__global__ void __launch_bounds__(512) k_stream_read(const uint4* __restrict__ buf, size_t n16, int passes,
                                                     uint32_t* __restrict__ sink) {
  uint32_t acc = 0;
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  for (int p = 0; p < passes; ++p) {
    // each pass starts the threads at a different offset, so that a thread
    // never re-reads its own lines from L1-like structures
    const size_t start = (blockIdx.x * (size_t)blockDim.x + threadIdx.x + (size_t)p * 4099 * 32) % stride;
    for (size_t i = start; i < n16; i += stride) {
      uint4 v;
      asm volatile("ld.global.cg.v4.u32 {%0,%1,%2,%3}, [%4];"
                   : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
                   : "l"(buf + i));
      acc ^= v.x ^ v.y ^ v.z ^ v.w;
    }
  }
  if (acc == 0x9e3779b9u) *sink = acc;  // keeps the loads live; practically never stores
}

}  // namespace mr

using namespace mr;

extern "C" int mr_stream_read_probe(const void* dev_buf, size_t bytes, int32_t passes, uint32_t* dev_sink,
                                    void* stream) {
  clear_error();
  if (!dev_buf || !dev_sink || passes <= 0) return set_error(MR_ERR_ARG, "mr_stream_read_probe: bad argument");
  if (bytes < 16 || (bytes & 15) || ((uintptr_t)dev_buf & 15))
    return set_error(MR_ERR_ARG, "mr_stream_read_probe: buffer must be 16-byte aligned and a multiple of 16 bytes");
  const int grid = sm_count() * 4;
  k_stream_read<<<grid, 512, 0, (cudaStream_t)stream>>>((const uint4*)dev_buf, bytes / 16, passes, dev_sink);
  MR_CUDA(cudaGetLastError());
  return MR_OK;
}
