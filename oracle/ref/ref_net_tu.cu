// Translation unit that compiles the reference's core/radiancePredict.cu
// (found through -I <reference>/core) and adds a loader that overwrites its
// compiled-in weight arrays with a blob - TEST INFRASTRUCTURE ONLY.
//
// The static_asserts check, at compile time, that every entry of this
// project's blob layout (include/mrpnn_weights.h) names an array of the same
// size in the reference's core/NNWeight.cuh.
#include "radiancePredict.cu"

#include "../../include/mrpnn_weights.h"

#define MR_REF_CHECK(name, n) static_assert(sizeof(name) == (n) * sizeof(float), #name " size");
MR_WEIGHT_LIST(MR_REF_CHECK)
#undef MR_REF_CHECK

extern "C" int ref_load_weights(const float* blob, long count) {
  if (count != MR_WEIGHT_TOTAL) return 1;
  long off = 0;
#define MR_REF_LOAD(name, n)                                                   \
  if (cudaMemcpyToSymbol(name, blob + off, (n) * sizeof(float)) != cudaSuccess) \
    return 2;                                                                  \
  off += (n);
  MR_WEIGHT_LIST(MR_REF_LOAD)
#undef MR_REF_LOAD
  return 0;
}

// Copy the compiled-in (reference) weights out as a blob.
extern "C" int ref_read_weights(float* blob, long count) {
  if (count != MR_WEIGHT_TOTAL) return 1;
  long off = 0;
#define MR_REF_READ(name, n)                                                     \
  if (cudaMemcpyFromSymbol(blob + off, name, (n) * sizeof(float)) != cudaSuccess) \
    return 2;                                                                    \
  off += (n);
  MR_WEIGHT_LIST(MR_REF_READ)
#undef MR_REF_READ
  return 0;
}
