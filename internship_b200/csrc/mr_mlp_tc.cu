// Tensor-core (tcgen05) operand images of the network. Filled in by the
// BF16/FP8 path; the fp32 path uses the flat blob directly.
#include "mr_internal.h"

namespace mr {

int pack_network(Network* n) {
  n->packed = nullptr;
  n->packed_bytes = 0;
  return MR_OK;
}

void free_packed(Network* n) {
  if (n->packed) cudaFree(n->packed);
  n->packed = nullptr;
  n->packed_bytes = 0;
}

}  // namespace mr
