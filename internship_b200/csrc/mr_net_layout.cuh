// Compile-time offsets of the weight arrays inside the flat blob
// (layout of include/mrpnn_weights.h = declaration order of core/NNWeight.cuh).
#pragma once
#include "../../include/mrpnn_weights.h"

namespace mr {

struct WeightTable {
  int off[MR_W_COUNT];
  int size[MR_W_COUNT];
};

constexpr WeightTable make_weight_table() {
  WeightTable t{};
  int o = 0, i = 0;
#define MR_W_ROW(name, n) t.off[i] = o; t.size[i] = (n); o += (n); ++i;
  MR_WEIGHT_LIST(MR_W_ROW)
#undef MR_W_ROW
  return t;
}
constexpr WeightTable kWT = make_weight_table();
static_assert(kWT.off[MR_W_COUNT - 1] + kWT.size[MR_W_COUNT - 1] == MR_WEIGHT_TOTAL, "weight blob size");

// Offset of weight array ID as a compile-time integral constant (usable in
// device code).
template <int ID>
struct WOff {
  static constexpr int value = make_weight_table().off[ID];
};
#define WOFF(name) (::mr::WOff<MR_W_##name>::value)

}  // namespace mr
