// k_row_split.cu -- the RowOps of the FP32 row shapes, whose three levels
// (row_kernel's GEN) compile in translation units of their own
// (k_row_f32_v*_g*.cu): the register row transforms make each level's kernels
// long to compile, and one unit per level lets the build run them in parallel.
#include "launch.h"

namespace mrm {
namespace {

template <typename R, int V>
cudaError_t row_launch_split(int stage, bool stats, const RowLaunch& a, int istep, int flags) {
  if (a.gen == 2) return row_gen_ops<R, V, 2>().launch(stage, stats, a, istep, flags);
  if (a.gen == 1) return row_gen_ops<R, V, 1>().launch(stage, stats, a, istep, flags);
  return row_gen_ops<R, V, 0>().launch(stage, stats, a, istep, flags);
}

template <typename R, int V>
const RowOps& split_ops() {
  static const RowOps ops = [] {
    RowOps o{row_launch_split<R, V>, {}};
    const RowGenOps* g[3] = {&row_gen_ops<R, V, 0>(), &row_gen_ops<R, V, 1>(), &row_gen_ops<R, V, 2>()};
    for (int l = 0; l < 3; ++l)
      for (int q = 0; q < 6; ++q) o.fn[l][q] = g[l]->fn[q];
    return o;
  }();
  return ops;
}

}  // namespace

template <>
const RowOps& row_ops<float, 0>() { return split_ops<float, 0>(); }
template <>
const RowOps& row_ops<float, 1>() { return split_ops<float, 1>(); }
template <>
const RowOps& row_ops<float, 2>() { return split_ops<float, 2>(); }
template <>
const RowOps& row_ops<float, 3>() { return split_ops<float, 3>(); }
template <>
const RowOps& row_ops<float, 4>() { return split_ops<float, 4>(); }

}  // namespace mrm
