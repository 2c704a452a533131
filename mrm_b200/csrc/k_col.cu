// k_col.cu -- dispatch over the compiled column shapes (k_col_*.cu) and row
// shapes (k_row_*.cu), and the shared-memory limits of their kernels.
#include <map>
#include <mutex>
#include <utility>

#include "kernels.cuh"
#include "launch.h"

namespace mrm {
namespace {

template <typename R>
const ColOps* col_ops_of(int v) {
  if (v < 0 || v >= col_variant_count<R>()) return nullptr;
  if constexpr (sizeof(R) == sizeof(float)) {
    switch (v) {
      case 0: return &col_ops<float, 0>();
      case 1: return &col_ops<float, 1>();
      default: return &col_ops<float, 2>();
    }
  } else {
    switch (v) {
      case 0: return &col_ops<double, 0>();
      default: return &col_ops<double, 1>();
    }
  }
}

template <typename R>
const void* col_fn_any(int v) {
  const ColOps* o = col_ops_of<R>(v);
  return o ? o->fn : nullptr;
}

template <typename R>
cudaError_t col_launch_any(int v, const ColLaunch& a, int istep, int flags) {
  const ColOps* o = col_ops_of<R>(v);
  return o ? o->launch(a, istep, flags) : cudaErrorInvalidValue;
}

}  // namespace

cudaError_t allow_smem(const void* kern, size_t bytes) {
  static std::mutex mu;
  static std::map<std::pair<int, const void*>, size_t> cur;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lock(mu);
  size_t& c = cur[std::make_pair(dev, kern)];
  if (bytes <= c) return cudaSuccess;
  e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (e == cudaSuccess) c = bytes;
  return e;
}

// ---------------- row shapes (kernels in k_row_*.cu) ----------------
template <typename R>
static const RowOps* row_ops_of(int v) {
  if (v < 0 || v >= row_variant_count<R>()) return nullptr;
  if constexpr (sizeof(R) == sizeof(float)) {
    switch (v) {
      case 0: return &row_ops<float, 0>();
      case 1: return &row_ops<float, 1>();
      case 2: return &row_ops<float, 2>();
      case 3: return &row_ops<float, 3>();
      default: return &row_ops<float, 4>();
    }
  } else {
    switch (v) {
      case 0: return &row_ops<double, 0>();
      case 1: return &row_ops<double, 1>();
      default: return &row_ops<double, 2>();
    }
  }
}

template <typename R>
static cudaError_t launch_row_any(int v, int stage, bool stats, const RowLaunch& a, int istep, int flags) {
  const RowOps* o = row_ops_of<R>(v);
  return o ? o->launch(stage, stats, a, istep, flags) : cudaErrorInvalidValue;
}
template <typename R>
static cudaError_t row_allow_any(int v, const size_t* smem6) {
  const RowOps* o = row_ops_of<R>(v);
  if (!o) return cudaErrorInvalidValue;
  for (int g = 0; g < 3; ++g)
    for (int q = 0; q < kRowSlots; ++q) {
      cudaError_t e = allow_smem(o->fn[g][q], smem6[q]);
      if (e != cudaSuccess) return e;
    }
  return cudaSuccess;
}
template <typename R>
static cudaError_t row_occ_any(int v, int stage, size_t smem, int* blocks) {
  const RowOps* o = row_ops_of<R>(v);
  if (!o) return cudaErrorInvalidValue;
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks, o->fn[0][row_slot(stage, false)],
                                                       row_variant<R>(v).block, smem);
}
template <typename R>
static cudaError_t row_load_any(int v) {
  const RowOps* o = row_ops_of<R>(v);
  if (!o) return cudaErrorInvalidValue;
  for (int g = 0; g < 3; ++g)
    for (int q = 0; q < kRowSlots; ++q) {
      cudaFuncAttributes fa;
      cudaError_t e = cudaFuncGetAttributes(&fa, o->fn[g][q]);
      if (e != cudaSuccess) return e;
    }
  return cudaSuccess;
}
template <typename R>
static cudaError_t row_static_any(int v, int stage, bool stats, size_t* bytes) {
  const RowOps* o = row_ops_of<R>(v);
  if (!o) return cudaErrorInvalidValue;
  cudaFuncAttributes fa;
  cudaError_t e = cudaFuncGetAttributes(&fa, o->fn[1][row_slot(stage, stats)]);
  if (e == cudaSuccess) *bytes = fa.sharedSizeBytes;
  return e;
}

template <>
cudaError_t launch_row<float>(int v, int stage, bool stats, const RowLaunch& a, int istep, int flags) {
  return launch_row_any<float>(v, stage, stats, a, istep, flags);
}
template <>
cudaError_t launch_row<double>(int v, int stage, bool stats, const RowLaunch& a, int istep, int flags) {
  return launch_row_any<double>(v, stage, stats, a, istep, flags);
}
template <>
cudaError_t row_allow_smem<float>(int v, const size_t* smem6) { return row_allow_any<float>(v, smem6); }
template <>
cudaError_t row_allow_smem<double>(int v, const size_t* smem6) { return row_allow_any<double>(v, smem6); }
template <>
cudaError_t row_occupancy<float>(int v, int stage, size_t smem, int* b) { return row_occ_any<float>(v, stage, smem, b); }
template <>
cudaError_t row_occupancy<double>(int v, int stage, size_t smem, int* b) { return row_occ_any<double>(v, stage, smem, b); }
template <>
cudaError_t row_load<float>(int v) { return row_load_any<float>(v); }
template <>
cudaError_t row_load<double>(int v) { return row_load_any<double>(v); }
template <>
cudaError_t row_static_smem<float>(int v, int stage, bool stats, size_t* b) { return row_static_any<float>(v, stage, stats, b); }
template <>
cudaError_t row_static_smem<double>(int v, int stage, bool stats, size_t* b) { return row_static_any<double>(v, stage, stats, b); }

// ---------------- column shapes ----------------
template <>
cudaError_t launch_col<float>(int v, const ColLaunch& a, int istep, int flags) {
  return col_launch_any<float>(v, a, istep, flags);
}
template <>
cudaError_t launch_col<double>(int v, const ColLaunch& a, int istep, int flags) {
  return col_launch_any<double>(v, a, istep, flags);
}

template <typename R>
static cudaError_t col_allow_any(int v, size_t smem) {
  if (v < 0 || v >= col_variant_count<R>()) return cudaErrorInvalidValue;
  return allow_smem(col_fn_any<R>(v), smem);
}
template <>
cudaError_t col_allow_smem<float>(int v, size_t smem) { return col_allow_any<float>(v, smem); }
template <>
cudaError_t col_allow_smem<double>(int v, size_t smem) { return col_allow_any<double>(v, smem); }

template <typename R>
static cudaError_t col_occ_any(int v, size_t smem, int* blocks) {
  if (v < 0 || v >= col_variant_count<R>()) return cudaErrorInvalidValue;
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks, col_fn_any<R>(v), col_variant<R>(v).block, smem);
}
template <>
cudaError_t col_occupancy<float>(int v, size_t smem, int* blocks) { return col_occ_any<float>(v, smem, blocks); }
template <>
cudaError_t col_occupancy<double>(int v, size_t smem, int* blocks) { return col_occ_any<double>(v, smem, blocks); }

// ---------------- register column kernel shapes (k_creg_*.cu) ----------------
static const ColOps* creg_ops_of(int v) {
  switch (v) {
    case 0: return &creg_ops<0>();
    case 1: return &creg_ops<1>();
    case 2: return &creg_ops<2>();
    default: return nullptr;
  }
}
cudaError_t launch_creg(int v, const ColLaunch& a, int istep, int flags) {
  const ColOps* o = creg_ops_of(v);
  return o ? o->launch(a, istep, flags) : cudaErrorInvalidValue;
}
cudaError_t creg_allow_smem(int v, size_t smem) {
  const ColOps* o = creg_ops_of(v);
  return o ? allow_smem(o->fn, smem) : cudaErrorInvalidValue;
}
cudaError_t creg_occupancy(int v, size_t smem, int* blocks) {
  const ColOps* o = creg_ops_of(v);
  return o ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks, o->fn, kCreg[v].block, smem)
           : cudaErrorInvalidValue;
}
cudaError_t creg_load(int v) {
  const ColOps* o = creg_ops_of(v);
  if (!o) return cudaErrorInvalidValue;
  cudaFuncAttributes fa;
  return cudaFuncGetAttributes(&fa, o->fn);
}

template <typename R>
static cudaError_t col_load_any(int v) {
  if (v < 0 || v >= col_variant_count<R>()) return cudaErrorInvalidValue;
  cudaFuncAttributes fa;
  return cudaFuncGetAttributes(&fa, col_fn_any<R>(v));
}
template <>
cudaError_t col_load<float>(int v) { return col_load_any<float>(v); }
template <>
cudaError_t col_load<double>(int v) { return col_load_any<double>(v); }

}  // namespace mrm
