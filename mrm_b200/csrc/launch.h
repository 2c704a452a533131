// launch.h -- host-side interface between the engine (mrm_gpu.cu) and the
// translation units that compile the row and column kernels (k_row_f32.cu,
// k_row_f64.cu, k_col.cu), so that the heavy kernel instantiations build in
// parallel.  Kernel shapes are compiled variants; the engine picks one per
// launch (default heuristic or the autotuner).
#pragma once
#include <cuda_runtime.h>

#include "common.cuh"

namespace mrm {

// Row kernel shapes: at most `rpb` grid rows per block, `block` threads,
// `minb` resident blocks per SM requested from the register allocator, FFT
// grids of at most 2^lgmax columns (row transforms of 2^(lgmax-1) points).
struct RowVariant {
  int rpb, block, minb, lgmax;
};
constexpr int kRowVariantsF32 = 5;
constexpr RowVariant kRowF32[kRowVariantsF32] = {
    {1, 256, 4, 12}, {1, 128, 8, 12}, {2, 256, 3, 11}, {4, 256, 2, 10}, {8, 256, 2, 8}};
constexpr int kRowVariantsF64 = 3;
constexpr RowVariant kRowF64[kRowVariantsF64] = {{1, 256, 2, 12}, {2, 256, 2, 11}, {8, 256, 1, 8}};
template <typename R>
constexpr int row_variant_count() { return sizeof(R) == sizeof(float) ? kRowVariantsF32 : kRowVariantsF64; }
template <typename R>
constexpr RowVariant row_variant(int v) { return sizeof(R) == sizeof(float) ? kRowF32[v] : kRowF64[v]; }

// Column kernel shapes (the columns per task are chosen at run time).
struct ColVariant {
  int block, minb;
};
constexpr int kColVariantsF32 = 3;
constexpr ColVariant kColF32[kColVariantsF32] = {{256, 3}, {128, 6}, {256, 2}};
constexpr int kColVariantsF64 = 2;
constexpr ColVariant kColF64[kColVariantsF64] = {{256, 1}, {128, 2}};
template <typename R>
constexpr int col_variant_count() { return sizeof(R) == sizeof(float) ? kColVariantsF32 : kColVariantsF64; }
template <typename R>
constexpr ColVariant col_variant(int v) { return sizeof(R) == sizeof(float) ? kColF32[v] : kColF64[v]; }

// Register column kernel shapes (colreg.cuh: FP32 runs of one layer with
// 256..1024-point columns); the column shape index selects one of these for
// those runs and one of kColF32 for the others.
struct CregVariant {
  int block, minb;
};
constexpr int kCregVariants = 3;
constexpr CregVariant kCreg[kCregVariants] = {{128, 4}, {256, 2}, {128, 5}};

struct RowLaunch;
// entry points of one compiled row shape (defined in its own translation unit)
struct RowOps {
  cudaError_t (*launch)(int stage, bool stats, const RowLaunch& a, int istep, int flags);
  // [level][slot]: slots kInit, kPred, kCorr, kCorr with reductions, kEval,
  // kPred with reductions; level 0 fast, 1 general, 2 general with the
  // LLB / MT / Zhang integrators (row_kernel's GEN)
  const void* fn[3][6];
};
template <typename R, int V>
const RowOps& row_ops();
// the kernels of one level of a shape whose levels compile in translation
// units of their own (the FP32 shapes: k_row_f32_v*_g*.cu, assembled into
// row_ops by k_row_split.cu)
struct RowGenOps {
  cudaError_t (*launch)(int stage, bool stats, const RowLaunch& a, int istep, int flags);
  const void* fn[6];
};
template <typename R, int V, int GEN>
const RowGenOps& row_gen_ops();

struct RowLaunch {
  cudaStream_t st;
  const void* runs;  // RunDev<R>[]
  const Task* tasks;
  const void* tw;    // Cx<R> global twiddle table
  double* part;
  int* err;
  int ntasks;
  size_t smem;
  int stage_cap;
  bool pdl;          // programmatic stream serialization with the previous kernel
  int gen;           // the instantiation level (row_kernel's GEN: 1 for llg_type 2/-2, write heads ...,
                     // 2 with the LLB / MT / Zhang integrators)
};

struct ColLaunch {
  cudaStream_t st;
  const void* runs;
  const Task* tasks;
  const void* tw;
  int* err;
  int ntasks;
  size_t smem;
  bool pdl;
  // register column kernel: persistent blocks (0: one per task) and the
  // twiddle entries its shared memory holds
  int blocks = 0;
  int tw_cap = 0;
};

// entry points of one compiled column shape (defined in its own translation unit)
struct ColOps {
  cudaError_t (*launch)(const ColLaunch& a, int istep, int flags);
  const void* fn;
};
template <typename R, int V>
const ColOps& col_ops();
// entry points of one register column kernel shape (k_creg_*.cu)
template <int V>
const ColOps& creg_ops();

// stage: kInit, kPred, kCorr, kEval; stats selects the corrector with reductions
template <typename R>
cudaError_t launch_row(int variant, int stage, bool stats, const RowLaunch& a, int istep, int flags);
// launch slots of the row stages: kInit, kPred, kCorr, kCorr with reductions,
// kEval, kPred with reductions (the single-stage integrator's last step)
constexpr int kRowSlots = 6;
inline int row_slot(int stage, bool stats) {
  return stage == 0 ? 0 : stage == 1 ? (stats ? 5 : 1) : stage == 2 ? (stats ? 3 : 2) : 4;
}
// lets each stage kernel of a variant use smem6[slot] bytes of dynamic shared
// memory on the current device (the limit only grows)
template <typename R>
cudaError_t row_allow_smem(int variant, const size_t* smem6);
template <typename R>
cudaError_t row_occupancy(int variant, int stage, size_t smem, int* blocks_per_sm);
// loads every stage's code (CUDA lazy loading would load it at first launch)
template <typename R>
cudaError_t row_load(int variant);
// static shared memory of a stage (bytes)
template <typename R>
cudaError_t row_static_smem(int variant, int stage, bool stats, size_t* bytes);

template <typename R>
cudaError_t launch_col(int variant, const ColLaunch& a, int istep, int flags);
template <typename R>
cudaError_t col_allow_smem(int variant, size_t smem);
template <typename R>
cudaError_t col_occupancy(int variant, size_t smem, int* blocks_per_sm);
template <typename R>
cudaError_t col_load(int variant);
// the register column kernel (FP32)
cudaError_t launch_creg(int variant, const ColLaunch& a, int istep, int flags);
cudaError_t creg_allow_smem(int variant, size_t smem);
cudaError_t creg_occupancy(int variant, size_t smem, int* blocks_per_sm);
cudaError_t creg_load(int variant);

// launches with or without programmatic stream serialization
template <typename... KArgs, typename... Args>
cudaError_t launch_kernel(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st, bool pdl,
                          Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = pdl ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, kern, static_cast<KArgs>(args)...);
}

// raises a kernel's dynamic shared-memory limit on the current device; the
// limit only grows, so engines sharing a kernel never lower it for each other
cudaError_t allow_smem(const void* kern, size_t bytes);

}  // namespace mrm
