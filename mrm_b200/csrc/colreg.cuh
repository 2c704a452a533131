// colreg.cuh -- register-resident column transform with the tensor product
// (FP32 runs of one layer, FFT columns of 256..1024 points), sm_100a.
//
// The column half of get_demag (src/demag.f90:113-127): for one k_x column
// of the three M^ half spectra, the forward FFT along y, H^ = N^ M^ with the
// FP64-built tensor spectrum, and the inverse FFT along y.  One column is
// transformed by NT = N/8 threads; every thread keeps eight elements of each
// of the three components in registers through the whole transform:
//
//   stage 0 (global -> registers): thread t loads rows t + k NT, k < 8 (the
//       zero padding of an open boundary, rows >= N/2, is neither loaded nor
//       transformed), radix-2^R0 butterflies over the top position bits;
//   stages 1..S-1: radix-8 butterflies, each preceded by an exchange of the
//       elements through shared memory (one barrier of the column's threads);
//   after the last forward stage thread t holds positions 8t..8t+7 of the
//       mixed-radix digit-reversed order (fft.cuh ip_freq) and multiplies them
//       by the tensor in registers (the tensor is stored in that order);
//   the inverse stages run in the reverse order (decimation in time) and the
//       last one writes rows < ny of H^ straight to global memory.
//
// Positions, radices and twiddle tables are those of the in-place passes of
// fft.cuh (the same Cooley-Tukey plan, the same tables), so both column
// kernels compute the same transform.  Exchange buffer: the three components
// of a column, N elements each, at swizzled offsets xswz(p).
#pragma once
#include "kernels.cuh"

namespace mrm {

constexpr int kCregMinLg = 8, kCregMaxLg = 10;

// A stage over the three components in the column's buffer: each component's
// eight elements at the thread's positions of the stage are read, transformed
// and written back in place (no other thread touches them in this stage).
template <int LGN, int STAGE, bool INV>
MRM_D void creg_stage(Cx<float>* __restrict__ buf, int t, const Cx<float>* __restrict__ tw) {
  using P = RegPlan<LGN>;
  constexpr int B = P::dbit(STAGE);
  Cx<float> w[8];
  reg_twiddles<LGN, STAGE>(w, t, tw);
  const int a = xswz(reg_base<B>(t));
#pragma unroll 1
  for (int q = 0; q < 3; ++q) {
    Cx<float>* b = buf + q * P::N;
    Cx<float> v[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) v[k] = b[a ^ xswz(k << B)];
    if constexpr (INV) reg_inv<LGN, STAGE>(v, w);
    else reg_fwd<LGN, STAGE, false>(v, w);
#pragma unroll
    for (int k = 0; k < 8; ++k) b[a ^ xswz(k << B)] = v[k];
  }
}

// The column's tensor at the thread's product positions 8t..8t+7: six
// components (xx, yy, zz, xy, xz, yz) of N reals in position order per k_x
// column; the xz and yz spectra are imaginary (the stored real times i) and
// the sign of the odd components in the upper half of k_y is folded in.
// Loaded at the start of a column's transform, used by its product.
struct CregTensor {
  float4 t[6][2];
};
MRM_D void creg_tensor_load(CregTensor& T, const float* __restrict__ tk, int t, int n) {
#pragma unroll
  for (int c = 0; c < 6; ++c)
#pragma unroll
    for (int h = 0; h < 2; ++h) T.t[c][h] = __ldg(reinterpret_cast<const float4*>(tk + (size_t)c * n + 8 * t) + h);
}

// H^ = N^ M^ at the thread's positions 8t..8t+7 (the last stage's positions)
// of the column's buffer.
template <int LGN>
MRM_D void creg_product(Cx<float>* __restrict__ buf, const CregTensor& T, int t) {
  constexpr int N = 1 << LGN;
  const int a = xswz(t << 3);
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const int at = a ^ k;  // xswz(k) = k for k < 8
    const int h = k >> 2, i = k & 3;
    auto comp = [&](int c) {
      const float4& v = T.t[c][h];
      return i == 0 ? v.x : i == 1 ? v.y : i == 2 ? v.z : v.w;
    };
    const float xx = comp(0), yy = comp(1), zz = comp(2), xy = comp(3), xz = comp(4), yz = comp(5);
    const Cx<float> mx = buf[at], my = buf[N + at], mz = buf[2 * N + at];
    buf[at] = Cx<float>{fmaf(xx, mx.x, fmaf(xy, my.x, -xz * mz.y)), fmaf(xx, mx.y, fmaf(xy, my.y, xz * mz.x))};
    buf[N + at] = Cx<float>{fmaf(xy, mx.x, fmaf(yy, my.x, -yz * mz.y)), fmaf(xy, mx.y, fmaf(yy, my.y, yz * mz.x))};
    buf[2 * N + at] = Cx<float>{fmaf(zz, mz.x, -fmaf(xz, mx.y, yz * my.y)), fmaf(zz, mz.y, fmaf(xz, mx.x, yz * my.x))};
  }
}

// Shared memory of a block of BLOCK threads: the column pass tables (room
// for tw_cap entries, the longest columns of the launch), the exchange
// buffers (three components of every column of the block: 3 N (BLOCK / (N/8))
// = 24 BLOCK elements whatever N), then the staging area of one M^ tile.
MRM_HD constexpr int creg_cols(int lgpy, int block) { return block >> (lgpy - 3); }
MRM_HD constexpr int creg_xb_count(int block) { return 24 * block; }
MRM_HD constexpr int creg_stage_bytes(int nys, int lgct) { return 3 * (nys << lgct) * (int)sizeof(Cx<float>); }
MRM_HD constexpr int creg_smem(int tw_cap, int block, int stage_bytes) {
  return (tw_cap + creg_xb_count(block)) * (int)sizeof(Cx<float>) + stage_bytes;
}

// The column c of a task (global column k): forward transform, product,
// inverse transform.  stg: the task's M^ tile staged in shared memory
// ([plane][nys][T]); after every thread has its stage-0 elements in
// registers, `staged_read` runs (the block then may reuse the staging area);
// live: c is one of the task's columns (the others take part in the barriers
// only).
template <int LGN, bool HALF, class AFTER>
MRM_D void creg_body(const RunDev<float>& rd, int k, int t, int c, bool live, const Cx<float>* __restrict__ tw,
                     const Cx<float>* __restrict__ stg, Cx<float>* __restrict__ buf, const AFTER& staged_read) {
  using P = RegPlan<LGN>;
  constexpr int N = P::N, NT = P::NT, KIN = HALF ? 4 : 8;
  constexpr int B0 = P::dbit(0);
  const int ny = rd.ny, lgct = rd.lgct, cs = k & ((1 << lgct) - 1);
  const int pstride = rd.nys << lgct;
  Cx<float>* const spech = rd.spech;
  const int phs = rd.phs;
  // stage 0 from the staged tile: rows t + kk NT of every component
  Cx<float> v0[3][KIN];
#pragma unroll
  for (int q = 0; q < 3; ++q)
#pragma unroll
    for (int kk = 0; kk < KIN; ++kk) {
      const int j = t + kk * NT;
      v0[q][kk] = j < ny ? stg[q * pstride + (j << lgct) + cs] : Cx<float>{0.f, 0.f};
    }
  __syncthreads();
  staged_read();
  {
    Cx<float> w[8];
    reg_twiddles<LGN, 0>(w, t, tw);
    const int a = xswz(reg_base<B0>(t));
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      Cx<float> v[8];
#pragma unroll
      for (int kk = 0; kk < 8; ++kk) v[kk] = kk < KIN ? v0[q][kk] : Cx<float>{0.f, 0.f};
      reg_fwd<LGN, 0, HALF>(v, w);
#pragma unroll
      for (int kk = 0; kk < 8; ++kk) buf[q * N + (a ^ xswz(kk << B0))] = v[kk];
    }
  }
  // the tensor slice: its loads land during the remaining forward stages
  reg_sync<NT>(c);
  creg_stage<LGN, 1, false>(buf, t, tw);
  reg_sync<NT>(c);
  creg_stage<LGN, 2, false>(buf, t, tw);
  if constexpr (P::S == 4) {
    reg_sync<NT>(c);
    creg_stage<LGN, 3, false>(buf, t, tw);
  }
  // the last stage's positions are the thread's own: no barrier before the product
  if (live) {
    CregTensor T;
    creg_tensor_load(T, rd.tens + (size_t)k * 6 * N, t, N);
    creg_product<LGN>(buf, T, t);
  }
  if constexpr (P::S == 4) {
    creg_stage<LGN, 3, true>(buf, t, tw);
    reg_sync<NT>(c);
  }
  creg_stage<LGN, 2, true>(buf, t, tw);
  reg_sync<NT>(c);
  creg_stage<LGN, 1, true>(buf, t, tw);
  reg_sync<NT>(c);
  if (live) {
    // inverse stage 0 and the H^ rows, row-major [plane][ny][phs]
    Cx<float> w[8];
    reg_twiddles<LGN, 0>(w, t, tw);
    const int a = xswz(reg_base<B0>(t));
    Cx<float>* dst = spech + k;
#pragma unroll 1
    for (int q = 0; q < 3; ++q) {
      Cx<float> v[8];
#pragma unroll
      for (int kk = 0; kk < 8; ++kk) v[kk] = buf[q * N + (a ^ xswz(kk << B0))];
      reg_inv<LGN, 0>(v, w);
#pragma unroll
      for (int kk = 0; kk < KIN; ++kk) {
        const int j = t + kk * NT;
        if (j < ny) dst[((size_t)q * ny + j) * phs] = v[kk];
      }
    }
  }
  // the buffers are free for the block's next task
  __syncthreads();
}

template <int LGN, int BLOCK, class AFTER>
MRM_D void creg_column(const RunDev<float>& rd, int k0, int nc, const Cx<float>* tw, Cx<float>* xb,
                       const Cx<float>* stg, const AFTER& staged_read) {
  using P = RegPlan<LGN>;
  static_assert(P::NT <= BLOCK && BLOCK % P::NT == 0, "a block holds whole columns");
  static_assert(P::NT >= 32, "a column is one or more whole warps");
  static_assert(P::NT == 32 || BLOCK / P::NT <= 4, "named barriers 1..4");
  const int c = threadIdx.x / P::NT, t = threadIdx.x % P::NT;
  const bool live = c < nc;
  Cx<float>* buf = xb + c * 3 * P::N;
  if (rd.py >= 2 * rd.ny) creg_body<LGN, true>(rd, k0 + c, t, c, live, tw, stg, buf, staged_read);
  else creg_body<LGN, false>(rd, k0 + c, t, c, live, tw, stg, buf, staged_read);
}

// A task (run, first column k0, columns nc <= BLOCK / (py/8), all in one M^
// tile) is checked against the compiled shape and the launch's shared memory.
MRM_D bool creg_task_ok(const RunDev<float>& rd, int k0, int nc, int block, int tw_cap, int stage_cap) {
  const int lgpy = rd.lgpy, T = 1 << rd.lgct, ph = (rd.px >> 1) + 1;
  return lgpy >= kCregMinLg && lgpy <= kCregMaxLg && rd.nl == 1 && nc >= 1 && k0 >= 0 && k0 + nc <= ph &&
         nc <= creg_cols(lgpy, block) && (k0 & (T - 1)) == 0 && nc <= T && col_tw_count(lgpy) <= tw_cap &&
         creg_stage_bytes(rd.nys, rd.lgct) <= stage_cap;
}

// Persistent blocks: block b takes tasks b, b + G, b + 2G, ... (G blocks).
// While a task is transformed, the next task's M^ tile is already on its way
// into the staging area (a bulk copy issued as soon as every thread has read
// the current tile), and each thread's tensor values are loaded at the start
// of its column, so neither input is waited for.  The twiddles are copied
// again only when the next task's column length differs.
template <int BLOCK, int MINB>
__global__ void __launch_bounds__(BLOCK, MINB) creg_kernel(const RunDev<float>* __restrict__ runs,
                                                           const Task* __restrict__ tasks, int ntasks,
                                                           const Cx<float>* __restrict__ twg, int istep, int flags,
                                                           int tw_cap, int* __restrict__ err) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ uint64_t bars[2];  // 0: twiddles, 1: the staged tile
  pdl_launch_dependents();
  Cx<float>* tws = reinterpret_cast<Cx<float>*>(smem_raw);
  Cx<float>* xb = tws + tw_cap;
  Cx<float>* stg = xb + creg_xb_count(BLOCK);
  const int stage_cap = (int)dynamic_smem_bytes() - (tw_cap + creg_xb_count(BLOCK)) * (int)sizeof(Cx<float>);
  if (threadIdx.x == 0) {
    mbar_init(&bars[0], 1);
    mbar_init(&bars[1], 1);
    mbar_fence_init();
  }
  __syncthreads();
  pdl_wait();  // every task's M^ tile comes from the previous kernel
  // a task's work: live (active run with demag, step within its budget) and shape-checked
  auto live_task = [&](int i) -> bool {
    const Task tk = tasks[i];
    const RunDev<float>& rd = runs[tk.x];
    if (!rd.active || !rd.demag) return false;
    return (flags & kFlagForce) || step_due(rd, rd.step + istep);
  };
  // thread 0: the tile of task i into the staging area (nothing for a task
  // without work), completing phase `ph` of bars[1]
  auto start_tile = [&](int i) {
    const Task tk = tasks[i];
    const RunDev<float>& rd = runs[tk.x];
    if (live_task(i) && creg_task_ok(rd, tk.y, tk.z, BLOCK, tw_cap, stage_cap)) {
      const int lgct = rd.lgct, T = 1 << lgct, ph = (rd.px >> 1) + 1, ntile = (ph + T - 1) >> lgct;
      const int plane = rd.nys << lgct;
      const Cx<float>* src = rd.specx + (((size_t)(tk.y >> lgct) * rd.nys) << lgct);
      const size_t pstride = ((size_t)ntile * rd.nys) << lgct;
      for (int q = 0; q < 3; ++q)
        bulk_copy(&bars[1], stg + q * plane, src + q * pstride, (uint32_t)(plane * sizeof(Cx<float>)));
    }
    mbar_arrive(&bars[1]);
  };
  int i = blockIdx.x;
  if (i >= ntasks) return;
  if (threadIdx.x == 0) start_tile(i);
  uint32_t tile_phase = 0, tw_phase = 0;
  int tw_lg = -1;
  for (; i < ntasks; i += gridDim.x) {
    const int nxt = i + gridDim.x;
    const Task tk = tasks[i];
    const RunDev<float>& rd = runs[tk.x];
    const bool work = live_task(i);
    const bool shape_ok = creg_task_ok(rd, tk.y, tk.z, BLOCK, tw_cap, stage_cap);
    if (work && !shape_ok && threadIdx.x == 0) atomicOr(err, kErrShape);
    const int lgpy = rd.lgpy;
    if (work && shape_ok && lgpy != tw_lg) {
      // (re)load the pass tables of this column length: the previous task's
      // threads are past their last use (the body ends with a block barrier)
      if (threadIdx.x == 0) {
        bulk_copy(&bars[0], tws, twg + rd.tw_col, (uint32_t)(col_tw_count(lgpy) * sizeof(Cx<float>)));
        mbar_arrive(&bars[0]);
      }
      const bool ok = mbar_wait(&bars[0], tw_phase);
      tw_phase ^= 1;
      tw_lg = lgpy;
      if (__syncthreads_or(!ok)) {
        if (threadIdx.x == 0) atomicOr(err, kErrBarrierTimeout);
        mbar_wait(&bars[0], tw_phase ^ 1);
        mbar_wait(&bars[1], tile_phase);
        return;
      }
    }
    const bool ok = mbar_wait(&bars[1], tile_phase);
    tile_phase ^= 1;
    if (__syncthreads_or(!ok)) {
      if (threadIdx.x == 0) atomicOr(err, kErrBarrierTimeout);
      mbar_wait(&bars[1], tile_phase ^ 1);
      return;
    }
    auto next_tile = [&]() {
      if (threadIdx.x == 0 && nxt < ntasks) start_tile(nxt);
    };
    if (!(work && shape_ok)) {
      // the staging area was not written: the next tile may start at once
      __syncthreads();
      next_tile();
      continue;
    }
    switch (lgpy) {
      case 8: creg_column<8, BLOCK>(rd, tk.y, tk.z, tws, xb, stg, next_tile); break;
      case 9: creg_column<9, BLOCK>(rd, tk.y, tk.z, tws, xb, stg, next_tile); break;
      default: creg_column<10, BLOCK>(rd, tk.y, tk.z, tws, xb, stg, next_tile); break;
    }
  }
}

}  // namespace mrm
