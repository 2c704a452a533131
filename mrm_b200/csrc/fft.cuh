// fft.cuh -- block-cooperative Stockham FFTs in shared memory (sm_100a).
//
// Replaces the FFTW r2c/c2r plans of src/fftw.f90:37-93 (unnormalised,
// forward sign -1).  Two forms:
//
//  * the hot-path form (block_fft_c): every length, pass, stride and twiddle
//    offset is a compile-time constant.  A batch of nb complex sequences of
//    length n = 2^lgn, sequence b at buf + b*seq_stride(n), is transformed by
//    radix-8 passes plus one radix-2/4 pass for the remaining bits (Stockham
//    autosort: natural-order result, ping-pong between two buffers, one
//    __syncthreads per pass).  Intermediate passes use the swizzled layout
//    swz(i) = i ^ ((i >> 3) & 15), a permutation inside each group of 16
//    elements under which the stride-8 stores of the first pass, the runs of
//    8 of the second and the contiguous loads all touch distinct banks; the
//    input of the first pass and the output of the last are natural order.
//    Each pass reads its twiddles from its own table, entry (r-1)*Ns + k =
//    e^{-2 pi i k r / (Ns R)}, so a warp reads consecutive entries.
//  * the run-time form (block_fft): sizes at run time, padded layout, twiddles
//    from the 4096-entry table; used by the once-per-run FP64 tensor FFT.
#pragma once
#include "common.cuh"

namespace mrm {

// ---------------- hot-path form ----------------

MRM_HD constexpr int swz(int i) { return i ^ ((i >> 3) & 15); }
// complex stride of one sequence of length n in the hot-path buffers (even,
// so that every sequence starts 16-byte aligned in FP32)
MRM_HD constexpr int seq_stride(int n) { return n == 64 ? n + 8 : n + 2; }

// radix plan of length 2^lgn: passes of 3 bits, the last takes the remaining 1..3
MRM_HD constexpr int pass_lgr(int lgn, int lgns) { return (lgn - lgns) >= 3 ? 3 : lgn - lgns; }
// twiddles of all passes of a length-2^lgn transform
MRM_HD constexpr int pass_tw_count(int lgn) {
  int total = 0, lgns = 0;
  while (lgns < lgn) {
    const int lgr = pass_lgr(lgn, lgns);
    if (lgns > 0) total += ((1 << lgr) - 1) << lgns;
    lgns += lgr;
  }
  return total;
}
MRM_HD constexpr int even_up(int x) { return (x + 1) & ~1; }
// Row-kernel twiddle block for an FFT grid of 2^lgpx columns (real transform
// of length px through a complex one of length M = px/2): the post/pre-
// processing twiddles e^{-2 pi i k/px}, k <= M (padded to even), then the
// pass tables of the length-M transform.
MRM_HD constexpr int row_tw_post(int lgpx) { return even_up((1 << (lgpx - 1)) + 1); }
MRM_HD constexpr int row_tw_count(int lgpx) { return row_tw_post(lgpx) + even_up(pass_tw_count(lgpx - 1)); }
// Column-kernel twiddle block for 2^lgpy rows: the pass tables of that length.
MRM_HD constexpr int col_tw_count(int lgpy) { return even_up(pass_tw_count(lgpy)); }
// offsets of the blocks in the global table: row blocks for lg = 1..kTwLog, then column blocks
MRM_HD constexpr int row_tw_off(int lgpx) {
  int o = 0;
  for (int l = 1; l < lgpx; ++l) o += row_tw_count(l);
  return o;
}
MRM_HD constexpr int col_tw_off(int lgpy) {
  int o = row_tw_off(kTwLog + 1);
  for (int l = 1; l < lgpy; ++l) o += col_tw_count(l);
  return o;
}
MRM_HD constexpr int tw_table_size() { return col_tw_off(kTwLog + 1); }

template <typename R, int S>
MRM_D void dft2(Cx<R>* v) {
  Cx<R> a = v[0], b = v[1];
  v[0] = cadd(a, b);
  v[1] = csub(a, b);
}

template <typename R, int S>
MRM_D void dft4(Cx<R>& a0, Cx<R>& a1, Cx<R>& a2, Cx<R>& a3) {
  // S = -1 forward, +1 inverse
  Cx<R> t0 = cadd(a0, a2), t1 = csub(a0, a2), t2 = cadd(a1, a3);
  Cx<R> t3 = cmul_i(csub(a1, a3), (R)S);
  a0 = cadd(t0, t2);
  a2 = csub(t0, t2);
  a1 = cadd(t1, t3);
  a3 = csub(t1, t3);
}

template <typename R, int S>
MRM_D void dft8(Cx<R>* v) {
  Cx<R> e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
  Cx<R> o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
  dft4<R, S>(e0, e1, e2, e3);
  dft4<R, S>(o0, o1, o2, o3);
  const R h = (R)0.70710678118654752440084436210485;
  // w8^k = e^{S*2*pi*i*k/8}
  const Cx<R> w1 = {h, (R)S * h}, w3 = {-h, (R)S * h};
  o1 = cmul(o1, w1);
  o2 = cmul_i(o2, (R)S);
  o3 = cmul(o3, w3);
  v[0] = cadd(e0, o0);
  v[4] = csub(e0, o0);
  v[1] = cadd(e1, o1);
  v[5] = csub(e1, o1);
  v[2] = cadd(e2, o2);
  v[6] = csub(e2, o2);
  v[3] = cadd(e3, o3);
  v[7] = csub(e3, o3);
}

// One Stockham pass with every size known at compile time.  LGN: log2
// length; LGR: log2 radix; LGNS: log2 of the sub-transform length so far;
// OFF: offset of this pass's table in the pass tables; PIN/POUT: swizzled
// input/output; NBMAX: upper bound of nb (0: none, run-time loop); BLOCK:
// threads of the block.
template <typename R, int LGN, int LGR, int LGNS, int OFF, bool PIN, bool POUT, int S, int NBMAX, int BLOCK>
MRM_D void stockham_pass_c(const Cx<R>* __restrict__ in, Cx<R>* __restrict__ out, int nb,
                           const Cx<R>* __restrict__ twp) {
  constexpr int RADIX = 1 << LGR;
  constexpr int LGNR = LGN - LGR;
  constexpr int NR = 1 << LGNR;
  constexpr int NS = 1 << LGNS;
  constexpr int STRIDE = seq_stride(1 << LGN);
  const int total = nb << LGNR;
  auto body = [&](int q) {
    const int b = q >> LGNR, j = q & (NR - 1);
    const Cx<R>* src = in + b * STRIDE;
    Cx<R>* dst = out + b * STRIDE;
    Cx<R> v[RADIX];
#pragma unroll
    for (int r = 0; r < RADIX; ++r) {
      const int i = j + r * NR;
      v[r] = src[PIN ? swz(i) : i];
    }
    const int k = j & (NS - 1);
    if constexpr (LGNS > 0) {
#pragma unroll
      for (int r = 1; r < RADIX; ++r) {
        Cx<R> w = twp[OFF + (r - 1) * NS + k];
        if (S > 0) w.y = -w.y;
        v[r] = cmul(v[r], w);
      }
    }
    if constexpr (RADIX == 8) dft8<R, S>(v);
    else if constexpr (RADIX == 4) dft4<R, S>(v[0], v[1], v[2], v[3]);
    else dft2<R, S>(v);
    const int idxD = ((j >> LGNS) << (LGNS + LGR)) + k;
#pragma unroll
    for (int r = 0; r < RADIX; ++r) {
      const int i = idxD + r * NS;
      dst[POUT ? swz(i) : i] = v[r];
    }
  };
  constexpr int ITERS = NBMAX > 0 ? ((NBMAX << LGNR) + BLOCK - 1) / BLOCK : 0;
  if constexpr (NBMAX > 0 && ITERS <= 2) {
#pragma unroll
    for (int it = 0; it < ITERS; ++it) {
      const int q = threadIdx.x + it * BLOCK;
      if (q < total) body(q);
    }
  } else {
#pragma unroll 1
    for (int q = threadIdx.x; q < total; q += BLOCK) body(q);
  }
}

// Radix-8 plan of length 2^LGN unrolled at compile time.  Pass P reads the
// swizzled layout when P > 0 and writes it unless it is the last pass.
template <typename R, int LGN, int S, int P, int LGNS, int OFF, int NBMAX, int BLOCK>
MRM_D Cx<R>* fft_c_from(Cx<R>* a, Cx<R>* b, int nb, const Cx<R>* __restrict__ twp) {
  constexpr int REM = LGN - LGNS;
  if constexpr (REM <= 0) {
    return a;
  } else {
    constexpr int LGR = REM >= 3 ? 3 : REM;
    constexpr bool LAST = (REM - LGR) == 0;
    stockham_pass_c<R, LGN, LGR, LGNS, OFF, (P > 0), !LAST, S, NBMAX, BLOCK>(a, b, nb, twp);
    __syncthreads();
    constexpr int NEXT_OFF = OFF + (LGNS > 0 ? ((1 << LGR) - 1) << LGNS : 0);
    return fft_c_from<R, LGN, S, P + 1, LGNS + LGR, NEXT_OFF, NBMAX, BLOCK>(b, a, nb, twp);
  }
}

// Transforms nb sequences held (natural order) in `a`, sequence stride
// seq_stride(n); `b` is scratch of the same size; twp: the pass tables of
// length 2^lgn.  Returns the buffer holding the (natural-order) result.  The
// caller must __syncthreads() before the call.  Lengths above 2^LGMAX are
// not compiled in (the caller checks lgn <= LGMAX).
template <typename R, int S, int NBMAX, int BLOCK, int LGMAX = 12>
MRM_D Cx<R>* block_fft_c(Cx<R>* a, Cx<R>* b, int lgn, int nb, const Cx<R>* __restrict__ twp) {
  switch (lgn) {
    case 1: return fft_c_from<R, 1, S, 0, 0, 0, NBMAX, BLOCK>(a, b, nb, twp);
    case 2: return fft_c_from<R, 2, S, 0, 0, 0, NBMAX, BLOCK>(a, b, nb, twp);
    case 3: return fft_c_from<R, 3, S, 0, 0, 0, NBMAX, BLOCK>(a, b, nb, twp);
    case 4: return fft_c_from<R, 4, S, 0, 0, 0, NBMAX, BLOCK>(a, b, nb, twp);
    case 5: return fft_c_from<R, 5, S, 0, 0, 0, NBMAX, BLOCK>(a, b, nb, twp);
    case 6: return fft_c_from<R, 6, S, 0, 0, 0, NBMAX, BLOCK>(a, b, nb, twp);
    case 7: if constexpr (LGMAX >= 7) return fft_c_from<R, 7, S, 0, 0, 0, NBMAX, BLOCK>(a, b, nb, twp); else return a;
    case 8: if constexpr (LGMAX >= 8) return fft_c_from<R, 8, S, 0, 0, 0, NBMAX, BLOCK>(a, b, nb, twp); else return a;
    case 9: if constexpr (LGMAX >= 9) return fft_c_from<R, 9, S, 0, 0, 0, NBMAX, BLOCK>(a, b, nb, twp); else return a;
    case 10: if constexpr (LGMAX >= 10) return fft_c_from<R, 10, S, 0, 0, 0, NBMAX, BLOCK>(a, b, nb, twp); else return a;
    case 11: if constexpr (LGMAX >= 11) return fft_c_from<R, 11, S, 0, 0, 0, NBMAX, BLOCK>(a, b, nb, twp); else return a;
    default: if constexpr (LGMAX >= 12) return fft_c_from<R, 12, S, 0, 0, 0, NBMAX, BLOCK>(a, b, nb, twp); else return a;
  }
}

// ---------------- in-place form (column kernel) ----------------
//
// Cooley-Tukey passes that overwrite their own inputs, so one buffer holds a
// transform.  The forward transform decimates in frequency (butterfly, then
// twiddles) from natural order to the mixed-radix digit-reversed order of
// ip_freq(); the inverse decimates in time (twiddles, then butterfly) from that
// order back to natural order, so a pointwise product between the two needs no
// reordering.  The passes are the Stockham plan's (same radices, same tables):
// pass (LGNS, LGR) combines the elements blk*L + j0 + m*S (S = 2^LGNS,
// L = S*2^LGR, j0 < S, m < 2^LGR) with the twiddles e^{-2 pi i j0 m / L}, table
// entry (m-1)*S + j0; the forward transform runs the passes from the largest S
// down, the inverse from S = 1 up.  Elements are read and written through the
// caller's functors ld(h, c, j) / st(h, c, j, v) (h: sequence group, c: column
// within a tile of 2^lgT columns, j: element), so the first forward pass can
// read global memory and the last inverse pass write it.  Consecutive threads
// take consecutive columns c, then consecutive butterflies.

// S of the pass the forward transform of length 2^lgn starts with (its radix takes the remaining bits)
MRM_HD constexpr int ip_top(int lgn) { return 3 * ((lgn - 1) / 3); }

// frequency held at position p after the in-place forward transform of length 2^lgn
MRM_HD constexpr int ip_freq(int p, int lgn) {
  int k = 0, shift = 0, lgns = ip_top(lgn), lgr = lgn - lgns;
  while (true) {
    k |= ((p >> lgns) & ((1 << lgr) - 1)) << shift;
    shift += lgr;
    if (lgns == 0) break;
    lgns -= 3;
    lgr = 3;
  }
  return k;
}

// offset of the pass with sub-length 2^lgns_at in the pass tables of length 2^lgn
MRM_HD constexpr int pass_tw_off(int lgn, int lgns_at) {
  int total = 0, lgns = 0;
  while (lgns < lgns_at) {
    const int lgr = pass_lgr(lgn, lgns);
    if (lgns > 0) total += ((1 << lgr) - 1) << lgns;
    lgns += lgr;
  }
  return total;
}

template <typename R, int S, int RADIX>
MRM_D void dft_r(Cx<R>* v) {
  if constexpr (RADIX == 8) dft8<R, S>(v);
  else if constexpr (RADIX == 4) dft4<R, S>(v[0], v[1], v[2], v[3]);
  else dft2<R, S>(v);
}

// Element access of the in-place passes.  An accessor maps the butterfly
// start (h: sequence group, c: column within a tile of 2^lgT columns, base:
// element index) to a pointer and gives the element stride of a pass of span
// NS, so the 2^LGR elements base + m*NS of a butterfly sit at ptr + m*stride:
//   ptr(h, c, base), stride(NS), valid(j) (false: the element is outside the
//   data: read as zero, not written).
// One in-place pass over nh sequence groups (columns c >= nc skipped).  HALF:
// the upper half of the elements (m >= RADIX/2) is zero on input (forward) or
// not wanted on output (inverse); set only on the pass that spans the whole
// length, where m alone decides j >= 2^LGN / 2.
template <typename R, int LGN, int LGNS, bool INV, bool HALF, int BLOCK, class IN, class OUT>
MRM_D void ip_pass(int lgT, int nc, int nh, const Cx<R>* __restrict__ twp, const IN& in, const OUT& out) {
  constexpr int LGR = pass_lgr(LGN, LGNS);
  constexpr int RADIX = 1 << LGR, NS = 1 << LGNS, LGB = LGN - LGR;
  constexpr int OFF = pass_tw_off(LGN, LGNS);
  constexpr int MIN = HALF && !INV ? RADIX / 2 : RADIX;  // inputs that can be non-zero
  constexpr int MOUT = HALF && INV ? RADIX / 2 : RADIX;  // outputs that are stored
  static_assert(!HALF || LGNS + LGR == LGN, "HALF applies to the pass spanning the whole length");
  const int total = nh << (LGB + lgT);
  const int tmask = (1 << lgT) - 1;
  const int es_in = in.stride(NS), es_out = out.stride(NS);
  for (int q = threadIdx.x; q < total; q += BLOCK) {
    const int c = q & tmask;
    if (c >= nc) continue;
    const int bf = (q >> lgT) & ((1 << LGB) - 1), h = q >> (LGB + lgT);
    const int j0 = bf & (NS - 1), base = ((bf >> LGNS) << (LGNS + LGR)) + j0;
    Cx<R> v[RADIX];
    {
      const Cx<R>* pi = in.ptr(h, c, base);
#pragma unroll
      for (int m = 0; m < RADIX; ++m)
        v[m] = (m < MIN && in.valid(base + m * NS)) ? pi[m * es_in] : Cx<R>{(R)0, (R)0};
    }
    if constexpr (INV && LGNS > 0) {
#pragma unroll
      for (int m = 1; m < RADIX; ++m) v[m] = cmul(v[m], cconj(twp[OFF + (m - 1) * NS + j0]));
    }
    dft_r<R, INV ? 1 : -1, RADIX>(v);
    if constexpr (!INV && LGNS > 0) {
#pragma unroll
      for (int m = 1; m < RADIX; ++m) v[m] = cmul(v[m], twp[OFF + (m - 1) * NS + j0]);
    }
    Cx<R>* po = out.ptr(h, c, base);
#pragma unroll
    for (int m = 0; m < MOUT; ++m)
      if (out.valid(base + m * NS)) po[m * es_out] = v[m];
  }
}

// forward passes LGNS, LGNS-3, ..., 0 through acc, each followed by __syncthreads
template <typename R, int LGN, int LGNS, int BLOCK, class ACC>
MRM_D void ip_fwd_from(int lgT, int nc, int nh, const Cx<R>* __restrict__ twp, const ACC& acc) {
  ip_pass<R, LGN, LGNS, false, false, BLOCK>(lgT, nc, nh, twp, acc, acc);
  __syncthreads();
  if constexpr (LGNS >= 3) ip_fwd_from<R, LGN, LGNS - 3, BLOCK>(lgT, nc, nh, twp, acc);
}
// inverse passes LGNS, LGNS+3, ..., top; the top one writes through last (no barrier after it)
template <typename R, int LGN, int LGNS, bool HALF, int BLOCK, class ACC, class LAST>
MRM_D void ip_inv_from(int lgT, int nc, int nh, const Cx<R>* __restrict__ twp, const ACC& acc, const LAST& last) {
  if constexpr (LGNS == ip_top(LGN)) {
    ip_pass<R, LGN, LGNS, true, HALF, BLOCK>(lgT, nc, nh, twp, acc, last);
  } else {
    ip_pass<R, LGN, LGNS, true, false, BLOCK>(lgT, nc, nh, twp, acc, acc);
    __syncthreads();
    ip_inv_from<R, LGN, LGNS + 3, HALF, BLOCK>(lgT, nc, nh, twp, acc, last);
  }
}

// Forward transform of length 2^LGN: the first pass reads through first, the
// rest through acc; every pass writes through acc; ends with __syncthreads.
// HALF: elements j >= 2^LGN / 2 are zero (not read).  The caller must
// __syncthreads() before the call if first reads shared memory.
template <typename R, int LGN, bool HALF, int BLOCK, class FIRST, class ACC>
MRM_D void ip_fft_fwd(int lgT, int nc, int nh, const Cx<R>* __restrict__ twp, const FIRST& first, const ACC& acc) {
  constexpr int TOP = ip_top(LGN);
  ip_pass<R, LGN, TOP, false, HALF, BLOCK>(lgT, nc, nh, twp, first, acc);
  __syncthreads();
  if constexpr (TOP >= 3) ip_fwd_from<R, LGN, TOP - 3, BLOCK>(lgT, nc, nh, twp, acc);
}
// Inverse transform of length 2^LGN (unnormalised) from digit-reversed order:
// every pass reads through acc, the last writes through last and the others
// through acc.  HALF: only elements j < 2^LGN / 2 are written by the last pass.
// The caller must __syncthreads() before the call.
template <typename R, int LGN, bool HALF, int BLOCK, class ACC, class LAST>
MRM_D void ip_fft_inv(int lgT, int nc, int nh, const Cx<R>* __restrict__ twp, const ACC& acc, const LAST& last) {
  ip_inv_from<R, LGN, 0, HALF, BLOCK>(lgT, nc, nh, twp, acc, last);
}

// ---------------- run-time form (tensor FFT) ----------------

MRM_HD int pad_stride(int n) { return n + (n >> 4) + 1; }
MRM_D int padi(int i) { return i + (i >> 4); }

// One Stockham pass.  PIN / POUT: input / output use the padded layout.
template <typename R, int RADIX, int LGR, int S>
MRM_D void stockham_pass(const Cx<R>* __restrict__ in, Cx<R>* __restrict__ out, int lgn, int nb,
                         int stride, int lgNs, bool pin, bool pout, const Cx<R>* __restrict__ tw,
                         int lgtw) {
  const int lgnR = lgn - LGR;
  const int nR = 1 << lgnR;
  const int Ns = 1 << lgNs;
  const int total = nb << lgnR;
  for (int q = threadIdx.x; q < total; q += blockDim.x) {
    const int b = q >> lgnR, j = q & (nR - 1);
    const Cx<R>* src = in + b * stride;
    Cx<R>* dst = out + b * stride;
    Cx<R> v[RADIX];
#pragma unroll
    for (int r = 0; r < RADIX; ++r) {
      const int i = j + r * nR;
      v[r] = src[pin ? padi(i) : i];
    }
    const int k = j & (Ns - 1);
    if (lgNs > 0) {
      const int sh = lgtw - lgNs - LGR;
#pragma unroll
      for (int r = 1; r < RADIX; ++r) {
        Cx<R> w = tw[(r * k) << sh];
        if (S > 0) w.y = -w.y;
        v[r] = cmul(v[r], w);
      }
    }
    if (RADIX == 8) dft8<R, S>(v);
    else if (RADIX == 4) dft4<R, S>(v[0], v[1], v[2], v[3]);
    else dft2<R, S>(v);
    const int idxD = ((j >> lgNs) << (lgNs + LGR)) + k;
#pragma unroll
    for (int q2 = 0; q2 < RADIX; ++q2) {
      const int i = idxD + q2 * Ns;
      dst[pout ? padi(i) : i] = v[q2];
    }
  }
}

// Transforms nb sequences held (unpadded) in `a` with radix-8 passes and a
// radix-2/4 tail; `b` is scratch of the same size; stride >= pad_stride(n);
// tw: e^{-2 pi i k / 2^lgtw}.  Returns the buffer holding the (unpadded)
// result.  The caller must __syncthreads() before the call.
template <typename R, int S>
MRM_D Cx<R>* block_fft(Cx<R>* a, Cx<R>* b, int lgn, int nb, int stride,
                       const Cx<R>* __restrict__ tw, int lgtw) {
  int lgNs = 0;
  const int nfull = lgn / 3;
  const int tail = lgn - nfull * 3;
  const int npass = nfull + (tail ? 1 : 0);
  int p = 0;
  for (int q = 0; q < nfull; ++q, ++p) {
    stockham_pass<R, 8, 3, S>(a, b, lgn, nb, stride, lgNs, p > 0, p < npass - 1, tw, lgtw);
    __syncthreads();
    Cx<R>* t = a; a = b; b = t;
    lgNs += 3;
  }
  if (tail) {
    if (tail == 2) stockham_pass<R, 4, 2, S>(a, b, lgn, nb, stride, lgNs, p > 0, false, tw, lgtw);
    else stockham_pass<R, 2, 1, S>(a, b, lgn, nb, stride, lgNs, p > 0, false, tw, lgtw);
    __syncthreads();
    Cx<R>* t = a; a = b; b = t;
  }
  return a;
}

// e^{-2 pi i k / 2^lg} from the 4096-entry table of the run-time form
template <typename R>
MRM_D Cx<R> twiddle(const Cx<R>* __restrict__ tw, int k, int lg) {
  return tw[k << (kTwLog - lg)];
}

// programmatic dependent launch (sm_90+): let the next kernel in the stream
// start its independent prologue / wait for the previous kernel's results
MRM_D void pdl_launch_dependents() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
MRM_D void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

}  // namespace mrm
