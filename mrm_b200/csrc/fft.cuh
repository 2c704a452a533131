// fft.cuh -- block-cooperative Stockham FFT in shared memory (sm_100a).
//
// Replaces the FFTW r2c/c2r plans of src/fftw.f90:37-93 (unnormalised,
// forward sign -1).  A batch of `nb` complex sequences of length n = 2^lgn,
// sequence b at buf + b*stride, is transformed with radix-16 passes and one
// radix-8/4/2 pass for the remainder (Stockham autosort: natural-order
// output, ping-pong between two shared buffers, one __syncthreads per pass).
// Intermediate passes use a padded layout (one spare slot per 16 elements)
// so the stride-R stores of the early passes hit distinct banks; the input of
// the first pass and the output of the last pass are unpadded.  `stride`
// must be >= fft_stride(n).  Twiddles come from a table tw[k] = e^{-2 pi i k / 2^lgtw}
// (FP64-accurate values) with 2^lgtw >= n, normally staged in shared memory.
#pragma once
#include "common.cuh"

namespace mrm {

MRM_HD int fft_stride(int n) { return n + (n >> 4) + 1; }
MRM_D int padi(int i) { return i + (i >> 4); }

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

// 16-point DFT as 4 x 4 (radix-4 over stride 4, twiddles w16^(k1 n2), radix-4);
// the outputs are left in digit-reversed order (see dft16_out)
template <typename R, int S>
MRM_D void dft16(Cx<R>* v) {
  const R c1 = (R)0.92387953251128675612818318939679;  // cos(pi/8)
  const R s1 = (R)0.38268343236508977172845998403040;  // sin(pi/8)
  const R h = (R)0.70710678118654752440084436210485;
#pragma unroll
  for (int n2 = 0; n2 < 4; ++n2) dft4<R, S>(v[n2], v[n2 + 4], v[n2 + 8], v[n2 + 12]);
  // after this, v[n2 + 4*k1] holds the k1-th output of column n2; twiddle w16^(k1*n2)
  const Cx<R> w1 = {c1, (R)S * s1}, w2 = {h, (R)S * h}, w3 = {s1, (R)S * c1};
  const Cx<R> w6 = {-h, (R)S * h}, w9 = {-c1, (R)S * (-s1)};
  // k1=1: n2=1..3 -> w^1, w^2, w^3 ; k1=2 -> w^2, w^4, w^6 ; k1=3 -> w^3, w^6, w^9
  v[5] = cmul(v[5], w1);
  v[6] = cmul(v[6], w2);
  v[7] = cmul(v[7], w3);
  v[9] = cmul(v[9], w2);
  v[10] = cmul_i(v[10], (R)S);
  v[11] = cmul(v[11], w6);
  v[13] = cmul(v[13], w3);
  v[14] = cmul(v[14], w6);
  v[15] = cmul(v[15], w9);
#pragma unroll
  for (int k1 = 0; k1 < 4; ++k1) dft4<R, S>(v[4 * k1], v[4 * k1 + 1], v[4 * k1 + 2], v[4 * k1 + 3]);
  // v[4*k1 + k2] now holds output k = k1 + 4*k2 (digit-reversed); dft16_out maps it back
}

// output index of v[q] after dft16
MRM_HD constexpr int dft16_out(int q) { return (q >> 2) + 4 * (q & 3); }

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
    if (RADIX == 16) dft16<R, S>(v);
    else if (RADIX == 8) dft8<R, S>(v);
    else if (RADIX == 4) dft4<R, S>(v[0], v[1], v[2], v[3]);
    else dft2<R, S>(v);
    const int idxD = ((j >> lgNs) << (lgNs + LGR)) + k;
#pragma unroll
    for (int q = 0; q < RADIX; ++q) {
      const int r = (RADIX == 16) ? dft16_out(q) : q;
      const int i = idxD + r * Ns;
      dst[pout ? padi(i) : i] = v[q];
    }
  }
}

// One Stockham pass with every size known at compile time (LGN: log2 length,
// LGR: log2 radix, LGNS: log2 of the current sub-transform length, TWL: log2
// of the twiddle table length, PIN/POUT: padded input/output layout).
template <typename R, int LGN, int LGR, int LGNS, int TWL, bool PIN, bool POUT, int S>
MRM_D void stockham_pass_c(const Cx<R>* __restrict__ in, Cx<R>* __restrict__ out, int nb,
                           const Cx<R>* __restrict__ tw) {
  constexpr int RADIX = 1 << LGR;
  constexpr int LGNR = LGN - LGR;
  constexpr int NR = 1 << LGNR;
  constexpr int NS = 1 << LGNS;
  constexpr int STRIDE = (1 << LGN) + ((1 << LGN) >> 4) + 1;  // fft_stride(n)
  const int total = nb << LGNR;
  for (int q = threadIdx.x; q < total; q += blockDim.x) {
    const int b = q >> LGNR, j = q & (NR - 1);
    const Cx<R>* src = in + b * STRIDE;
    Cx<R>* dst = out + b * STRIDE;
    Cx<R> v[RADIX];
#pragma unroll
    for (int r = 0; r < RADIX; ++r) {
      const int i = j + r * NR;
      v[r] = src[PIN ? i + (i >> 4) : i];
    }
    const int k = j & (NS - 1);
    if constexpr (LGNS > 0) {
#pragma unroll
      for (int r = 1; r < RADIX; ++r) {
        Cx<R> w = tw[(k * r) << (TWL - LGNS - LGR)];
        if (S > 0) w.y = -w.y;
        v[r] = cmul(v[r], w);
      }
    }
    if constexpr (RADIX == 16) dft16<R, S>(v);
    else if constexpr (RADIX == 8) dft8<R, S>(v);
    else if constexpr (RADIX == 4) dft4<R, S>(v[0], v[1], v[2], v[3]);
    else dft2<R, S>(v);
    const int idxD = ((j >> LGNS) << (LGNS + LGR)) + k;
#pragma unroll
    for (int q2 = 0; q2 < RADIX; ++q2) {
      const int r = (RADIX == 16) ? dft16_out(q2) : q2;
      const int i = idxD + r * NS;
      dst[POUT ? i + (i >> 4) : i] = v[q2];
    }
  }
}

// Radix-8 Stockham plan of length 2^LGN unrolled at compile time (the final
// pass takes the 1, 2 or 3 remaining bits).  Pass P reads layout PIN = (P>0),
// writes POUT = (P < last).
template <typename R, int LGN, int TWL, int S, int P, int LGNS>
MRM_D Cx<R>* fft_c_from(Cx<R>* a, Cx<R>* b, int nb, const Cx<R>* __restrict__ tw) {
  constexpr int REM = LGN - LGNS;
  if constexpr (REM <= 0) {
    return a;
  } else {
    constexpr int LGR = REM >= 3 ? 3 : REM;
    constexpr bool LAST = (REM - LGR) == 0;
    stockham_pass_c<R, LGN, LGR, LGNS, TWL, (P > 0), !LAST, S>(a, b, nb, tw);
    __syncthreads();
    return fft_c_from<R, LGN, TWL, S, P + 1, LGNS + LGR>(b, a, nb, tw);
  }
}

// Transforms nb sequences held (unpadded) in `a`, sequence stride
// fft_stride(n); `b` is scratch of the same size.  Returns the buffer holding
// the (unpadded) result.  The caller must __syncthreads() before the call.
// TWOFF: the twiddle table has length 2^(lgn + TWOFF).
template <typename R, int S, int TWOFF>
MRM_D Cx<R>* block_fft_c(Cx<R>* a, Cx<R>* b, int lgn, int nb, const Cx<R>* __restrict__ tw) {
  switch (lgn) {
    case 1: return fft_c_from<R, 1, 1 + TWOFF, S, 0, 0>(a, b, nb, tw);
    case 2: return fft_c_from<R, 2, 2 + TWOFF, S, 0, 0>(a, b, nb, tw);
    case 3: return fft_c_from<R, 3, 3 + TWOFF, S, 0, 0>(a, b, nb, tw);
    case 4: return fft_c_from<R, 4, 4 + TWOFF, S, 0, 0>(a, b, nb, tw);
    case 5: return fft_c_from<R, 5, 5 + TWOFF, S, 0, 0>(a, b, nb, tw);
    case 6: return fft_c_from<R, 6, 6 + TWOFF, S, 0, 0>(a, b, nb, tw);
    case 7: return fft_c_from<R, 7, 7 + TWOFF, S, 0, 0>(a, b, nb, tw);
    case 8: return fft_c_from<R, 8, 8 + TWOFF, S, 0, 0>(a, b, nb, tw);
    case 9: return fft_c_from<R, 9, 9 + TWOFF, S, 0, 0>(a, b, nb, tw);
    case 10: return fft_c_from<R, 10, 10 + TWOFF, S, 0, 0>(a, b, nb, tw);
    case 11: return fft_c_from<R, 11, 11 + TWOFF, S, 0, 0>(a, b, nb, tw);
    default: return fft_c_from<R, 12, 12, S, 0, 0>(a, b, nb, tw);  // TWOFF = 0 at the 4096 limit
  }
}

// Radix plan: the largest radix R in {16, 8, 4} whose passes keep at least
// half the block busy (nb * n / R >= BLOCK / 2); small batches use radix 4
// so that more threads share each pass.
MRM_D int fft_radix(int lgn, int nb, int block) {
  const int n = 1 << lgn;
  if ((nb * n) / 16 >= block / 2 && lgn >= 4) return 16;
  if ((nb * n) / 8 >= block / 2 && lgn >= 3) return 8;
  return 4;
}

template <typename R, int RADIX, int LGR, int S>
MRM_D Cx<R>* fft_passes(Cx<R>* a, Cx<R>* b, int lgn, int nb, int stride,
                        const Cx<R>* __restrict__ tw, int lgtw) {
  int lgNs = 0;
  const int nfull = lgn / LGR;
  const int tail = lgn - nfull * LGR;  // 0..LGR-1 remaining bits
  const int npass = nfull + (tail ? 1 : 0);
  int p = 0;
  for (int q = 0; q < nfull; ++q, ++p) {
    stockham_pass<R, RADIX, LGR, S>(a, b, lgn, nb, stride, lgNs, p > 0, p < npass - 1, tw, lgtw);
    __syncthreads();
    Cx<R>* t = a; a = b; b = t;
    lgNs += LGR;
  }
  if (tail) {
    if (tail == 3) stockham_pass<R, 8, 3, S>(a, b, lgn, nb, stride, lgNs, p > 0, false, tw, lgtw);
    else if (tail == 2) stockham_pass<R, 4, 2, S>(a, b, lgn, nb, stride, lgNs, p > 0, false, tw, lgtw);
    else stockham_pass<R, 2, 1, S>(a, b, lgn, nb, stride, lgNs, p > 0, false, tw, lgtw);
    __syncthreads();
    Cx<R>* t = a; a = b; b = t;
  }
  return a;
}

// Transforms nb sequences held (unpadded) in `a`; `b` is scratch of the same
// size.  Returns the buffer holding the (unpadded) result.  The caller must
// __syncthreads() before the call; on return the result is complete.
template <typename R, int S>
MRM_D Cx<R>* block_fft(Cx<R>* a, Cx<R>* b, int lgn, int nb, int stride,
                       const Cx<R>* __restrict__ tw, int lgtw) {
  const int radix = fft_radix(lgn, nb, blockDim.x);
  if (radix == 16) return fft_passes<R, 16, 4, S>(a, b, lgn, nb, stride, tw, lgtw);
  if (radix == 8) return fft_passes<R, 8, 3, S>(a, b, lgn, nb, stride, tw, lgtw);
  return fft_passes<R, 4, 2, S>(a, b, lgn, nb, stride, tw, lgtw);
}

// e^{-2 pi i k / 2^lg} from the 4096-entry global table
template <typename R>
MRM_D Cx<R> twiddle(const Cx<R>* __restrict__ tw, int k, int lg) {
  return tw[k << (kTwLog - lg)];
}

// Stages tw_s[k] = e^{-2 pi i k / 2^lg}, k < 2^lg, from the global table.
template <typename R>
MRM_D void stage_twiddles(Cx<R>* __restrict__ tw_s, const Cx<R>* __restrict__ tw, int lg) {
  const int n = 1 << lg;
  for (int k = threadIdx.x; k < n; k += blockDim.x) tw_s[k] = tw[k << (kTwLog - lg)];
}

// Fills tw_s[k] = e^{-2 pi i k / 2^lg}, k < 2^lg, with sincospi (accurate to
// about one ulp; no memory round trip).
MRM_D void make_twiddles(Cx<float>* __restrict__ tw_s, int lg) {
  const int n = 1 << lg;
  for (int k = threadIdx.x; k < n; k += blockDim.x) {
    float s, c;
    sincospif(-2.0f * (float)k / (float)n, &s, &c);
    tw_s[k] = Cx<float>{c, s};
  }
}
MRM_D void make_twiddles(Cx<double>* __restrict__ tw_s, int lg) {
  const int n = 1 << lg;
  for (int k = threadIdx.x; k < n; k += blockDim.x) {
    double s, c;
    sincospi(-2.0 * (double)k / (double)n, &s, &c);
    tw_s[k] = Cx<double>{c, s};
  }
}

// programmatic dependent launch (sm_90+): let the next kernel in the stream
// start its independent prologue / wait for the previous kernel's results
MRM_D void pdl_launch_dependents() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
MRM_D void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

}  // namespace mrm
