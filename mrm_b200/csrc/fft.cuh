// fft.cuh -- block-cooperative Stockham FFT in shared memory (sm_100a).
//
// Replaces the FFTW r2c/c2r plans of src/fftw.f90:37-93 (unnormalised,
// forward sign -1).  A batch of `nb` complex sequences of length n = 2^lgn,
// sequence b at buf + b*stride, is transformed with radix-8 passes and one
// final radix-4 or radix-2 pass (Stockham autosort: natural-order output,
// ping-pong between two shared buffers, one __syncthreads per pass).
// Twiddles come from one FP64-accurate table of e^{-2 pi i k / 4096}.
#pragma once
#include "common.cuh"

namespace mrm {

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
  Cx<R> w1 = {h, (R)S * h}, w3 = {-h, (R)S * h};
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

template <typename R, int RADIX, int LGR, int S>
MRM_D void stockham_pass(const Cx<R>* __restrict__ in, Cx<R>* __restrict__ out, int lgn, int nb,
                         int stride, int lgNs, const Cx<R>* __restrict__ tw) {
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
    for (int r = 0; r < RADIX; ++r) v[r] = src[j + r * nR];
    const int k = j & (Ns - 1);
    if (lgNs > 0) {
      const int sh = kTwLog - lgNs - LGR;
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
    for (int r = 0; r < RADIX; ++r) dst[idxD + r * Ns] = v[r];
  }
}

// Transforms nb sequences held in `a`; `b` is scratch of the same size.
// Returns the buffer that holds the result.  The caller must __syncthreads()
// before the call (data in `a` complete); on return the result is complete.
template <typename R, int S>
MRM_D Cx<R>* block_fft(Cx<R>* a, Cx<R>* b, int lgn, int nb, int stride,
                       const Cx<R>* __restrict__ tw) {
  int lgNs = 0;
  int rem = lgn;
  while (rem >= 3) {
    stockham_pass<R, 8, 3, S>(a, b, lgn, nb, stride, lgNs, tw);
    __syncthreads();
    Cx<R>* t = a; a = b; b = t;
    lgNs += 3;
    rem -= 3;
  }
  if (rem == 2) {
    stockham_pass<R, 4, 2, S>(a, b, lgn, nb, stride, lgNs, tw);
    __syncthreads();
    Cx<R>* t = a; a = b; b = t;
  } else if (rem == 1) {
    stockham_pass<R, 2, 1, S>(a, b, lgn, nb, stride, lgNs, tw);
    __syncthreads();
    Cx<R>* t = a; a = b; b = t;
  }
  return a;
}

// e^{-2 pi i k / 2^lg} from the 4096-entry table
template <typename R>
MRM_D Cx<R> twiddle(const Cx<R>* __restrict__ tw, int k, int lg) {
  return tw[k << (kTwLog - lg)];
}

}  // namespace mrm
