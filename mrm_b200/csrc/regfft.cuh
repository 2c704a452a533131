// regfft.cuh -- register-resident FFT stages (FP32) and the row transforms
// built from them, sm_100a.
//
// A sequence of N = 2^LGN points is transformed by NT = N/8 threads, each
// holding eight elements in registers.  Stage 0 is a radix-2^R0 pass over the
// top position bits, the others radix-8 passes; between stages the elements
// move through a shared exchange buffer at swizzled offsets, and each thread
// reads and writes only its own positions of a stage, so one barrier of the
// sequence's threads separates two stages.  The forward transform decimates in
// frequency from natural order to the mixed-radix digit-reversed order of
// fft.cuh's ip_freq (position 8t + k holds frequency ip_freq(8t) + k N/8);
// the inverse decimates in time from that order back to natural order.
// Radices, positions and twiddle tables are those of fft.cuh's in-place
// passes.
#pragma once
#include "fft.cuh"

namespace mrm {

// Exchange-buffer swizzle in 8-byte elements: bits 0..3 xored with bits 3..6.
// It is linear over xor, and for every stage's access pattern of a half warp
// (16 consecutive threads, one register slot) it puts the 16 elements on
// distinct bank pairs for N = 256 .. 2048 (checked by enumeration).
MRM_HD constexpr int xswz(int p) { return p ^ ((p >> 3) & 15); }

// Stage plan of an N = 2^LGN point sequence: S stages; stage 0 has radix
// 2^R0 over the top R0 position bits, the others radix 8.  In stage s a
// thread's eight elements differ in the three position bits from dbit(s)
// (its register digit); the other bits are the thread index.
template <int LGN>
struct RegPlan {
  static constexpr int N = 1 << LGN, NT = N / 8, S = (LGN + 2) / 3, R0 = LGN - 3 * (S - 1);
  MRM_HD static constexpr int dbit(int s) { return s == 0 ? LGN - 3 : LGN - R0 - 3 * s; }
  // log2 of the butterfly stride of stage s (the LGNS of its pass table)
  MRM_HD static constexpr int lgd(int s) { return s == 0 ? LGN - R0 : dbit(s); }
};

// position of a thread's element 0 in a stage whose register digit starts at bit B
template <int B>
MRM_D int reg_base(int t) {
  return (t & ((1 << B) - 1)) | ((t >> B) << (B + 3));
}

// forward radix-8 DFT of four inputs (inputs 4..7 are zero)
MRM_D void dft8_half_in(Cx<float>* v) {
  const float h = 0.70710678118654752440f;
  Cx<float> e0 = v[0], e1 = v[1], e2 = v[2], e3 = v[3];
  Cx<float> o0 = e0, o1 = cmul(e1, Cx<float>{h, -h}), o2 = cmul_i(e2, -1.f), o3 = cmul(e3, Cx<float>{-h, -h});
  dft4<float, -1>(e0, e1, e2, e3);
  dft4<float, -1>(o0, o1, o2, o3);
  v[0] = e0;
  v[2] = e1;
  v[4] = e2;
  v[6] = e3;
  v[1] = o0;
  v[3] = o1;
  v[5] = o2;
  v[7] = o3;
}

// The twiddles of a thread's butterflies in stage STAGE (shared by the three
// components): w[jl * R + m] = e^{-2 pi i j0 m / L} for the radix-R
// butterfly jl of the thread (one for radix 8; 8/R for a stage 0 of radix 2
// or 4), m >= 1; none when the stage's stride is 1.
template <int LGN, int STAGE>
MRM_D void reg_twiddles(Cx<float> (&w)[8], int t, const Cx<float>* __restrict__ tw) {
  using P = RegPlan<LGN>;
  constexpr int LGD = P::lgd(STAGE), D = 1 << LGD, OFF = pass_tw_off(LGN, LGD);
  constexpr int R = STAGE == 0 ? (1 << P::R0) : 8, NB = 8 / R;
  if constexpr (D > 1) {
#pragma unroll
    for (int jl = 0; jl < NB; ++jl) {
      const int j0 = STAGE == 0 ? t + (jl << (LGN - 3)) : (t & (D - 1));
#pragma unroll
      for (int m = 1; m < R; ++m) w[jl * R + m] = tw[OFF + (m - 1) * D + j0];
    }
  }
}

// Forward stage STAGE (decimation in frequency: butterfly, then twiddles) on
// one component's eight elements; element k of the register digit is v[k].
// HALF: positions >= N/2 are zero on input (stage 0).
template <int LGN, int STAGE, bool HALF>
MRM_D void reg_fwd(Cx<float> (&v)[8], const Cx<float> (&w)[8]) {
  using P = RegPlan<LGN>;
  constexpr int D = 1 << P::lgd(STAGE);
  if constexpr (STAGE == 0 && P::R0 < 3) {
    constexpr int R = 1 << P::R0, NB = 8 / R;
#pragma unroll
    for (int jl = 0; jl < NB; ++jl) {
      Cx<float> u[R];
#pragma unroll
      for (int m = 0; m < R; ++m) u[m] = v[jl + NB * m];
      if constexpr (HALF) {
        if constexpr (R == 4) {
          const Cx<float> a0 = u[0], a1 = u[1];
          u[0] = cadd(a0, a1);
          u[1] = cadd(a0, cmul_i(a1, -1.f));
          u[2] = csub(a0, a1);
          u[3] = cadd(a0, cmul_i(a1, 1.f));
        } else {
          u[1] = u[0];
        }
      } else {
        if constexpr (R == 4) dft4<float, -1>(u[0], u[1], u[2], u[3]);
        else dft2<float, -1>(u);
      }
#pragma unroll
      for (int m = 1; m < R; ++m) u[m] = cmul(u[m], w[jl * R + m]);
#pragma unroll
      for (int m = 0; m < R; ++m) v[jl + NB * m] = u[m];
    }
  } else {
    if constexpr (STAGE == 0 && HALF) dft8_half_in(v);
    else dft8<float, -1>(v);
    if constexpr (D > 1) {
#pragma unroll
      for (int m = 1; m < 8; ++m) v[m] = cmul(v[m], w[m]);
    }
  }
}

// Inverse stage STAGE (decimation in time: conjugate twiddles, then the
// butterfly with the + sign), unnormalised, on one component.
template <int LGN, int STAGE>
MRM_D void reg_inv(Cx<float> (&v)[8], const Cx<float> (&w)[8]) {
  using P = RegPlan<LGN>;
  constexpr int D = 1 << P::lgd(STAGE);
  if constexpr (STAGE == 0 && P::R0 < 3) {
    constexpr int R = 1 << P::R0, NB = 8 / R;
#pragma unroll
    for (int jl = 0; jl < NB; ++jl) {
      Cx<float> u[R];
      u[0] = v[jl];
#pragma unroll
      for (int m = 1; m < R; ++m) u[m] = cmul(v[jl + NB * m], cconj(w[jl * R + m]));
      if constexpr (R == 4) dft4<float, 1>(u[0], u[1], u[2], u[3]);
      else dft2<float, 1>(u);
#pragma unroll
      for (int m = 0; m < R; ++m) v[jl + NB * m] = u[m];
    }
  } else {
    if constexpr (D > 1) {
#pragma unroll
      for (int m = 1; m < 8; ++m) v[m] = cmul(v[m], cconj(w[m]));
    }
    dft8<float, 1>(v);
  }
}

// barrier of the NT threads of sequence group c (threads c NT .. c NT + NT - 1):
// their lanes of the warp, or named barrier 1 + c (c < 4; the barrier ids are
// immediates, so a kernel reserves barriers 0..4 only)
template <int NT>
MRM_D void reg_sync(int c) {
  if constexpr (NT < 32) {
    __syncwarp(((1u << NT) - 1) << ((c * NT) & 31));
  } else if constexpr (NT == 32) {
    __syncwarp();
  } else {
    switch (c) {
      case 0: asm volatile("bar.sync 1, %0;" ::"n"(NT) : "memory"); break;
      case 1: asm volatile("bar.sync 2, %0;" ::"n"(NT) : "memory"); break;
      case 2: asm volatile("bar.sync 3, %0;" ::"n"(NT) : "memory"); break;
      default: asm volatile("bar.sync 4, %0;" ::"n"(NT) : "memory"); break;
    }
  }
}


// One stage on a single sequence in its exchange buffer b (in place at the
// thread's positions of the stage).
template <int LGN, int STAGE, bool INV>
MRM_D void reg_stage1(Cx<float>* __restrict__ b, int t, const Cx<float>* __restrict__ tw) {
  using P = RegPlan<LGN>;
  constexpr int B = P::dbit(STAGE);
  Cx<float> w[8];
  reg_twiddles<LGN, STAGE>(w, t, tw);
  const int a = xswz(reg_base<B>(t));
  Cx<float> v[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) v[k] = b[a ^ xswz(k << B)];
  if constexpr (INV) reg_inv<LGN, STAGE>(v, w);
  else reg_fwd<LGN, STAGE, false>(v, w);
#pragma unroll
  for (int k = 0; k < 8; ++k) b[a ^ xswz(k << B)] = v[k];
}

// ---------------- row transforms (real signals of 2M = 2^(LGM+1) points) ----------------
//
// The real row x[0 .. 2M) is handled as z[n] = x[2n] + i x[2n+1], n < M, with
// the half-spectrum relations of the reference's r2c / c2r plans
// (fftw.f90:37-93): X[k] = (Y[k] + conj Y[M-k]) / 2 - i w^k (Y[k] - conj Y[M-k]) / 2
// for Y = FFT_M(z), w = e^{-2 pi i / 2M}; the inverse forms Z[k] = e + i w^-k o,
// e = X[k] + conj X[M-k], o = X[k] - conj X[M-k], and z = IFFT_M(Z).

// Inverse: X (M + 1 spectrum values, natural order) -> z[n] for n < nz into
// out; xb: the sequence's exchange buffer (M elements).  Thread t gathers the
// pre-processed spectrum at its first stage's positions, the digit-reversed
// frequencies ft + k M/8 (ft = ip_freq(8t)), so no reordering pass is needed.
// out may be X itself: every gather is behind at least one barrier of the
// group (LGM >= 4: two or more stages).
template <int LGM>
MRM_D void rrow_inverse(const Cx<float>* X, Cx<float>* __restrict__ xb, Cx<float>* out, int t, int g, int nz,
                        const Cx<float>* __restrict__ twpost, const Cx<float>* __restrict__ twpass) {
  using P = RegPlan<LGM>;
  constexpr int M = P::N, NT = P::NT, S = P::S;
  static_assert(S >= 2, "a barrier between the gather and the output");
  const int ft = ip_freq(8 * t, LGM);
  Cx<float> v[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const int f = ft + k * NT;
    Cx<float> a = X[f], b = X[M - f];
    if (f == 0) {  // self-conjugate bins: imaginary parts ignored (c2r)
      a.y = 0.f;
      b.y = 0.f;
    }
    const Cx<float> e = cadd(a, cconj(b));
    const Cx<float> o = csub(a, cconj(b));
    const Cx<float> w = cconj(twpost[f]);  // e^{+2 pi i f / 2M}
    v[k] = cadd(e, cmul_i(cmul(o, w), 1.f));
  }
  {
    Cx<float> w[8];
    reg_twiddles<LGM, S - 1>(w, t, twpass);
    reg_inv<LGM, S - 1>(v, w);
    const int a = xswz(t << 3);  // stage S-1 positions 8t + k
#pragma unroll
    for (int k = 0; k < 8; ++k) xb[a ^ k] = v[k];
  }
  reg_sync<NT>(g);
  if constexpr (S >= 4) {
    reg_stage1<LGM, 2, true>(xb, t, twpass);
    reg_sync<NT>(g);
  }
  if constexpr (S >= 3) {
    reg_stage1<LGM, 1, true>(xb, t, twpass);
    reg_sync<NT>(g);
  }
  Cx<float> w[8];
  reg_twiddles<LGM, 0>(w, t, twpass);
  constexpr int B0 = P::dbit(0);
  const int a = xswz(reg_base<B0>(t));
#pragma unroll
  for (int k = 0; k < 8; ++k) v[k] = xb[a ^ xswz(k << B0)];
  reg_inv<LGM, 0>(v, w);
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const int n = t + k * NT;  // stage 0 positions: natural order
    if (n < nz) out[n] = v[k];
  }
}

// Forward: z (natural order, n < M; HALF: zero for n >= M/2 and not read) ->
// Y = FFT_M(z) in natural order into nat, which may be the input itself (every
// load is behind at least one barrier of the group); xb: the exchange buffer.
// The group's threads are synchronised on return.
template <int LGM, bool HALF>
MRM_D void rrow_forward(const Cx<float>* in, Cx<float>* __restrict__ xb, Cx<float>* nat, int t, int g,
                        const Cx<float>* __restrict__ twpass) {
  using P = RegPlan<LGM>;
  constexpr int NT = P::NT, S = P::S, KIN = HALF ? 4 : 8;
  static_assert(S >= 2, "a barrier between the loads and the output");
  Cx<float> v[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) v[k] = k < KIN ? in[t + k * NT] : Cx<float>{0.f, 0.f};
  {
    Cx<float> w[8];
    reg_twiddles<LGM, 0>(w, t, twpass);
    reg_fwd<LGM, 0, HALF>(v, w);
    constexpr int B0 = P::dbit(0);
    const int a = xswz(reg_base<B0>(t));
#pragma unroll
    for (int k = 0; k < 8; ++k) xb[a ^ xswz(k << B0)] = v[k];
  }
  reg_sync<NT>(g);
  if constexpr (S >= 3) {
    reg_stage1<LGM, 1, false>(xb, t, twpass);
    reg_sync<NT>(g);
  }
  if constexpr (S >= 4) {
    reg_stage1<LGM, 2, false>(xb, t, twpass);
    reg_sync<NT>(g);
  }
  Cx<float> w[8];
  reg_twiddles<LGM, S - 1>(w, t, twpass);
  const int a = xswz(t << 3);
#pragma unroll
  for (int k = 0; k < 8; ++k) v[k] = xb[a ^ k];
  reg_fwd<LGM, S - 1, false>(v, w);
  const int ft = ip_freq(8 * t, LGM);
#pragma unroll
  for (int k = 0; k < 8; ++k) nat[ft + k * NT] = v[k];
  reg_sync<NT>(g);
}

}  // namespace mrm
