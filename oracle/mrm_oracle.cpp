// mrm_oracle.cpp -- TEST INFRASTRUCTURE, not product code.
//
// CPU restatement (FP64, OpenMP) of the reference's per-timestep grain dynamics
// (com-entonos/mrm), used only as the checker: by tests/, by
// __graft_entry__.smoke() and by bench.py's cpu_baseline / --impl reference leg.
// The product path (mrm_b200/libmrm_gpu.so) never links or calls this file.
//
// Parity status: the reference is Fortran + FFTW and cannot be compiled in this
// environment (no Fortran compiler, no FFTW), so this restatement is pinned by
//   * numpy's independent MT19937 (tempering/twist of random.f90) and
//     numpy's independent Philox4x64-10 (the GPU thermal stream),
//   * closed-form physics (Stoner-Wohlfarth switching, Larmor precession,
//     demag sum rules and tensor symmetries),
//   * a direct FP64 O(N^2) demag summation against the FFT convolution,
//   * numpy's pocketfft for the unnormalised r2c/c2r semantics of fftw.f90.
// It is NOT pinned against outputs of the reference binary ("parity unpinned").
//
// Each routine cites the reference file:line it restates (paths relative to the
// reference project root).

#include <quadmath.h>
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

using cd = std::complex<double>;

namespace orc {

// ---------------------------------------------------------------------------
// MT19937 with the reference's 1998-style seeding: src/random.f90:9-10,166-213
// ---------------------------------------------------------------------------
struct MT {
  uint32_t mt[624];
  int mti;
  int iset;
  double gset;
};

static void mt_create(MT* s, int seed) {
  // random.f90:173-181: iseed=4357+|seed|; mt(0)=iseed; mt(i)=69069*mt(i-1) (32-bit wrap)
  int32_t iseed = 4357 + std::abs(seed);
  s->mt[0] = (uint32_t)iseed;
  for (int i = 1; i < 624; ++i) s->mt[i] = 69069u * s->mt[i - 1];
  s->iset = 0;
  s->mti = 624;
  s->gset = 0.0;
}

static uint32_t mt_next_u32(MT* s) {
  // random.f90:191-207 (twist with UMASK/LMASK/MATA, tempering TMASKB/TMASKC)
  const uint32_t UM = 0x80000000u, LM = 0x7fffffffu, MATA = 0x9908b0dfu;
  const int N = 624, M = 397;
  if (s->mti >= N) {
    uint32_t j;
    for (int i = 0; i < N - M; ++i) {
      j = (s->mt[i] & UM) | (s->mt[i + 1] & LM);
      s->mt[i] = s->mt[i + M] ^ (j >> 1) ^ ((j & 1u) ? MATA : 0u);
    }
    for (int i = N - M; i < N - 1; ++i) {
      j = (s->mt[i] & UM) | (s->mt[i + 1] & LM);
      s->mt[i] = s->mt[i + M - N] ^ (j >> 1) ^ ((j & 1u) ? MATA : 0u);
    }
    j = (s->mt[N - 1] & UM) | (s->mt[0] & LM);
    s->mt[N - 1] = s->mt[M - 1] ^ (j >> 1) ^ ((j & 1u) ? MATA : 0u);
    s->mti = 0;
  }
  uint32_t y = s->mt[s->mti++];
  y ^= (y >> 11);
  y ^= (y << 7) & 0x9d2c5680u;
  y ^= (y << 15) & 0xefc60000u;
  y ^= (y >> 18);
  return y;
}

static double mt_uniform(MT* s) {
  // random.f90:208-212: unsigned value / 2^32, in [0,1)
  return (double)mt_next_u32(s) / 4294967296.0;
}

static double mt_normal(MT* s) {
  // random.f90:215-229: polar Box-Muller with a cached second deviate
  if (s->iset != 0) {
    s->iset = 0;
    return s->gset;
  }
  double v1, v2, rsq;
  v1 = 2.0 * mt_uniform(s) - 1.0;
  v2 = 2.0 * mt_uniform(s) - 1.0;
  rsq = v1 * v1 + v2 * v2;
  while (rsq >= 1.0 || rsq == 0.0) {
    v1 = 2.0 * mt_uniform(s) - 1.0;
    v2 = 2.0 * mt_uniform(s) - 1.0;
    rsq = v1 * v1 + v2 * v2;
  }
  double f = std::sqrt(-2.0 * std::log(rsq) / rsq);
  s->gset = v1 * f;
  s->iset = 1;
  return v2 * f;
}

// ---------------------------------------------------------------------------
// Philox4x64-10 (Salmon et al., SC'11) + Box-Muller: the counter-based thermal
// stream of the GPU path (the reference draws MT serially instead).  The same
// definition lives in mrm_b200/csrc/philox.cuh; numpy.random.Philox pins it.
// ---------------------------------------------------------------------------
static inline void mulhilo64(uint64_t a, uint64_t b, uint64_t* hi, uint64_t* lo) {
  unsigned __int128 p = (unsigned __int128)a * b;
  *hi = (uint64_t)(p >> 64);
  *lo = (uint64_t)p;
}

static void philox4x64(const uint64_t ctr_in[4], const uint64_t key_in[2], uint64_t out[4]) {
  const uint64_t M0 = 0xD2E7470EE14C6C93ull, M1 = 0xCA5A826395121157ull;
  const uint64_t W0 = 0x9E3779B97F4A7C15ull, W1 = 0xBB67AE8584CAA73Bull;
  uint64_t c0 = ctr_in[0], c1 = ctr_in[1], c2 = ctr_in[2], c3 = ctr_in[3];
  uint64_t k0 = key_in[0], k1 = key_in[1];
  for (int r = 0; r < 10; ++r) {
    uint64_t hi0, lo0, hi1, lo1;
    mulhilo64(M0, c0, &hi0, &lo0);
    mulhilo64(M1, c2, &hi1, &lo1);
    uint64_t n0 = hi1 ^ c1 ^ k0;
    uint64_t n1 = lo1;
    uint64_t n2 = hi0 ^ c3 ^ k1;
    uint64_t n3 = lo0;
    c0 = n0; c1 = n1; c2 = n2; c3 = n3;
    k0 += W0; k1 += W1;
  }
  out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

// Thermal normals of one grain at one Heun step: counter (grain, step, stream, 0),
// key (seed, 0x6d726d).  u = ((x>>11)+0.5)/2^53, Box-Muller pairs (u0,u1),(u2,u3).
static void philox_normal3(uint64_t seed, uint64_t stream, uint64_t step, uint64_t grain,
                           double n[3]) {
  uint64_t ctr[4] = {grain, step, stream, 0ull};
  uint64_t key[2] = {seed, 0x6d726dull};
  uint64_t r[4];
  philox4x64(ctr, key, r);
  const double s53 = 1.0 / 9007199254740992.0;
  double u0 = ((double)(r[0] >> 11) + 0.5) * s53;
  double u1 = ((double)(r[1] >> 11) + 0.5) * s53;
  double u2 = ((double)(r[2] >> 11) + 0.5) * s53;
  const double twopi = 6.283185307179586476925286766559;
  double ra = std::sqrt(-2.0 * std::log(u0));
  double rb = std::sqrt(-2.0 * std::log(u2));
  double u3 = ((double)(r[3] >> 11) + 0.5) * s53;
  n[0] = ra * std::cos(twopi * u1);
  n[1] = ra * std::sin(twopi * u1);
  n[2] = rb * std::cos(twopi * u3);
}

// ---------------------------------------------------------------------------
// Magnetostatic tensor: src/tensor_element.f90:13-102 (volume_averaged_n),
// :219-261 (plane_to_plane), src/tensor.f90:82-216 (calculate_tensor).
// ---------------------------------------------------------------------------
static inline double fsign(double a, double b) { return std::copysign(std::fabs(a), b); }

static inline double g1(double x, double y, double z, double d) {
  // tensor_element.f90:78-87
  double r = x * y * z * std::atan(y * z / fsign(std::max(1.0e-300, std::fabs(x) * d), x));
  r += 0.5 * y * (z * z - x * x) * std::log(std::max(1.0e-300, d - y));
  r += 0.5 * z * (y * y - x * x) * std::log(std::max(1.0e-300, d - z));
  r += (y * y + z * z - 2.0 * x * x) * d / 6.0;
  return r;
}

static inline double g2(double z, double x, double y, double d) {
  // tensor_element.f90:89-100 (argument order g2(z,x,y,d) as in the reference)
  double r = -x * y * z * std::log(std::max(1.0e-300, d + z));
  r += y * (y * y - 3.0 * z * z) * std::log(std::max(1.0e-300, d + x)) / 6.0;
  r += x * (x * x - 3.0 * z * z) * std::log(std::max(1.0e-300, d + y)) / 6.0;
  r += 0.5 * x * x * z * std::atan(y * z / fsign(std::max(1.0e-300, std::fabs(x) * d), x));
  r += 0.5 * y * y * z * std::atan(x * z / fsign(std::max(1.0e-300, std::fabs(y) * d), y));
  r += z * z * z * std::atan(x * y / fsign(std::max(1.0e-300, std::fabs(z) * d), z)) / 6.0;
  r += x * y * d / 3.0;
  return r;
}

// n(a,b) -= t(a,b); n stored row-major n[a*3+b] with a = first Fortran index.
static void volume_averaged_n(double rx, double ry, double rz, double xs, double ys, double zs,
                              double xo, double yo, double zo, double n[9]) {
  (void)yo;
  // tensor_element.f90:31: dyo uses xo (reference quirk, harmless for dx=dy)
  const double dxo[2] = {-0.5 * xo, 0.5 * xo}, dyo[2] = {-0.5 * xo, 0.5 * xo},
               dzo[2] = {-0.5 * zo, 0.5 * zo};
  const double dxs[2] = {-0.5 * xs, 0.5 * xs}, dys[2] = {-0.5 * ys, 0.5 * ys},
               dzs[2] = {-0.5 * zs, 0.5 * zs};
  double t[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int i6 = 1; i6 <= 2; ++i6)
    for (int i5 = 1; i5 <= 2; ++i5)
      for (int i4 = 1; i4 <= 2; ++i4)
        for (int i3 = 1; i3 <= 2; ++i3) {
          double dx = -rx + dxo[i3 - 1] - dxs[i6 - 1];
          for (int i2 = 1; i2 <= 2; ++i2) {
            double dy = -ry + dyo[i2 - 1] - dys[i5 - 1];
            for (int i1 = 1; i1 <= 2; ++i1) {
              double dz = -rz + dzo[i1 - 1] - dzs[i4 - 1];
              double d = std::sqrt(dx * dx + dy * dy + dz * dz);
              if (d != 0.0) {
                double sgn = ((i1 + i2 + i3 + i4 + i5 + i6 - 1) % 2 == 0) ? 1.0 : -1.0;
                t[0] += sgn * g1(dx, dy, dz, d);  // t(1,1)
                t[4] += sgn * g1(dy, dz, dx, d);  // t(2,2)
                t[8] += sgn * g1(dz, dx, dy, d);  // t(3,3)
                double x = sgn * g2(dx, dy, dz, d);
                t[7] += x;  // t(3,2)
                t[5] += x;  // t(2,3)
                x = sgn * g2(dy, dz, dx, d);
                t[6] += x;  // t(3,1)
                t[2] += x;  // t(1,3)
                x = sgn * g2(dz, dx, dy, d);
                t[3] += x;  // t(2,1)
                t[1] += x;  // t(1,2)
              }
            }
          }
        }
  for (int k = 0; k < 9; ++k) n[k] -= t[k];
}

// Quadruple-precision (binary128, libquadmath) evaluation of the same
// closed forms, for an offset (ix dx, iy dy, rz) with integer ix, iy: the
// exact-arithmetic value of the reference's formula to ~1e-30, against which
// the FP64 evaluation's cancellation noise and the device's double-double
// tensor are measured (test infrastructure).
using q128 = __float128;
static inline q128 q_sign(q128 a, q128 b) { return signbitq(b) ? -fabsq(a) : fabsq(a); }
static inline q128 q_max(q128 a, q128 b) { return a < b ? b : a; }
static inline q128 q_g1(q128 x, q128 y, q128 z, q128 d) {
  const q128 tiny = (q128)1.0e-300;
  q128 r = x * y * z * atanq(y * z / q_sign(q_max(tiny, fabsq(x) * d), x));
  r += (q128)0.5 * y * (z * z - x * x) * logq(q_max(tiny, d - y));
  r += (q128)0.5 * z * (y * y - x * x) * logq(q_max(tiny, d - z));
  r += (y * y + z * z - (q128)2 * x * x) * d / (q128)6;
  return r;
}
static inline q128 q_g2(q128 z, q128 x, q128 y, q128 d) {
  const q128 tiny = (q128)1.0e-300;
  q128 r = -x * y * z * logq(q_max(tiny, d + z));
  r += y * (y * y - (q128)3 * z * z) * logq(q_max(tiny, d + x)) / (q128)6;
  r += x * (x * x - (q128)3 * z * z) * logq(q_max(tiny, d + y)) / (q128)6;
  r += (q128)0.5 * x * x * z * atanq(y * z / q_sign(q_max(tiny, fabsq(x) * d), x));
  r += (q128)0.5 * y * y * z * atanq(x * z / q_sign(q_max(tiny, fabsq(y) * d), y));
  r += z * z * z * atanq(x * y / q_sign(q_max(tiny, fabsq(z) * d), z)) / (q128)6;
  r += x * y * d / (q128)3;
  return r;
}
static void volume_averaged_n_q(int ix, int iy, double dxc, double dyc, double rzd, double xsd, double ysd,
                                double zsd, double xod, double zod, q128 n[9]) {
  const q128 rx = (q128)ix * (q128)dxc, ry = (q128)iy * (q128)dyc, rz = (q128)rzd;
  const q128 xs = xsd, ys = ysd, zs = zsd, xo = xod, zo = zod, h = (q128)0.5;
  const q128 dxo[2] = {-h * xo, h * xo}, dyo[2] = {-h * xo, h * xo}, dzo[2] = {-h * zo, h * zo};
  const q128 dxs[2] = {-h * xs, h * xs}, dys[2] = {-h * ys, h * ys}, dzs[2] = {-h * zs, h * zs};
  q128 t[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int i6 = 1; i6 <= 2; ++i6)
    for (int i5 = 1; i5 <= 2; ++i5)
      for (int i4 = 1; i4 <= 2; ++i4)
        for (int i3 = 1; i3 <= 2; ++i3) {
          const q128 dx = -rx + dxo[i3 - 1] - dxs[i6 - 1];
          for (int i2 = 1; i2 <= 2; ++i2) {
            const q128 dy = -ry + dyo[i2 - 1] - dys[i5 - 1];
            for (int i1 = 1; i1 <= 2; ++i1) {
              const q128 dz = -rz + dzo[i1 - 1] - dzs[i4 - 1];
              const q128 d = sqrtq(dx * dx + dy * dy + dz * dz);
              if (d != 0) {
                const q128 sgn = ((i1 + i2 + i3 + i4 + i5 + i6 - 1) % 2 == 0) ? 1 : -1;
                t[0] += sgn * q_g1(dx, dy, dz, d);
                t[4] += sgn * q_g1(dy, dz, dx, d);
                t[8] += sgn * q_g1(dz, dx, dy, d);
                q128 x = sgn * q_g2(dx, dy, dz, d);
                t[7] += x;
                t[5] += x;
                x = sgn * q_g2(dy, dz, dx, d);
                t[6] += x;
                t[2] += x;
                x = sgn * q_g2(dz, dx, dy, d);
                t[3] += x;
                t[1] += x;
              }
            }
          }
        }
  for (int k = 0; k < 9; ++k) n[k] -= t[k];
}

// plane_to_plane: out[((a*3+b)*ny + j)*nx + i] = t(a,b) at FFT index (i,j)
static void plane_to_plane(int nx, int ny, double dx, double dy, double dz, double dzo, double rz,
                           int n_imgxi, int n_imgyi, double* out) {
  const int n_imgx = std::max(0, n_imgxi);
  const int n_imgy = std::max(0, n_imgxi);  // tensor_element.f90:230 (uses the x count)
  (void)n_imgyi;
  std::fill(out, out + (size_t)9 * nx * ny, 0.0);
  const int jlo = -ny / 2, jhi = ny / 2, ilo = -nx / 2, ihi = nx / 2;
  const int nj = jhi - jlo + 1, ni = ihi - ilo + 1;
  // compute each offset's t in parallel, then accumulate serially in the
  // reference's loop order (two offsets can share one FFT slot for even n)
  std::vector<double> tt((size_t)nj * ni * 9);
#pragma omp parallel for schedule(dynamic, 4) collapse(2)
  for (int jj = 0; jj < nj; ++jj)
    for (int ii = 0; ii < ni; ++ii) {
      int j = jlo + jj, i = ilo + ii;
      int yp0 = -n_imgy * (1 - std::max(0, j / ((ny + 1) / 2)));
      int yp1 = n_imgy * (1 + std::min(0, j / ((ny + 1) / 2)));
      int xp0 = -n_imgx * (1 - std::max(0, i / ((nx + 1) / 2)));
      int xp1 = n_imgx * (1 + std::min(0, i / ((nx + 1) / 2)));
      double t[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
      for (int ny_img = yp0; ny_img <= yp1; ++ny_img)
        for (int nx_img = xp0; nx_img <= xp1; ++nx_img) {
          double rx = (double)i * dx + (double)nx_img * dx * (double)nx;
          double ry = (double)j * dy + (double)ny_img * dy * (double)ny;
          volume_averaged_n(rx, ry, rz, dx, dy, dz, dx, dy, dzo, t);
        }
      std::memcpy(&tt[((size_t)jj * ni + ii) * 9], t, sizeof(t));
    }
  for (int jj = 0; jj < nj; ++jj)
    for (int ii = 0; ii < ni; ++ii) {
      int j = jlo + jj, i = ilo + ii;
      int fi = ((nx - i) % nx + nx) % nx, fj = ((ny - j) % ny + ny) % ny;
      const double* t = &tt[((size_t)jj * ni + ii) * 9];
      for (int c = 0; c < 9; ++c) out[((size_t)c * ny + fj) * nx + fi] += t[c];
    }
}

// calculate_tensor (tensor.f90:82-216).  n2d layout = Fortran n2d(nx,ny,9,ko,ks):
// n2d[(((ks*nl + ko)*9 + c)*ny + j)*nx + i], c = 3*(field comp) + (source comp).
static void calculate_tensor(int nx, int ny, int nl, double dx, double dy, const double* dz,
                             const double* il_space, int imx, int imy, double space_to_sul,
                             double sul_mu, double head_mu, double fly_height, double* n2d) {
  std::fill(n2d, n2d + (size_t)nx * ny * 9 * nl * nl, 0.0);
  bool sul_p = (sul_mu > 1.0), head_p = (head_mu > 1.0);  // tensor.f90:20,105,111
  double mus = 0.0, mush = 0.0;
  if (sul_p) mus = std::max(0.0, (std::max(1.0, sul_mu) - 1.0) / (std::max(1.0, sul_mu) + 1.0));
  if (head_p) mush = std::max(0.0, (std::max(1.0, head_mu) - 1.0) / (std::max(1.0, head_mu) + 1.0));
  std::vector<double> hdz(nl);
  hdz[0] = fly_height;
  for (int ks = 1; ks < nl; ++ks) hdz[ks] = hdz[ks - 1] + dz[ks - 1] + il_space[ks];
  for (int k = 0; k < nl; ++k) hdz[k] += 0.5 * dz[k];
  std::vector<double> nn((size_t)9 * nx * ny);
  const size_t plane = (size_t)nx * ny;
  double zsb = space_to_sul;
  for (int ks = nl - 1; ks >= 0; --ks) {
    double zst = zsb + dz[ks];
    double zob = space_to_sul;
    for (int ko = nl - 1; ko >= 0; --ko) {
      double zot = zob + dz[ko];
      double* dst = n2d + ((size_t)ks * nl + ko) * 9 * plane;
      // nn(:,:,a,b) -> n2d(:,:,3*(b-1)+a): dst[c=3*b+a] = t(a,b)
      plane_to_plane(nx, ny, dx, dy, dz[ks], dz[ko], 0.5 * (zst - zot + zsb - zob), imx, imy,
                     nn.data());
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b)
          for (size_t p = 0; p < plane; ++p) dst[(3 * b + a) * plane + p] = nn[(a * 3 + b) * plane + p];
      if (sul_p) {
        plane_to_plane(nx, ny, dx, dy, dz[ks], dz[ko], 0.5 * (-zst - zot - zsb - zob), imx, imy,
                       nn.data());
        for (int a = 0; a < 3; ++a) {
          double f = (a < 2) ? -mus : mus;  // tensor.f90:167
          for (int b = 0; b < 3; ++b)
            for (size_t p = 0; p < plane; ++p) dst[(3 * b + a) * plane + p] += f * nn[(a * 3 + b) * plane + p];
        }
      }
      if (head_p) {
        plane_to_plane(nx, ny, dx, dy, dz[ks], dz[ko], hdz[ks] + hdz[ko], imx, imy, nn.data());
        for (int a = 0; a < 3; ++a) {
          double f = (a < 2) ? -mush : mush;  // tensor.f90:177
          for (int b = 0; b < 3; ++b)
            for (size_t p = 0; p < plane; ++p) dst[(3 * b + a) * plane + p] += f * nn[(a * 3 + b) * plane + p];
        }
      }
      double norm = 1.0 / (dx * dy * dz[ko] * (double)nx * (double)ny);  // tensor.f90:183
      for (size_t p = 0; p < 9 * plane; ++p) dst[p] *= norm;
      zob = zot + il_space[ko];
    }
    zsb = zst + il_space[ks];
  }
}

// ---------------------------------------------------------------------------
// FFT with FFTW's unnormalised r2c / c2r semantics (fftw.f90:37-93), in FP64
// or FP32 (the reference's default build links the single-precision FFTW,
// Makefile:171-180, and its FFTD=1 build the double one).  Real rows go
// through a complex transform of half the length (even lengths); radix-2
// iterative passes for powers of two with per-pass twiddle tables, a direct
// DFT for other lengths (test sizes only).  Complex products are written out
// so that no library call checks for infinities in the inner loops.
// ---------------------------------------------------------------------------
template <typename T>
static inline std::complex<T> cmul(std::complex<T> a, std::complex<T> b) {
  return {a.real() * b.real() - a.imag() * b.imag(), a.real() * b.imag() + a.imag() * b.real()};
}

template <typename T>
struct FFT1 {
  using C = std::complex<T>;
  int n = 0;
  bool pow2 = true;
  std::vector<C> tw;     // e^{-2 pi i k/n}, k < n
  std::vector<C> ptw;    // pass tables: for len = 2, 4, ..., n: e^{-2 pi i k/len}, k < len/2
  std::vector<int> rev;
  void init(int n_) {
    n = n_;
    pow2 = (n > 0) && ((n & (n - 1)) == 0);
    tw.resize(n);
    for (int k = 0; k < n; ++k) {
      double a = -2.0 * M_PI * (double)k / (double)n;
      tw[k] = C((T)std::cos(a), (T)std::sin(a));
    }
    ptw.clear();
    rev.clear();
    if (pow2) {
      for (int len = 2; len <= n; len <<= 1)
        for (int k = 0; k < len / 2; ++k) {
          double a = -2.0 * M_PI * (double)k / (double)len;
          ptw.push_back(C((T)std::cos(a), (T)std::sin(a)));
        }
      rev.resize(n);
      int lg = 0;
      while ((1 << lg) < n) ++lg;
      for (int i = 0; i < n; ++i) {
        int r = 0;
        for (int b = 0; b < lg; ++b)
          if (i & (1 << b)) r |= 1 << (lg - 1 - b);
        rev[i] = r;
      }
    }
  }
  // in-place, sign -1 (forward) or +1 (backward), unnormalised
  void run(C* a, int sign, C* scratch) const {
    if (pow2) {
      for (int i = 0; i < n; ++i)
        if (i < rev[i]) std::swap(a[i], a[rev[i]]);
      const C* w0 = ptw.data();
      for (int len = 2; len <= n; len <<= 1) {
        const int half = len >> 1;
        for (int i = 0; i < n; i += len)
          for (int k = 0; k < half; ++k) {
            const C w = sign > 0 ? std::conj(w0[k]) : w0[k];
            const C u = a[i + k], v = cmul(a[i + k + half], w);
            a[i + k] = u + v;
            a[i + k + half] = u - v;
          }
        w0 += half;
      }
    } else {
      for (int k = 0; k < n; ++k) {
        C acc = 0;
        for (int j = 0; j < n; ++j) {
          C w = tw[(size_t)((long long)j * k % n)];
          if (sign > 0) w = std::conj(w);
          acc += cmul(a[j], w);
        }
        scratch[k] = acc;
      }
      for (int k = 0; k < n; ++k) a[k] = scratch[k];
    }
  }
};

template <typename T>
struct FFT2 {
  using C = std::complex<T>;
  int nx = 0, ny = 0, nh = 0;  // nh = nx/2+1
  FFT1<T> fx, fh, fy;          // fh: half length (real rows of even length)
  std::vector<C> twx;          // e^{-2 pi i k/nx}, k <= nx/2
  void init(int nx_, int ny_) {
    nx = nx_; ny = ny_; nh = nx / 2 + 1;
    fx.init(nx); fy.init(ny);
    if (nx % 2 == 0) fh.init(nx / 2);
    twx.resize(nh);
    for (int k = 0; k < nh; ++k) {
      double a = -2.0 * M_PI * (double)k / (double)nx;
      twx[k] = C((T)std::cos(a), (T)std::sin(a));
    }
  }
  // one real row -> its nh lowest bins
  void row_r2c(const T* r, C* out, std::vector<C>& z, std::vector<C>& scr) const {
    if (nx % 2 != 0) {
      for (int i = 0; i < nx; ++i) z[i] = C(r[i], 0);
      fx.run(z.data(), -1, scr.data());
      for (int k = 0; k < nh; ++k) out[k] = z[k];
      return;
    }
    const int m = nx / 2;
    for (int k = 0; k < m; ++k) z[k] = C(r[2 * k], r[2 * k + 1]);
    fh.run(z.data(), -1, scr.data());
    const C mi(0, -1);
    for (int k = 0; k < nh; ++k) {
      const C a = z[k % m], b = std::conj(z[(m - k) % m]);
      const C e = (a + b) * (T)0.5, o = (a - b) * (T)0.5;
      out[k] = e + cmul(mi, cmul(twx[k], o));
    }
  }
  // nh bins (Hermitian half) -> one real row, unnormalised; imaginary parts of
  // the self-conjugate bins ignored
  void row_c2r(const C* in, T* r, std::vector<C>& z, std::vector<C>& scr) const {
    if (nx % 2 != 0) {
      for (int k = 0; k < nh; ++k) z[k] = in[k];
      for (int k = nh; k < nx; ++k) z[k] = std::conj(in[nx - k]);
      z[0] = C(z[0].real(), 0);
      fx.run(z.data(), +1, scr.data());
      for (int i = 0; i < nx; ++i) r[i] = z[i].real();
      return;
    }
    const int m = nx / 2;
    const C pi(0, 1);
    for (int k = 0; k < m; ++k) {
      C a = in[k], b = in[m - k];
      if (k == 0) {
        a = C(a.real(), 0);
        b = C(b.real(), 0);
      }
      const C e = a + std::conj(b), o = a - std::conj(b);
      z[k] = e + cmul(pi, cmul(std::conj(twx[k]), o));
    }
    fh.run(z.data(), +1, scr.data());
    for (int k = 0; k < m; ++k) {
      r[2 * k] = z[k].real();
      r[2 * k + 1] = z[k].imag();
    }
  }
  // r[ny][nx] -> c[ny][nh]
  void r2c(const T* r, C* c) const {
#pragma omp parallel
    {
      std::vector<C> z(nx), scr(std::max(nx, ny));
#pragma omp for
      for (int j = 0; j < ny; ++j) row_r2c(r + (size_t)j * nx, c + (size_t)j * nh, z, scr);
    }
#pragma omp parallel
    {
      std::vector<C> col(ny), scr(std::max(nx, ny));
#pragma omp for
      for (int k = 0; k < nh; ++k) {
        for (int j = 0; j < ny; ++j) col[j] = c[(size_t)j * nh + k];
        fy.run(col.data(), -1, scr.data());
        for (int j = 0; j < ny; ++j) c[(size_t)j * nh + k] = col[j];
      }
    }
  }
  // c[ny][nh] (Hermitian half) -> r[ny][nx], unnormalised; c is destroyed
  void c2r(C* c, T* r) const {
#pragma omp parallel
    {
      std::vector<C> col(ny), scr(std::max(nx, ny));
#pragma omp for
      for (int k = 0; k < nh; ++k) {
        for (int j = 0; j < ny; ++j) col[j] = c[(size_t)j * nh + k];
        fy.run(col.data(), +1, scr.data());
        for (int j = 0; j < ny; ++j) c[(size_t)j * nh + k] = col[j];
      }
    }
#pragma omp parallel
    {
      std::vector<C> z(nx), scr(std::max(nx, ny));
#pragma omp for
      for (int j = 0; j < ny; ++j) row_c2r(c + (size_t)j * nh, r + (size_t)j * nx, z, scr);
    }
  }
};

// ---------------------------------------------------------------------------
// Simulation state (data_s src/data.f90:91-104, field_ss src/field.f90:15-35,
// llg_s src/llg.f90:16-25), restricted to the LLG path.
// ---------------------------------------------------------------------------
struct Layer {
  int N = 0;
  std::vector<double> ms, vol, axis, hk, hk_scale, ms_scale, alpha_scale;
  // cubic anisotropy (field.f90:377-395): cubic_axis(3,3,N), lab component k of
  // crystal axis i of grain n at cax[k + 3 i + 9 n]; empty: uniaxial layer
  // (construct_grain.f90:1620-1625 keeps one of the two per layer)
  std::vector<double> cax;
  double alpha = 1.0, gamma = 1.76e7, floor_ms = 0.01;
  std::vector<int> hx_idx, hx_nbr;  // CSR: hx_idx[N+1] cumulative, hx_nbr 0-based
  std::vector<double> hx;
  std::vector<int> uhx_idx, uhx_nbr, lhx_idx, lhx_nbr;  // interlayer (upper = layer-1)
  std::vector<double> uhx, lhx;
  std::vector<int> g2c_idx, g2c_i, g2c_j;  // grain -> cells (0-based i,j)
  std::vector<int> c2g;                    // cell -> grain (-1: empty), grid2grain
  // moving demag window (update_do_grain, data.f90:120-157): grains with a cell
  // in the window, and the first and last of them (min_n, max_n, 0-based)
  std::vector<char> do_grain;
  int min_n = 0, max_n = -1;
  // LLB integrator (llgp%llb, push_llb llg.f90:916-1064): spin, Tc and
  // lambdaMs per grain, the magnitude |m| per buffer (data.f90:202: 1)
  bool llb = false;
  int mode = 0, meq_bs = 0, garanin_tau = 0;  // mode 1: push_mt (llgp%mt)
  double spin = 1.0;
  std::vector<double> tc, lam_ms, mag[2];
  // super-Gaussian temperature profile (suprgaus_temp / ref_temp / set_temp):
  // the grain temperatures of the last field evaluation (get_applied)
  bool tprof = false;
  double tp_bg = 0, tp_dtemp = 0, tp_isx = 0, tp_isy = 0, tp_vx = 0, tp_vy = 0, tp_ox = 0, tp_oy = 0, tp_rx = 0,
         tp_ry = 0, tp_t0 = 0;
  int tp_expn = 2, tp_func = 0;
  double tp_t_start = -1e22, tp_t_end = 1e22, tp_s_start = 1, tp_s_end = 1, tp_scale = 1, tp_amp = 0, tp_fgamma = 0,
         tp_phase = 0, tp_param = 0, tp_duty = 0, tp_moddepth = 0, tp_dc = 0;
  std::vector<double> temp;
  // temperature scaling (temp_scaling_s, temp_scaling.f90:21-26; applied by
  // find_temp_scaling :365-430 at every field evaluation): the grains' Tc
  // (field%tc), power laws (1 - T/Tc)^e for Ms and Hk (negative: none), Ms
  // from |m| (use_mag_p), and the reduced tables T/Tc -> scale of Ms, alpha,
  // Hk and Hx (Hx's scale is computed but, as in the reference, used nowhere)
  bool tsc = false;
  std::vector<double> tsc_tc;
  double tsc_msexp = -1.0, tsc_hkexp = -1.0;
  bool tsc_mag = false;
  std::vector<double> tsc_t[4], tsc_v[4];
  std::vector<double> m[2], dm, h, hthm, hdemag, happ;
  // schedule: uniform field x linear ramp (applied.f90:863-883)
  double hdir[3] = {0, 0, 0};
  double t_start = -1e22, t_end = 1e22, s_start = 1.0, s_end = 1.0, scale = 1.0;
  // time function (applied.f90:328-377): 0 none (linear ramp), 1 SIN, 2 COS, 3 EXP, 4 STE, 5 NEW
  int func = 0;
  double amp = 0, fgamma = 0, phase = 0, param = 0, duty = 0, moddepth = 0, dc = 0;
  double temperature = 0.0;
  bool thermal = false;
  // moving write head (form 6; the config's head model, no reference counterpart):
  // Karlqvist field, gap centre at hd_x0 + hd_v (t - hd_t0), polarity from hd_bits
  bool head = false;
  double hd_gap = 0, hd_z = 1, hd_hg = 0, hd_v = 0, hd_x0 = 0, hd_t0 = 0, hd_tbit = 1;
  uint64_t hd_bits = 0;
  int hd_nbits = 1;
  // tabulated field profile (file_applied, applied.f90:711-813): tab_v(3, tnx, tny),
  // node positions, origin offset / velocity / reference / time origin
  bool tab = false;
  int tnx = 0, tny = 0;
  std::vector<double> tab_x, tab_y, tab_v;
  double tox = 0, toy = 0, tvx = 0, tvy = 0, trx = 0, try_ = 0, tt0 = 0;
  MT rng;
};

struct Stats {
  double t;
  long long step;
  double mave[3], mvar[3], have[3];
  double errmx, errmx1, mmag, energy;
  double mave_l[8][3], mvar_l[8][3], have_l[8][3], mms_l[8][3];
  double vol_l[8], msvol_l[8];
  long long nup_l[8];
  double errmx1_l[8];
};

struct Sim {
  int nx, ny, nl;
  int boundary;  // 0 periodic (reference), 1 open (zero-padded 2x)
  int images;
  double dx, dy;
  std::vector<double> dz, il_space;
  double space_to_sul = 0, sul_mu = 1, head_mu = 1, fly_height = 0;
  int px, py, ph;  // FFT grid and half width
  FFT2<double> fft;
  std::vector<cd> nhat;  // [ks][ko][9][py][ph]
  // FP32 FFT grids (the reference's default single-precision FFTW build): the
  // tensor spectrum from the FP64 real tensor cast to float, the M grid, its
  // spectrum and H in float; state and fields stay FP64
  int fft_bits = 64;
  FFT2<float> fft32;
  std::vector<std::complex<float>> nhat32;
  std::vector<double> n2d_real;  // the real tensor, kept to form either spectrum
  bool demag_on = true;
  std::vector<Layer> L;
  int in = 0;          // which m buffer is current (llg.f90 `in` toggle, 0 or 1)
  // moving demag window (window_m, data.f90:1-65): size (0: none), window%v,
  // window%offset, current origin
  int wnx = 0, wny = 0, wi0 = 0, wj0 = 0;
  double wvx = 0, wvy = 0, wox = 0, woy = 0;
  double t = 0.0;
  long long step = 0;
  int rng_mode = 0;  // 0: MT per layer (reference), 1: Philox (GPU stream)
  uint64_t seed = 1;
  // scratch
  std::vector<double> grid;
  std::vector<cd> spec;
  Stats last{};
};

// ----- tensor spectrum (demag.f90:255-267, computed here in FP64) -----
static void build_spectrum(Sim* s, const double* n2d_real) {
  const int nl = s->nl;
  const size_t plane = (size_t)s->px * s->py, hplane = (size_t)s->ph * s->py;
  s->n2d_real.assign(n2d_real, n2d_real + (size_t)nl * nl * 9 * plane);
  if (s->fft_bits == 32) {
    // demag.f90:255-267 with ffttr = single: the tensor cast to float, then its FFT
    std::vector<float> rf(plane);
    s->nhat32.assign((size_t)nl * nl * 9 * hplane, std::complex<float>(0, 0));
    for (int p = 0; p < nl * nl * 9; ++p) {
      for (size_t q = 0; q < plane; ++q) rf[q] = (float)n2d_real[p * plane + q];
      s->fft32.r2c(rf.data(), &s->nhat32[p * hplane]);
    }
    s->nhat.clear();
    return;
  }
  s->nhat.assign((size_t)nl * nl * 9 * hplane, cd(0, 0));
  for (int p = 0; p < nl * nl * 9; ++p) s->fft.r2c(n2d_real + p * plane, &s->nhat[p * hplane]);
  s->nhat32.clear();
}

// grain -> cell scatter of Ms*ms_scale*m (data.f90:322-390)
static void scatter_m(Sim* s, int buf, std::vector<double>& grid) {
  const size_t plane = (size_t)s->px * s->py;
  grid.assign((size_t)s->nl * 3 * plane, 0.0);
  for (int l = 0; l < s->nl; ++l) {
    Layer& Ly = s->L[l];
    const double* m = Ly.m[buf].data();
    for (int n = 0; n < Ly.N; ++n) {
      if (!Ly.do_grain[n]) continue;
      double f = Ly.ms[n] * Ly.ms_scale[n];
      for (int q = Ly.g2c_idx[n]; q < Ly.g2c_idx[n + 1]; ++q) {
        // get_mag with a window (data.f90:357-385): the cells inside it, shifted
        const int i = Ly.g2c_i[q] - s->wi0, j = Ly.g2c_j[q] - s->wj0;
        if (s->wnx && (i < 0 || j < 0 || i >= s->wnx || j >= s->wny)) continue;
        size_t cell = (size_t)j * s->px + i;
        for (int a = 0; a < 3; ++a) grid[((size_t)l * 3 + a) * plane + cell] = f * m[3 * n + a];
      }
    }
  }
}

// get_demag (demag.f90:33-135) + get_magnetostatic gather (field.f90:438-470)
template <typename T>
static void demag_conv(const FFT2<T>& fft, const std::vector<std::complex<T>>& nhat, int nl, size_t plane,
                       size_t hplane, T* grid) {
  using C = std::complex<T>;
  std::vector<C> X((size_t)nl * 3 * hplane), H((size_t)nl * 3 * hplane, C(0, 0));
  for (int p = 0; p < nl * 3; ++p) fft.r2c(&grid[p * plane], &X[p * hplane]);
  for (int ks = 0; ks < nl; ++ks)
    for (int ko = 0; ko < nl; ++ko) {
      const C* N = &nhat[((size_t)ks * nl + ko) * 9 * hplane];
      for (int a = 0; a < 3; ++a) {
        C* Ha = &H[((size_t)ko * 3 + a) * hplane];
        for (int b = 0; b < 3; ++b) {
          const C* Nab = N + (size_t)(3 * a + b) * hplane;
          const C* Xb = &X[((size_t)ks * 3 + b) * hplane];
#pragma omp parallel for
          for (size_t q = 0; q < hplane; ++q) Ha[q] += cmul(Nab[q], Xb[q]);
        }
      }
    }
  for (int p = 0; p < nl * 3; ++p) fft.c2r(&H[p * hplane], &grid[p * plane]);
}

static void demag_from_grid(Sim* s, std::vector<double>& grid) {
  const int nl = s->nl;
  const size_t plane = (size_t)s->px * s->py, hplane = (size_t)s->ph * s->py;
  if (s->fft_bits == 32) {
    // M grid, spectra and H in float (get_mag's real(., ffttr)), back to FP64 fields
    std::vector<float> gf(grid.size());
#pragma omp parallel for
    for (size_t q = 0; q < grid.size(); ++q) gf[q] = (float)grid[q];
    demag_conv<float>(s->fft32, s->nhat32, nl, plane, hplane, gf.data());
#pragma omp parallel for
    for (size_t q = 0; q < grid.size(); ++q) grid[q] = (double)gf[q];
    return;
  }
  demag_conv<double>(s->fft, s->nhat, nl, plane, hplane, grid.data());
}

static void gather_demag(Sim* s, const std::vector<double>& grid) {
  const size_t plane = (size_t)s->px * s->py;
  for (int l = 0; l < s->nl; ++l) {
    Layer& Ly = s->L[l];
    for (int n = 0; n < Ly.N; ++n) {
      if (!Ly.do_grain[n]) continue;
      double y[3] = {0, 0, 0};
      for (int q = Ly.g2c_idx[n]; q < Ly.g2c_idx[n + 1]; ++q) {
        // get_magnetostatic with a window (field.f90:472-495): the cells inside
        // it, over all of the grain's cells
        const int i = Ly.g2c_i[q] - s->wi0, j = Ly.g2c_j[q] - s->wj0;
        if (s->wnx && (i < 0 || j < 0 || i >= s->wnx || j >= s->wny)) continue;
        size_t cell = (size_t)j * s->px + i;
        for (int a = 0; a < 3; ++a) y[a] += grid[((size_t)l * 3 + a) * plane + cell];
      }
      double cnt = (double)(Ly.g2c_idx[n + 1] - Ly.g2c_idx[n]);
      for (int a = 0; a < 3; ++a) Ly.hdemag[3 * n + a] = y[a] / cnt;
    }
  }
}

static void compute_demag(Sim* s, int buf) {
  if (!s->demag_on) {
    for (auto& Ly : s->L) std::fill(Ly.hdemag.begin(), Ly.hdemag.end(), 0.0);
    return;
  }
  scatter_m(s, buf, s->grid);
  demag_from_grid(s, s->grid);
  gather_demag(s, s->grid);
}

// funct (applied.f90:328-377); Fortran mod(x,g) = x - int(x/g)*g
static double funct(int f, double t, double g, double phase, double param, double duty,
                    double moddepth) {
  if (f == 7) return 1.0;  // ROT with the rotation angles present, |gamma| != 1 (applied.f90:378-383)
  if (f == 1) return std::sin(t * g + phase);
  if (f == 2) return std::cos(t * g + phase);
  if (f == 3) return std::exp(t * g + phase);
  if (f == 5) {  // NEW
    double x = g / param;
    const double y = std::exp(duty * x), w = std::exp(x);
    x = t + phase;
    if (x < 0.0) x = x + g * (1.0 + (double)(long long)std::fabs(x / g));
    x = std::fmod(x, g);
    if (x > duty * g) {
      x = std::exp((g - x) / param);
      return 1.0 - moddepth + x * (y - 1.0) * moddepth / (w - 1.0);
    }
    x = std::exp(-x / param);
    return 1.0 + x * (y - w) * moddepth / (w - 1.0);
  }
  if (f == 4) {  // STE
    double x = t + phase;
    if (x < 0.0) x = x + g * (1.0 + (double)(long long)std::fabs(x / g));
    x = std::fmod(x, g);
    if (x < 0.5 * param) return 2.0 * x / param;
    if (x < 0.5 * (g - param)) return 1.0;
    if (x < 0.5 * (g + param)) return (g - 2.0 * x) / param;
    if (x < g - 0.5 * param) return -1.0;
    return 2.0 * (x - g) / param;
  }
  return 0.0;
}

// applied field scale of one uniform field (applied.f90:866-883, set_fld :289-317)
static double ramp_scale(const Layer& Ly, double t) {
  if (Ly.func != 0)
    return (Ly.amp * funct(Ly.func, t, Ly.fgamma, Ly.phase, Ly.param, Ly.duty, Ly.moddepth) + Ly.dc) * Ly.scale;
  double u = (t - Ly.t_start) / (Ly.t_end - Ly.t_start);
  u = std::max(0.0, std::min(1.0, u));
  return ((Ly.s_end - Ly.s_start) * u + Ly.s_start) * Ly.scale;
}

// set (applied.f90:1757-1776), 0-based: for mesh cell i (centre (i+1/2) dd)
// the lower table node ind[i] and its weight f[i]
static void set_weights(double offset, int n, double dd, const std::vector<double>& pos, std::vector<int>& ind,
                        std::vector<double>& f) {
  const int npos = (int)pos.size();
  ind.assign(n, 0);
  f.assign(n, 0.0);
  int i0 = 2;  // 1-based node index, as the reference sweeps it
  for (int i = 1; i <= n; ++i) {
    const double x = (i - .5) * dd - offset;
    while (pos[i0 - 1] <= x && i0 < npos) ++i0;
    ind[i - 1] = std::min(npos - 1, i0 - 1) - 1;
    f[i - 1] = std::max(0.0, std::min(1.0, (pos[i0 - 1] - x) / (pos[i0 - 1] - pos[i0 - 2])));
  }
}

// get_appl's moving-profile branch (applied.f90:896-903: set, then interpolate
// :1471-1520 with the time scale s) and get_applied's average over each
// grain's cells (field.f90:546-560): h_app per grain into ha[3 N]
static void table_field(const Sim* s, const Layer& Ly, double t, double sc, std::vector<double>& ha) {
  std::vector<int> ix, iy;
  std::vector<double> fx, fy;
  set_weights(Ly.tox + Ly.tvx * (t - Ly.tt0) - Ly.trx, s->nx, s->dx, Ly.tab_x, ix, fx);
  set_weights(Ly.toy + Ly.tvy * (t - Ly.tt0) - Ly.try_, s->ny, s->dy, Ly.tab_y, iy, fy);
  auto F = [&](int c, int i, int j) { return Ly.tab_v[c + 3 * ((size_t)i + (size_t)Ly.tnx * j)]; };
  ha.assign(3 * (size_t)Ly.N, 0.0);
  for (int n = 0; n < Ly.N; ++n) {
    double y[3] = {0, 0, 0};
    for (int q = Ly.g2c_idx[n]; q < Ly.g2c_idx[n + 1]; ++q) {
      const int i = Ly.g2c_i[q], j = Ly.g2c_j[q];
      const double yf = sc * fy[j], yfc = sc * (1.0 - fy[j]);
      for (int c = 0; c < 3; ++c)
        y[c] += fx[i] * yf * F(c, ix[i], iy[j]) + (1.0 - fx[i]) * yf * F(c, ix[i] + 1, iy[j]) +
                fx[i] * yfc * F(c, ix[i], iy[j] + 1) + (1.0 - fx[i]) * yfc * F(c, ix[i] + 1, iy[j] + 1);
    }
    const double k = (double)(Ly.g2c_idx[n + 1] - Ly.g2c_idx[n]);
    for (int c = 0; c < 3; ++c) ha[3 * n + c] = y[c] / k;
  }
}

// Karlqvist field of a ring head at down-track offset u from the gap centre,
// distance z below it, deep-gap field hg (polarity included)
static void karlqvist(double u, double g, double z, double hg, double* hx, double* hz) {
  const double a = u + 0.5 * g, b = u - 0.5 * g;
  *hx = hg / M_PI * (std::atan(a / z) - std::atan(b / z));
  *hz = hg / (2.0 * M_PI) * std::log((b * b + z * z) / (a * a + z * z));
}

static double head_polarity(const Layer& Ly, double t) {
  long long k = (long long)std::floor((t - Ly.hd_t0) / Ly.hd_tbit);
  const long long nb = Ly.hd_nbits > 0 ? Ly.hd_nbits : 1;
  k %= nb;
  if (k < 0) k += nb;
  return ((Ly.hd_bits >> k) & 1ull) ? 1.0 : -1.0;
}

// x**n, n a non-negative integer (real**integer by squaring)
static double ipow(double x, int n) {
  double r = 1.0;
  while (n > 0) {
    if (n & 1) r *= x;
    x *= x;
    n >>= 1;
  }
  return r;
}

// the grains' temperatures at t (get_appl's temperature branch, applied.f90:
// 889-896 with set_sg / get_sg :1778-1809, then get_applied's average over a
// grain's cells plus the background, field.f90:546-560)
static void grain_temps(const Sim* s, Layer& Ly, double t) {
  Ly.temp.assign(Ly.N, Ly.temperature);
  if (!Ly.tprof) return;
  double sc;
  if (Ly.tp_func != 0) {
    sc = (Ly.tp_amp * funct(Ly.tp_func, t, Ly.tp_fgamma, Ly.tp_phase, Ly.tp_param, Ly.tp_duty, Ly.tp_moddepth) +
          Ly.tp_dc) * Ly.tp_scale;
  } else {
    const double u = std::max(0.0, std::min(1.0, (t - Ly.tp_t_start) / (Ly.tp_t_end - Ly.tp_t_start)));
    sc = ((Ly.tp_s_end - Ly.tp_s_start) * u + Ly.tp_s_start) * Ly.tp_scale;
  }
  const double sdt = Ly.tp_dtemp * sc;
  std::vector<double> fx(s->nx), fy(s->ny);
  const double delx = Ly.tp_rx - Ly.tp_vx * (t - Ly.tp_t0) - Ly.tp_ox, dely = Ly.tp_ry - Ly.tp_vy * (t - Ly.tp_t0) - Ly.tp_oy;
  for (int i = 1; i <= s->nx; ++i) fx[i - 1] = std::exp(-ipow((s->dx * (i - 0.5) + delx) * Ly.tp_isx, Ly.tp_expn));
  for (int j = 1; j <= s->ny; ++j) fy[j - 1] = std::exp(-ipow((s->dy * (j - 0.5) + dely) * Ly.tp_isy, Ly.tp_expn));
  for (int n = 0; n < Ly.N; ++n) {
    double x = 0.0;
    for (int q = Ly.g2c_idx[n]; q < Ly.g2c_idx[n + 1]; ++q) x += sdt * fy[Ly.g2c_j[q]] * fx[Ly.g2c_i[q]];
    Ly.temp[n] = x / (double)(Ly.g2c_idx[n + 1] - Ly.g2c_idx[n]) + Ly.tp_bg;
  }
}

// file_temp_scaling's reduction of a table as read (temp_scaling.f90:152-203):
// sorted by temperature (ties keep their order), equal temperatures merged
// pairwise from the top with the mean of their scales, an equal first pair of
// scales and an equal last pair trimmed, and the temperatures divided by the
// largest when it exceeds 5 (a table in K, normalised to T/Tc)
void reduce_scaling_table(int n, const double* t_in, const double* v_in, std::vector<double>& t_out,
                          std::vector<double>& v_out) {
  std::vector<std::pair<double, double>> d(n);
  for (int i = 0; i < n; ++i) d[i] = {t_in[i], v_in[i]};
  std::stable_sort(d.begin(), d.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
  std::vector<double> t(n), v(n);
  for (int i = 0; i < n; ++i) {
    t[i] = d[i].first;
    v[i] = d[i].second;
  }
  int k = 0;
  for (int i = n - 1; i >= 1; --i)  // 1-based i = n .. 2
    if (t[i - 1] == t[i]) {
      ++k;
      v[i - 1] = 0.5 * (v[i - 1] + v[i]);
      for (int j = i + 1; j < n; ++j) {  // 1-based j = i+1 .. n: entry j moves to j-1
        t[j - 1] = t[j];
        v[j - 1] = v[j];
      }
    }
  int m = std::max(1, n - k);
  if (m >= 2 && v[0] == v[1]) {
    for (int i = 1; i < m; ++i) {
      t[i - 1] = t[i];
      v[i - 1] = v[i];
    }
    --m;
  }
  if (m > 1 && v[m - 2] == v[m - 1]) --m;
  if (t[m - 1] > 5.0) {
    const double top = t[m - 1];
    for (int i = 0; i < m; ++i) t[i] /= top;
  }
  t_out.assign(t.begin(), t.begin() + m);
  v_out.assign(v.begin(), v.begin() + m);
}

// a scaling table at x = T/Tc: its first scale below the first node, its last
// above the last, linear in between (bisection, temp_scaling.f90:397-414)
static double table_scale(const std::vector<double>& tt, const std::vector<double>& vv, double x) {
  const int n = (int)tt.size();
  int k1 = 0, k2 = n - 1;
  double y;
  if (x <= tt[0]) {
    y = 0.0;
  } else if (x >= tt[k2]) {
    y = 0.0;
    k1 = k2;
  } else {
    while (k2 - k1 > 1) {
      const int k = (k2 + k1 + 2) / 2 - 1;  // the reference's (k2 + k1) / 2 on 1-based indices
      if (x < tt[k]) k2 = k;
      else k1 = k;
    }
    y = std::max(0.0, std::min(1.0, (x - tt[k1]) / (tt[k2] - tt[k1])));
  }
  return vv[k1] + y * (vv[k2] - vv[k1]);
}

// find_temp_scaling (temp_scaling.f90:365-430): the grains' ms_scale,
// alpha_scale and hk_scale from their temperature (the last grain_temps) and
// Tc, or ms_scale from |m| of buffer buf; tables with one node scale nothing
static void find_temp_scaling(Layer& Ly, int buf) {
  if (!Ly.tsc) return;
  std::vector<double>* val[3] = {&Ly.ms_scale, &Ly.alpha_scale, &Ly.hk_scale};
  for (int i = 0; i < 3; ++i) {
    std::vector<double>& v = *val[i];
    if (i == 0 && Ly.tsc_mag) {
      for (int n = 0; n < Ly.N; ++n) v[n] = std::min(1.0, std::max(0.0, std::abs(Ly.mag[buf][n])));
    } else if ((i == 0 && Ly.tsc_msexp >= 0.0) || (i == 2 && Ly.tsc_hkexp >= 0.0)) {
      const double e = i == 0 ? Ly.tsc_msexp : Ly.tsc_hkexp;
      for (int n = 0; n < Ly.N; ++n)
        v[n] = std::pow(std::min(1.0, std::max(0.0, 1.0 - Ly.temp[n] / Ly.tsc_tc[n])), e);
    } else if (Ly.tsc_t[i].size() > 1) {
      for (int n = 0; n < Ly.N; ++n)
        if (Ly.do_grain[n]) v[n] = table_scale(Ly.tsc_t[i], Ly.tsc_v[i], Ly.temp[n] / Ly.tsc_tc[n]);
    }
  }
}

// get_field (field.f90:160-273) for the LLG path; energy per grain summed into *energy
static void get_field(Sim* s, double t, int buf, double* energy) {
  // get_applied first (field.f90:183): the grains' temperatures and their
  // scaling, which the demag source already uses
  for (int l = 0; l < s->nl; ++l) {
    grain_temps(s, s->L[l], t);
    find_temp_scaling(s->L[l], buf);
  }
  compute_demag(s, buf);
  double e_tot = 0.0;
  for (int l = 0; l < s->nl; ++l) {
    Layer& Ly = s->L[l];
    double sc = Ly.head ? 0.0 : ramp_scale(Ly, t);
    std::vector<double> hat;
    if (Ly.tab) table_field(s, Ly, t, sc, hat);
    const double* m = Ly.m[buf].data();
    const double pol = Ly.head ? head_polarity(Ly, t) : 0.0;
    const double xh = Ly.hd_x0 + Ly.hd_v * (t - Ly.hd_t0);
    double el = 0.0;
#pragma omp parallel for reduction(+ : el)
    for (int n = 0; n < Ly.N; ++n) {
      if (!Ly.do_grain[n]) continue;  // field.f90:199-233 (a frozen grain keeps its last field)
      double ha[3] = {sc * Ly.hdir[0], sc * Ly.hdir[1], sc * Ly.hdir[2]};
      if (Ly.func == 7) {  // ROT: rot_fld's direction (cos, sin((2 gamma t + phase) acos(-1)), 0)
        const double th = (2.0 * Ly.fgamma * t + Ly.phase) * std::acos(-1.0);
        ha[0] = sc * std::cos(th);
        ha[1] = sc * std::sin(th);
        ha[2] = 0.0;
      }
      if (Ly.tab)
        for (int a = 0; a < 3; ++a) ha[a] = hat[3 * n + a];
      if (Ly.head) {
        // the grain's down-track position: centre of its (first) cell column
        const double x = ((double)Ly.g2c_i[Ly.g2c_idx[n]] + 0.5) * s->dx;
        double hx, hz;
        karlqvist(x - xh, Ly.hd_gap, Ly.hd_z, pol * Ly.hd_hg, &hx, &hz);
        ha[0] += hx;
        ha[2] += hz;
      }
      for (int a = 0; a < 3; ++a) Ly.happ[3 * n + a] = ha[a];
      const double* mn = m + 3 * n;
      const double* hd = &Ly.hdemag[3 * n];
      double en = -(mn[0] * (hd[0] + ha[0]) + mn[1] * (hd[1] + ha[1]) + mn[2] * (hd[2] + ha[2])) *
                  Ly.ms[n] * Ly.ms_scale[n];
      double h[3] = {ha[0] + hd[0], ha[1] + hd[1], ha[2] + hd[2]};
      // get_cubic_hk field.f90:377-395: direction cosines d1 in the crystal
      // frame, h = -hk_scale * A d3, d3_i = d1_i (K1 (d1_j^2 + d1_k^2) + K2 d1_j^2 d1_k^2);
      // the energy term keeps the reference's factors as written (:392-394)
      if (!Ly.cax.empty() && Ly.hk_scale[n] > 0.0) {
        const double* A = &Ly.cax[9 * n];
        double d1[3], d2[3], d3[3];
        for (int i = 0; i < 3; ++i) {
          d1[i] = A[3 * i] * mn[0] + A[3 * i + 1] * mn[1] + A[3 * i + 2] * mn[2];
          d2[i] = d1[i] * d1[i];
        }
        const double K1 = Ly.hk[2 * n], K2 = Ly.hk[2 * n + 1], hs = Ly.hk_scale[n];
        d3[0] = d1[0] * (K1 * (d2[1] + d2[2]) + K2 * d2[1] * d2[2]);
        d3[1] = d1[1] * (K1 * (d2[0] + d2[2]) + K2 * d2[0] * d2[2]);
        d3[2] = d1[2] * (K1 * (d2[0] + d2[1]) + K2 * d2[0] * d2[1]);
        for (int k = 0; k < 3; ++k) h[k] -= (A[k] * d3[0] + A[k + 3] * d3[1] + A[k + 6] * d3[2]) * hs;
        en += 0.5 * hs * Ly.ms[n] *
              (K1 * (d2[0] * d2[1] + d2[0] * d2[2] + d2[1] * d2[2]) + K2 * d2[0] * d2[1] * d2[2]) * hs * Ly.ms[n] *
              Ly.ms_scale[n];
      }
      // get_uni_hk field.f90:366-375 (no uniaxial axis on a cubic layer)
      if (Ly.cax.empty() && Ly.hk_scale[n] > 0.0) {
        const double* k = &Ly.axis[3 * n];
        double hks = mn[0] * k[0] + mn[1] * k[1] + mn[2] * k[2];
        double yy = 1.0 - hks * hks;
        double f = hks * (Ly.hk[2 * n] + Ly.hk[2 * n + 1] * yy) * Ly.hk_scale[n];
        for (int a = 0; a < 3; ++a) h[a] += f * k[a];
        en += 0.5 * yy * (Ly.hk[2 * n] + 0.5 * Ly.hk[2 * n + 1] * yy) * Ly.hk_scale[n] * Ly.ms[n] *
              Ly.ms_scale[n];
      }
      // get_intralayer_hx field.f90:350-363
      if (!Ly.hx_idx.empty()) {
        double hx[3] = {0, 0, 0};
        for (int q = Ly.hx_idx[n]; q < Ly.hx_idx[n + 1]; ++q) {
          int j = Ly.hx_nbr[q];
          double c = Ly.hx[q] * Ly.ms_scale[j];
          for (int a = 0; a < 3; ++a) hx[a] += c * m[3 * j + a];
        }
        en += -(hx[0] * mn[0] + hx[1] * mn[1] + hx[2] * mn[2]) * Ly.ms[n] * Ly.ms_scale[n];
        for (int a = 0; a < 3; ++a) h[a] += hx[a];
      }
      // get_interlayer_hx field.f90:326-348 (upper = layer l-1, lower = layer l+1)
      for (int side = 0; side < 2; ++side) {
        const std::vector<int>& idx = side == 0 ? Ly.uhx_idx : Ly.lhx_idx;
        const std::vector<int>& nbr = side == 0 ? Ly.uhx_nbr : Ly.lhx_nbr;
        const std::vector<double>& cf = side == 0 ? Ly.uhx : Ly.lhx;
        if (idx.empty()) continue;
        const Layer& Q = s->L[side == 0 ? l - 1 : l + 1];
        const double* mq = Q.m[buf].data();
        double hv[3] = {0, 0, 0};
        for (int q = idx[n]; q < idx[n + 1]; ++q) {
          int j = nbr[q];
          double c = cf[q] * Q.ms_scale[j];
          for (int a = 0; a < 3; ++a) hv[a] += c * mq[3 * j + a];
        }
        en += -(hv[0] * mn[0] + hv[1] * mn[1] + hv[2] * mn[2]) * Ly.ms_scale[n] * Ly.ms[n];
        for (int a = 0; a < 3; ++a) h[a] += hv[a];
      }
      for (int a = 0; a < 3; ++a) Ly.h[3 * n + a] = h[a];
      el += en * Ly.vol[n];
    }
    e_tot += el;
  }
  if (energy) *energy = e_tot;
}

// get_thermal (field.f90:397-436).  The LLB and MT runs draw it with no_ms_p
// (get_fields, llg.f90:363-365: llgp%llb or llgp%mt), the others through the
// |m| and ms_scale branches.
static void get_thermal(Sim* s) {
  const double kB = 1.380662e-16;
  for (int l = 0; l < s->nl; ++l) {
    Layer& Ly = s->L[l];
    if (!Ly.thermal) {
      std::fill(Ly.hthm.begin(), Ly.hthm.end(), 0.0);
      continue;
    }
    double tsigma = std::sqrt(2.0 * kB * Ly.alpha / Ly.gamma);
    for (int n = 0; n < Ly.N; ++n) {
      if (!Ly.do_grain[n]) continue;
      double x = 0.0;
      const double Tn = Ly.temp.empty() ? Ly.temperature : Ly.temp[n];  // field(i)%temp(n)
      if (Ly.llb && Ly.mode != 2)  // no_ms_p (field.f90:414-415)
        x = Ly.alpha_scale[n] * Tn / (Ly.ms[n] * Ly.vol[n]);
      else if (Ly.mag[s->in][n] != 1.0)  // field.f90:416-417
        x = Ly.alpha_scale[n] * Tn / (Ly.ms[n] * Ly.vol[n] * std::max(Ly.floor_ms, std::abs(Ly.mag[s->in][n])));
      else if (Ly.ms_scale[n] > 0.0)
        x = Ly.alpha_scale[n] * Tn / (Ly.ms[n] * Ly.vol[n] * std::max(Ly.floor_ms, Ly.ms_scale[n]));
      x = std::sqrt(x) * tsigma;
      double r[3];
      if (s->rng_mode == 0) {
        // random_normal3d (random.f90:231-249)
        for (int a = 0; a < 3; ++a) r[a] = mt_normal(&Ly.rng);
      } else {
        philox_normal3(s->seed, (uint64_t)l, (uint64_t)s->step, (uint64_t)n, r);
      }
      for (int a = 0; a < 3; ++a) Ly.hthm[3 * n + a] = x * r[a];
    }
  }
}

static inline void cross(const double* a, const double* b, double* c) {
  // transform.f90:16-20
  c[0] = a[1] * b[2] - a[2] * b[1];
  c[1] = a[2] * b[0] - a[0] * b[2];
  c[2] = a[0] * b[1] - a[1] * b[0];
}

// lv(x) = coth(x) - 1/x and its derivative (llg.f90:704-710,727-733)
static double lv(double x) { return std::abs(x) > 1e-2 ? 1.0 / std::tanh(x) - 1.0 / x : x / 3.0; }
static double dlv(double x) {
  if (std::abs(x) > 4e-3) {
    const double b = std::sinh(x);
    return 1.0 / (x * x) - 1.0 / (b * b);
  }
  return 1.0 / 3.0;
}

// push_llb (llg.f90:916-1064): the semi-implicit (|type| = 2, :935-999) and
// Heun (:1000-1047) branches and the |m| = 0 branch (:1048-1060), for one
// layer; iter 2: the first pass of a two-pass push, 1: the last (or only).
static void push_llb(Sim* s, int l, int type, int iter, double dt, double dt0, double* errmx_l, double* errmx1_l,
                     double* mmag1) {
  Layer& Ly = s->L[l];
  const int id = s->in;
  const double gmub_kb = 1.343427768e-4;  // llg.f90:924
  const double scale1 = -0.5 * Ly.gamma * dt;
  double em = 0.0, em1 = 0.0, mm = 0.0;
#pragma omp parallel for reduction(max : em, em1) reduction(+ : mm)
  for (int n = 0; n < Ly.N; ++n) {
    if (n < Ly.min_n || n > Ly.max_n) continue;
    const double T = Ly.temp[n];  // p%temp(n) of the last field evaluation
    double* mnext = &Ly.m[1 - id][3 * n];
    const double* mcur = &Ly.m[id][3 * n];
    double& magn = Ly.mag[1 - id][n];
    const double magc = Ly.mag[id][n];
    const double* hn = &Ly.h[3 * n];
    if (!Ly.do_grain[n]) {  // llg.f90:1061-1064 (the magnitude kept too)
      for (int a = 0; a < 3; ++a) {
        mnext[a] = mcur[a];
        Ly.dm[3 * n + a] = 0.0;
      }
      magn = magc;
      mm += magn * Ly.vol[n];
      continue;
    }
    const double lambdam = Ly.lam_ms[n] * (Ly.spin + 1.0) / Ly.spin;  // :931
    const double tc = Ly.tc[n];
    if (magc > 0.0 && std::abs(type) < 3) {
      // semi-implicit push of direction and magnitude (:935-999)
      const double scale11 = scale1;
      double m[3], mag, htot[3], mhtot, meq;
      auto tot = [&](const double* mm, double mg) {
        for (int a = 0; a < 3; ++a) htot[a] = hn[a] + lambdam * mg * mm[a];
        mhtot = std::sqrt(htot[0] * htot[0] + htot[1] * htot[1] + htot[2] * htot[2]);
        if (mhtot != 0.0)
          for (int a = 0; a < 3; ++a) htot[a] /= mhtot;
        meq = gmub_kb * Ly.spin * mhtot / T;
      };
      if (iter == 2 || type > 0) {
        for (int a = 0; a < 3; ++a) m[a] = mcur[a];
        mag = magc;
        tot(m, mag);
        mag = lv(meq) * (m[0] * htot[0] + m[1] * htot[1] + m[2] * htot[2]);
        mag = mag + (magc - mag) * std::exp(scale1 * 2.0 * Ly.alpha * lambdam * lambdam * T * T * lv(meq) /
                                            (3.0 * tc * tc * dlv(meq) * (mhtot + 1e-20)));
      } else {
        for (int a = 0; a < 3; ++a) m[a] = mnext[a];
        mag = magn;
      }
      tot(m, mag);
      const double aperp = Ly.alpha * (1.0 - lambdam * lv(meq) * T / (3.0 * mhtot * tc));
      const double apar = Ly.alpha * 2.0 * T / (3.0 * tc);
      const double scale2 = -aperp / (std::abs(mag) + 1e-20);
      double h[3], t[3], o[3], mo[3], tt[3], d[3];
      const double fh = std::sqrt(std::abs(scale2 / (Ly.alpha * Ly.alpha_scale[n] * dt0 * (std::abs(mag) + 1e-20))));
      for (int a = 0; a < 3; ++a) h[a] = hn[a] + Ly.hthm[3 * n + a] * fh;
      for (int a = 0; a < 3; ++a) m[a] = mcur[a];
      cross(m, h, t);
      const double y2 = t[0] * t[0] + t[1] * t[1] + t[2] * t[2];
      const double ms2 = Ly.ms[n] * Ly.ms[n];
      if (y2 > em * ms2) em = y2 / ms2;
      for (int a = 0; a < 3; ++a) o[a] = scale11 * h[a] + scale2 * m[a];
      cross(m, o, mo);
      for (int a = 0; a < 3; ++a) tt[a] = m[a] + mo[a];
      const double yy = 2.0 / (1.0 + o[0] * o[0] + o[1] * o[1] + o[2] * o[2]);
      cross(tt, o, d);
      for (int a = 0; a < 3; ++a) {
        d[a] *= yy;
        mnext[a] = m[a] + d[a];
      }
      double mm2[3];
      for (int a = 0; a < 3; ++a) mm2[a] = m[a] + 0.5 * d[a];
      tot(mm2, mag);
      const double sg = std::copysign(1.0, mag);
      mag = lv(meq) * (sg * mm2[0] * htot[0] + sg * mm2[1] * htot[1] + sg * mm2[2] * htot[2]);
      double q = mag + (magc - mag) * std::exp(scale1 * 4.0 * Ly.alpha * lambdam * lambdam * T * T * lv(meq) /
                                               (3.0 * tc * tc * dlv(meq) * (mhtot + 1e-20)));
      const double fp = std::sqrt(std::abs(apar / (Ly.alpha * Ly.alpha_scale[n] * dt0)));
      q = q - 2.0 * scale11 * (Ly.hthm[3 * n] * fp * mm2[0] + Ly.hthm[3 * n + 1] * fp * mm2[1] +
                               Ly.hthm[3 * n + 2] * fp * mm2[2]);
      magn = std::abs(q);
      if (q < 0.0) {
        const double r = std::sqrt(mm2[0] * mm2[0] + mm2[1] * mm2[1] + mm2[2] * mm2[2]);
        for (int a = 0; a < 3; ++a) {
          mnext[a] = -mm2[a] / r;
          d[a] = mnext[a] - m[a];
        }
      }
      const double ya = 0.5 * (magn + magc);
      double e[3];
      for (int a = 0; a < 3; ++a) e[a] = d[a] * ya + m[a] * (magn - magc);
      em1 = std::max(em1, e[0] * e[0] + e[1] * e[1] + e[2] * e[2]);
    } else if (magc > 0.0) {
      double m[3], mag;
      if (iter == 1) {
        for (int a = 0; a < 3; ++a) m[a] = mnext[a];
        mag = magn;
        if (mag <= 0.0) {
          mag = 0.0;
          const double y = std::sqrt(hn[0] * hn[0] + hn[1] * hn[1] + hn[2] * hn[2]);
          if (y != 0.0)
            for (int a = 0; a < 3; ++a) m[a] = hn[a] / y;
        }
      } else {
        for (int a = 0; a < 3; ++a) m[a] = mcur[a];
        mag = magc;
      }
      double htot[3];
      for (int a = 0; a < 3; ++a) htot[a] = hn[a] + lambdam * mag * m[a];
      const double mhtot = std::sqrt(htot[0] * htot[0] + htot[1] * htot[1] + htot[2] * htot[2]);
      if (mhtot != 0.0)
        for (int a = 0; a < 3; ++a) htot[a] /= mhtot;
      double meq = gmub_kb * Ly.spin * mhtot / T;
      const double aperp = Ly.alpha * (1.0 - lambdam * lv(meq) * T / (3.0 * mhtot * tc));
      const double apar = Ly.alpha * 2.0 * T / (3.0 * tc);
      double h[3], hpar[3], hperp[3];
      const double rt = std::sqrt(Ly.alpha * Ly.alpha_scale[n] * dt0);
      for (int a = 0; a < 3; ++a) h[a] = Ly.hthm[3 * n + a] / rt;
      const double hm = h[0] * m[0] + h[1] * m[1] + h[2] * m[2];
      for (int a = 0; a < 3; ++a) {
        hpar[a] = hm * m[a];
        hperp[a] = h[a] - hpar[a];
      }
      const double fpar = std::sqrt(apar), fperp = std::sqrt(std::max(0.0, aperp - apar) / (aperp * aperp));
      for (int a = 0; a < 3; ++a) {
        hpar[a] *= fpar;
        hperp[a] *= fperp;
      }
      const double scale11 = 2.0 * scale1;  // (type -3: no rescaling, :1029)
      const double mht = m[0] * htot[0] + m[1] * htot[1] + m[2] * htot[2];
      meq = apar * (lambdam / mhtot) * lambdam * 2.0 * scale1 * T * lv(meq) / (3.0 * dlv(meq) * tc) *
            (mag - lv(meq) * mht);
      double hh[3] = {hn[0] + hperp[0], hn[1] + hperp[1], hn[2] + hperp[2]}, t[3], mh[3], mt[3], d[3];
      cross(m, hh, t);
      cross(m, hn, mh);
      cross(m, t, mt);
      const double sg = std::copysign(std::min(0.5, std::abs(meq)), meq);
      for (int a = 0; a < 3; ++a) d[a] = scale11 * (mag * mh[a] + aperp * mt[a] + hpar[a]) + sg * m[a];
      if (iter == 1) {
        for (int a = 0; a < 3; ++a) d[a] = 0.5 * (d[a] + Ly.dm[3 * n + a]);
      } else {
        for (int a = 0; a < 3; ++a) Ly.dm[3 * n + a] = d[a];
      }
      const double y2 = t[0] * t[0] + t[1] * t[1] + t[2] * t[2];
      const double ms2 = Ly.ms[n] * Ly.ms[n];
      if (y2 > em * ms2) em = y2 / ms2;
      em1 = std::max(em1, d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
      double o[3];
      for (int a = 0; a < 3; ++a) o[a] = mcur[a] * magc + d[a];
      double y = std::sqrt(o[0] * o[0] + o[1] * o[1] + o[2] * o[2]);
      if (y > 0.0) {
        for (int a = 0; a < 3; ++a) mnext[a] = o[a] / y;
      } else {
        y = 0.0;
        for (int a = 0; a < 3; ++a) mnext[a] = -mcur[a];
      }
      magn = y;
    } else {
      const double y = std::sqrt(hn[0] * hn[0] + hn[1] * hn[1] + hn[2] * hn[2]);
      if (y > 0.0) {
        for (int a = 0; a < 3; ++a) mnext[a] = hn[a] / y;
        const double scale11 = 2.0 * scale1;
        const double meq = gmub_kb * Ly.spin * y / T;
        const double scale2 = lambdam * T / (3.0 * dlv(meq) * tc);
        magn = (y / scale2 + lv(meq)) * (1.0 - std::exp(scale11 * scale2 * 2.0 * T * Ly.alpha / (3.0 * tc)));
      } else {
        for (int a = 0; a < 3; ++a) mnext[a] = mcur[a];
        magn = magc;
      }
      em1 = std::max(em1, (magn - magc) * (magn - magc));
    }
    mm += magn * Ly.vol[n];
  }
  *errmx_l = em;
  *errmx1_l = em1;
  *mmag1 = mm;
}

// bs / dbs (llg.f90:390-408): Brillouin function and its derivative
static double bs(double x, double sp) {
  double b = x / (2.0 * sp);
  if (b != 0.0) b = ((2.0 * sp + 1.0) / std::tanh((2.0 * sp + 1.0) * b) - 1.0 / std::tanh(b)) / (2.0 * sp);
  return b;
}
static double dbs(double x, double sp) {
  double b = (1.0 + sp) / (3.0 * sp);
  if (x != 0.0) {
    b = x / (2.0 * sp);
    const double b1 = std::sinh(b);
    b = std::sinh(x + b);
    b = (1.0 / (b1 * b1) - (1.0 + 2.0 * sp) * (1.0 + 2.0 * sp) / (b * b)) / (4.0 * sp * sp);
  }
  return b;
}

// push_mt (llg.f90:735-915): the |type| = 2 explicit-rotation branch
// (:757-842) and the Heun branch (:843-906), for one layer.
static void push_mt(Sim* s, int l, int type, int iter, double dt, double dt0, double* errmx_l, double* errmx1_l,
                    double* mmag1) {
  Layer& Ly = s->L[l];
  const int id = s->in;
  const double gmub_kb = 1.343427768e-4;
  const double scale1 = -0.5 * Ly.gamma * dt, scale11 = 2.0 * scale1;
  const double sp = Ly.spin;
  double em = 0.0, em1 = 0.0, mm = 0.0;
#pragma omp parallel for reduction(max : em, em1) reduction(+ : mm)
  for (int n = 0; n < Ly.N; ++n) {
    if (n < Ly.min_n || n > Ly.max_n) continue;
    double* mnext = &Ly.m[1 - id][3 * n];
    const double* mcur = &Ly.m[id][3 * n];
    double& magn = Ly.mag[1 - id][n];
    double m[3] = {mcur[0], mcur[1], mcur[2]}, mag = Ly.mag[id][n];
    if (!Ly.do_grain[n]) {
      for (int a = 0; a < 3; ++a) {
        mnext[a] = m[a];
        Ly.dm[3 * n + a] = 0.0;
      }
      magn = mag;
      mm += magn * Ly.vol[n];
      continue;
    }
    const double T = Ly.temp[n];  // p%temp(n) of the last field evaluation
    double lambdam = Ly.lam_ms[n];
    if (!Ly.meq_bs) lambdam = lambdam * (sp + 1.0) / sp;
    double y = gmub_kb * sp / T;
    const double* hn = &Ly.h[3 * n];
    const double* th = &Ly.hthm[3 * n];
    const double ab = Ly.alpha_scale[n] * Ly.alpha;
    double htot[3], mhtot, meq, sig_p, sig_l, scale2, d[3], t[3], eta[3], o[3];
    auto norm_tot = [&]() {
      mhtot = std::sqrt(htot[0] * htot[0] + htot[1] * htot[1] + htot[2] * htot[2]);
      if (mhtot != 0.0)
        for (int a = 0; a < 3; ++a) htot[a] /= mhtot;
    };
    auto shape_eta = [&]() {  // eta = sqrt(sig_l/sig_p) (htot.eta) htot - htot x (htot x eta)
      double x1[3], x2[3];
      cross(htot, eta, x1);
      cross(htot, x1, x2);
      const double pe = htot[0] * eta[0] + htot[1] * eta[1] + htot[2] * eta[2];
      for (int a = 0; a < 3; ++a) eta[a] = std::sqrt(sig_l / sig_p) * pe * htot[a] - x2[a];
    };
    if (std::abs(type) < 3) {
      if (iter == 1 && type < 0) {
        for (int a = 0; a < 3; ++a) m[a] = mnext[a];
        mag = magn;
      }
      for (int a = 0; a < 3; ++a) htot[a] = hn[a] + lambdam * mag * m[a];
      norm_tot();
      meq = Ly.meq_bs ? bs(y * mhtot, sp) : lv(y * mhtot);
      if (Ly.garanin_tau) {
        sig_p = Ly.meq_bs ? meq / (y * mhtot * dbs(y * mhtot, sp) + 1e-80) : meq / (y * mhtot * dlv(y * mhtot) + 1e-80);
        scale2 = 2.0 * ab * sig_p / y;
      } else {
        scale2 = ab * lambdam;
      }
      if (iter == 1 && type < 0) {
        for (int a = 0; a < 3; ++a) m[a] = mcur[a];
        mag = Ly.mag[id][n];
      }
      cross(m, hn, t);
      const double y2 = t[0] * t[0] + t[1] * t[1] + t[2] * t[2];
      if (y2 > em * Ly.ms[n] * Ly.ms[n]) em = y2 / (Ly.ms[n] * Ly.ms[n]);
      // |type| = 2: explicit gyro-rotation and analytic decay (:801-803)
      for (int a = 0; a < 3; ++a) d[a] = (meq * htot[a] - mag * m[a]) * (1.0 - std::exp(scale1 * scale2));
      double w[3], r[3];
      for (int a = 0; a < 3; ++a) w[a] = mag * m[a] + d[a];
      cross(w, hn, r);
      for (int a = 0; a < 3; ++a) d[a] = d[a] + scale11 * r[a];
      for (int a = 0; a < 3; ++a) o[a] = mag * m[a] + d[a];
      for (int a = 0; a < 3; ++a) htot[a] = hn[a] + lambdam * o[a];
      norm_tot();
      if (Ly.meq_bs) {
        meq = bs(y * mhtot, sp);
        sig_p = meq / (y * mhtot + 1e-80);
        sig_l = dbs(y * mhtot, sp);
      } else {
        meq = lv(y * mhtot);
        sig_p = meq / (y * mhtot + 1e-80);
        sig_l = dlv(y * mhtot);
      }
      if (Ly.garanin_tau) {
        for (int a = 0; a < 3; ++a)
          eta[a] = dt * th[a] * Ly.gamma * sig_p * std::sqrt(2.0 / ((sig_l + 1e-80) * dt0));
        scale2 = 2.0 * ab * sig_p / (y * (sig_l + 1e-80));
      } else {
        for (int a = 0; a < 3; ++a) eta[a] = dt * th[a] * Ly.gamma * std::sqrt(lambdam * meq / ((mhtot + 1e-80) * dt0));
      }
      shape_eta();
      for (int a = 0; a < 3; ++a) d[a] = d[a] + (meq * htot[a] - o[a]) * (1.0 - std::exp(scale1 * scale2)) + eta[a];
      em1 = std::max(em1, d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    } else {
      if (iter == 1) {
        for (int a = 0; a < 3; ++a) m[a] = mnext[a];
        mag = magn;
        if (mag <= 0.0) {
          mag = 0.0;
          const double e = std::sqrt(hn[0] * hn[0] + hn[1] * hn[1] + hn[2] * hn[2]);
          if (e != 0.0)
            for (int a = 0; a < 3; ++a) m[a] = hn[a] / e;
        }
      }
      for (int a = 0; a < 3; ++a) htot[a] = hn[a] + lambdam * mag * m[a];
      norm_tot();
      y = y * mhtot;
      if (Ly.meq_bs) {
        meq = bs(y, sp);
        sig_l = dbs(y, sp);
        sig_p = meq / (y + 1e-22);
      } else {
        meq = lv(y);
        sig_l = dlv(y);
        sig_p = meq / (y + 1e-22);
      }
      if (Ly.garanin_tau) {
        for (int a = 0; a < 3; ++a)
          eta[a] = dt * th[a] * Ly.gamma * sig_p * std::sqrt(2.0 / ((sig_l + 1e-22) * dt0));
        shape_eta();
        scale2 = 2.0 * T * sig_p / (gmub_kb * sp * (sig_l + 1e-22));
      } else {
        for (int a = 0; a < 3; ++a) eta[a] = dt * th[a] * Ly.gamma * std::sqrt(lambdam * meq / ((mhtot + 1e-22) * dt0));
        shape_eta();
        scale2 = lambdam;
      }
      double mmg[3], r[3];
      for (int a = 0; a < 3; ++a) mmg[a] = m[a] * mag;
      cross(mmg, hn, r);
      for (int a = 0; a < 3; ++a) d[a] = scale11 * (r[a] + (mmg[a] - meq * htot[a]) * scale2 * ab) + eta[a];
      if (iter == 1) {
        for (int a = 0; a < 3; ++a) d[a] = 0.5 * (d[a] + Ly.dm[3 * n + a]);
      } else {
        for (int a = 0; a < 3; ++a) Ly.dm[3 * n + a] = d[a];
      }
      cross(m, hn, t);
      const double y2 = t[0] * t[0] + t[1] * t[1] + t[2] * t[2];
      if (y2 > em * Ly.ms[n] * Ly.ms[n]) em = y2 / (Ly.ms[n] * Ly.ms[n]);
      em1 = std::max(em1, d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
      for (int a = 0; a < 3; ++a) m[a] = mcur[a];
      mag = Ly.mag[id][n];
    }
    for (int a = 0; a < 3; ++a) o[a] = m[a] * mag + d[a];
    double e = std::sqrt(o[0] * o[0] + o[1] * o[1] + o[2] * o[2]);
    if (e > 0.0) {
      for (int a = 0; a < 3; ++a) mnext[a] = o[a] / e;
    } else {
      e = 0.0;
      for (int a = 0; a < 3; ++a) mnext[a] = -m[a];
    }
    magn = e;
    mm += magn * Ly.vol[n];
  }
  *errmx_l = em;
  *errmx1_l = em1;
  *mmag1 = mm;
}

// push_zhang (llg.f90:410-703): the |type| = 2 explicit-rotation branch
// (:428-510) and the Heun branch (:633-700), for one layer.
static void push_zhang(Sim* s, int l, int type, int iter, double dt, double dt0, double* errmx_l, double* errmx1_l,
                       double* mmag1) {
  Layer& Ly = s->L[l];
  const int id = s->in;
  const double gmub_kb = 1.343427768e-4;
  const double scale1 = -0.5 * Ly.gamma * dt;
  const double sp = Ly.spin;
  double em = 0.0, em1 = 0.0, mm = 0.0;
#pragma omp parallel for reduction(max : em, em1) reduction(+ : mm)
  for (int n = 0; n < Ly.N; ++n) {
    if (n < Ly.min_n || n > Ly.max_n) continue;
    double* mnext = &Ly.m[1 - id][3 * n];
    const double* mcur = &Ly.m[id][3 * n];
    double& magn = Ly.mag[1 - id][n];
    double m[3] = {mcur[0], mcur[1], mcur[2]}, mag = Ly.mag[id][n];
    if (!Ly.do_grain[n]) {
      for (int a = 0; a < 3; ++a) {
        mnext[a] = m[a];
        Ly.dm[3 * n + a] = 0.0;
      }
      magn = mag;
      mm += magn * Ly.vol[n];
      continue;
    }
    const double T = Ly.temp[n];
    double lambdam = Ly.lam_ms[n];
    if (!Ly.meq_bs) lambdam = lambdam * (sp + 1.0) / sp;
    double y = gmub_kb * sp / T;
    const double* hn = &Ly.h[3 * n];
    const double* th = &Ly.hthm[3 * n];
    double htot[3], mhtot, meq, scale2, d[3], t[3], o[3], h[3];
    auto norm_tot = [&]() {
      mhtot = std::sqrt(htot[0] * htot[0] + htot[1] * htot[1] + htot[2] * htot[2]);
      if (mhtot != 0.0)
        for (int a = 0; a < 3; ++a) htot[a] /= mhtot;
    };
    auto bsl = [&](double x) { return Ly.meq_bs ? bs(x, sp) : lv(x); };
    auto dbsl = [&](double x) { return Ly.meq_bs ? dbs(x, sp) : dlv(x); };
    if (std::abs(type) < 3) {
      if (iter == 1 && type < 0) {
        for (int a = 0; a < 3; ++a) m[a] = mnext[a];
        mag = magn;
      }
      for (int a = 0; a < 3; ++a) htot[a] = hn[a] + lambdam * mag * m[a];
      norm_tot();
      meq = bsl(y * mhtot);
      if (Ly.garanin_tau) {
        const double sig_p = meq / (y * mhtot * dbsl(y * mhtot) + 1e-80);
        scale2 = 2.0 * sig_p / y;
      } else {
        scale2 = lambdam;
      }
      double hthm[3];
      for (int a = 0; a < 3; ++a) hthm[a] = th[a] * std::sqrt(std::abs(scale2 * meq / (mhtot * mag * dt0 + 1e-80)));
      scale2 = Ly.alpha * Ly.alpha_scale[n] * scale2;
      if (iter == 1 && type < 0) {
        for (int a = 0; a < 3; ++a) m[a] = mcur[a];
        mag = Ly.mag[id][n];
      }
      for (int a = 0; a < 3; ++a) h[a] = hn[a] + hthm[a];
      cross(m, h, t);
      const double y2 = t[0] * t[0] + t[1] * t[1] + t[2] * t[2];
      if (y2 > em * Ly.ms[n] * Ly.ms[n]) em = y2 / (Ly.ms[n] * Ly.ms[n]);
      for (int a = 0; a < 3; ++a) d[a] = (meq * htot[a] - mag * m[a]) * (1.0 - std::exp(scale1 * scale2));
      double w[3], r[3];
      for (int a = 0; a < 3; ++a) w[a] = mag * m[a] + d[a];
      cross(w, h, r);
      for (int a = 0; a < 3; ++a) d[a] = d[a] + 2.0 * scale1 * r[a];
      for (int a = 0; a < 3; ++a) o[a] = mag * m[a] + d[a];
      for (int a = 0; a < 3; ++a) htot[a] = hn[a] + lambdam * o[a];
      norm_tot();
      meq = bsl(y * mhtot);
      if (Ly.garanin_tau) {
        const double sig_p = meq / (y * mhtot * dbsl(y * mhtot) + 1e-80);
        scale2 = 2.0 * sig_p / y;
      } else {
        scale2 = lambdam;
      }
      scale2 = Ly.alpha * Ly.alpha_scale[n] * scale2;
      for (int a = 0; a < 3; ++a) d[a] = d[a] + (meq * htot[a] - o[a]) * (1.0 - std::exp(scale1 * scale2));
      em1 = std::max(em1, d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    } else {
      const double scale11 = 2.0 * scale1;
      if (iter == 1) {
        for (int a = 0; a < 3; ++a) m[a] = mnext[a];
        mag = magn;
        if (mag <= 0.0) {
          mag = 0.0;
          y = std::sqrt(hn[0] * hn[0] + hn[1] * hn[1] + hn[2] * hn[2]);
          if (y != 0.0)
            for (int a = 0; a < 3; ++a) m[a] = hn[a] / y;
        }
      }
      for (int a = 0; a < 3; ++a) htot[a] = hn[a] + lambdam * mag * m[a];
      norm_tot();
      y = y * mhtot;
      meq = bsl(y);
      if (Ly.garanin_tau) {
        y = meq / (y * dbsl(y) + 1e-66);
        scale2 = 2.0 * T * y / (gmub_kb * sp);
      } else {
        scale2 = lambdam;
      }
      y = std::abs(scale2 * meq / (mhtot * mag + 1e-66));
      for (int a = 0; a < 3; ++a) h[a] = hn[a] + th[a] * std::sqrt(std::abs(y / dt0));
      scale2 = scale2 * Ly.alpha * Ly.alpha_scale[n];
      double mmg[3], r[3];
      for (int a = 0; a < 3; ++a) mmg[a] = m[a] * mag;
      cross(mmg, h, r);
      for (int a = 0; a < 3; ++a) d[a] = scale11 * (r[a] + (mmg[a] - meq * htot[a]) * scale2);
      if (iter == 1) {
        for (int a = 0; a < 3; ++a) d[a] = 0.5 * (d[a] + Ly.dm[3 * n + a]);
      } else {
        for (int a = 0; a < 3; ++a) Ly.dm[3 * n + a] = d[a];
      }
      cross(m, h, t);
      const double y2 = t[0] * t[0] + t[1] * t[1] + t[2] * t[2];
      if (y2 > em * Ly.ms[n] * Ly.ms[n]) em = y2 / (Ly.ms[n] * Ly.ms[n]);
      em1 = std::max(em1, d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
      for (int a = 0; a < 3; ++a) m[a] = mcur[a];
      mag = Ly.mag[id][n];
    }
    for (int a = 0; a < 3; ++a) o[a] = m[a] * mag + d[a];
    double e = std::sqrt(o[0] * o[0] + o[1] * o[1] + o[2] * o[2]);
    if (e > 0.0) {
      for (int a = 0; a < 3; ++a) mnext[a] = o[a] / e;
    } else {
      e = 0.0;
      for (int a = 0; a < 3; ++a) mnext[a] = -m[a];
    }
    magn = e;
    mm += magn * Ly.vol[n];
  }
  *errmx_l = em;
  *errmx1_l = em1;
  *mmag1 = mm;
}

// rotate_q (transform.f90:65-74): m -> w ** (0, m) ** w*
static void ref_rotate_q(const double w[4], const double m[3], double t[3]) {
  const double w1 = w[0] * w[0], w2 = w[1] * w[1], w3 = w[2] * w[2], w4 = w[3] * w[3];
  t[0] = 2.0 * (m[2] * (w[0] * w[2] + w[1] * w[3]) + m[1] * (w[1] * w[2] - w[0] * w[3])) + m[0] * (w1 + w2 - w3 - w4);
  t[1] = 2.0 * (m[0] * (w[0] * w[3] + w[1] * w[2]) + m[2] * (w[2] * w[3] - w[0] * w[1])) + m[1] * (w1 + w3 - w2 - w4);
  t[2] = 2.0 * (m[1] * (w[0] * w[1] + w[2] * w[3]) + m[0] * (w[1] * w[3] - w[0] * w[2])) + m[2] * (w1 + w4 - w3 - w2);
}

// rotate_2 (transform.f90:97-115) as push_llg calls it (norm0 present, norm1 absent)
static void ref_rotate_2(double theta0, const double u0[3], double theta1, const double u1[3], const double m[3],
                         double t[3]) {
  double st1 = 0.5 * theta1, st0 = 0.5 * theta0, ct0, ct1;
  double t0[3] = {u0[0], u0[1], u0[2]};
  ct0 = std::sqrt(t0[0] * t0[0] + t0[1] * t0[1] + t0[2] * t0[2]);
  if (ct0 != 0.0) {
    for (int a = 0; a < 3; ++a) t0[a] /= ct0;
  } else {
    t0[0] = 0.0; t0[1] = 0.0; t0[2] = 1.0;
    st0 = 0.0;
  }
  const double* t1 = u1;
  if (st0 == 0.0 && st0 == st1) {
    for (int a = 0; a < 3; ++a) t[a] = m[a];
    return;
  }
  ct1 = std::cos(st1); st1 = std::sin(st1);
  ct0 = std::cos(st0); st0 = std::sin(st0);
  const double w[4] = {ct0 * ct1 - (t0[0] * t1[0] + t0[1] * t1[1] + t0[2] * t1[2]) * st0 * st1,
                       t0[0] * ct1 * st0 + (t1[0] * ct0 + (t1[1] * t0[2] - t0[1] * t1[2]) * st0) * st1,
                       t0[1] * ct1 * st0 + (t1[1] * ct0 + (t1[2] * t0[0] - t0[2] * t1[0]) * st0) * st1,
                       t0[2] * ct1 * st0 + (t1[2] * ct0 + (t1[0] * t0[1] - t0[0] * t1[1]) * st0) * st1};
  ref_rotate_q(w, m, t);
}

// push_llg (llg.f90:1066-1155): one stage for one layer.
// Heun (type -3) branch :1122-1139, analytic rotations (|type| = 1)
// :1093-1107, Boris/semi-implicit (|type| = 2) :1109-1118.
static void push_llg(Sim* s, int l, int type, int iter, double dt, double dt0, double* errmx_l,
                     double* errmx1_l, double* mmag1) {
  Layer& Ly = s->L[l];
  const int id = s->in;  // current buffer; next buffer = 1-id
  const double scale1 = -0.5 * Ly.gamma * dt;
  double em = 0.0, em1 = 0.0, mm = 0.0;
  const double sdt0 = std::sqrt(dt0);
#pragma omp parallel for reduction(max : em, em1) reduction(+ : mm)
  for (int n = 0; n < Ly.N; ++n) {
    if (n < Ly.min_n || n > Ly.max_n) continue;  // llg.f90:1081
    double h[3];
    for (int a = 0; a < 3; ++a) h[a] = Ly.hthm[3 * n + a] / sdt0 + Ly.h[3 * n + a];
    double* mnext = &Ly.m[1 - id][3 * n];
    const double* mcur = &Ly.m[id][3 * n];
    if (!Ly.do_grain[n]) {
      // a frozen grain keeps its state (llg.f90:1149-1152)
      for (int a = 0; a < 3; ++a) {
        mnext[a] = mcur[a];
        Ly.dm[3 * n + a] = 0.0;
      }
    } else if (Ly.ms_scale[n] > 0.0) {
      double m[3] = {mcur[0], mcur[1], mcur[2]};
      double t[3], d[3], y;
      const double ms2 = Ly.ms[n] * Ly.ms[n];
      if (std::abs(type) < 3) {
        cross(m, h, t);
        y = t[0] * t[0] + t[1] * t[1] + t[2] * t[2];
        if (y > em * ms2) em = y / ms2;
        double scale2 = Ly.alpha_scale[n] * Ly.alpha;
        if (std::abs(type) != 2) {
          // analytic rotations (llg.f90:1093-1107): precession |scale11| about
          // h, damping turn th0 - 2 atan(exp(scale11 scale2) tan(th0/2)) about m x o
          double yv = h[0] * h[0] + h[1] * h[1] + h[2] * h[2];
          if (yv > 0.0) {
            yv = std::sqrt(yv);
            const double scale11 = 2.0 * scale1 * yv / (1.0 + scale2 * scale2);
            const double o[3] = {h[0] / yv, h[1] / yv, h[2] / yv};
            const double th0 = std::acos(std::min(1.0, std::max(-1.0, o[0] * m[0] + o[1] * m[1] + o[2] * m[2])));
            double mo[3], r[3];
            cross(m, o, mo);
            ref_rotate_2(th0 - 2.0 * std::atan(std::exp(scale11 * scale2) * std::tan(0.5 * th0)), mo,
                         std::abs(scale11), o, m, r);
            for (int a = 0; a < 3; ++a) d[a] = r[a] - m[a];
          } else {
            d[0] = d[1] = d[2] = 0.0;
          }
        } else {
          // |type| == 2: semi-implicit (Boris) push, llg.f90:1115-1118
          double o[3] = {scale1 * h[0] - scale2 * m[0], scale1 * h[1] - scale2 * m[1],
                         scale1 * h[2] - scale2 * m[2]};
          double mo[3];
          cross(m, o, mo);
          double tt[3] = {m[0] + mo[0], m[1] + mo[1], m[2] + mo[2]};
          double yy = 2.0 / (1.0 + o[0] * o[0] + o[1] * o[1] + o[2] * o[2]);
          double to[3];
          cross(tt, o, to);
          for (int a = 0; a < 3; ++a) d[a] = yy * to[a];
        }
        em1 = std::max(em1, d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
        for (int a = 0; a < 3; ++a) mnext[a] = m[a] + d[a];
      } else {
        double scale2 = Ly.alpha_scale[n] * Ly.alpha;
        double scale11 = 2.0 * scale1 / (1.0 + scale2 * scale2);
        if (iter == 1)
          for (int a = 0; a < 3; ++a) m[a] = mnext[a];  // second (corrector) stage
        cross(m, h, t);
        double mt[3];
        cross(m, t, mt);
        for (int a = 0; a < 3; ++a) d[a] = scale11 * (t[a] + scale2 * mt[a]);
        if (iter == 1) {
          for (int a = 0; a < 3; ++a) d[a] = 0.5 * (d[a] + Ly.dm[3 * n + a]);
        } else {
          for (int a = 0; a < 3; ++a) Ly.dm[3 * n + a] = d[a];
        }
        y = t[0] * t[0] + t[1] * t[1] + t[2] * t[2];
        if (y > em * ms2) em = y / ms2;
        em1 = std::max(em1, d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
        for (int a = 0; a < 3; ++a) mnext[a] = mcur[a] + d[a];
        y = mnext[0] * mnext[0] + mnext[1] * mnext[1] + mnext[2] * mnext[2];
        if (y > 0.0) {
          double r = std::sqrt(y);
          for (int a = 0; a < 3; ++a) mnext[a] /= r;
        }
      }
    } else {
      // ms_scale <= 0: m along h (llg.f90:1140-1148)
      double hh[3] = {Ly.h[3 * n], Ly.h[3 * n + 1], Ly.h[3 * n + 2]};
      double y = std::sqrt(hh[0] * hh[0] + hh[1] * hh[1] + hh[2] * hh[2]);
      if (y > 0.0)
        for (int a = 0; a < 3; ++a) mnext[a] = hh[a] / y;
      else
        for (int a = 0; a < 3; ++a) mnext[a] = mcur[a];
    }
    mm += std::sqrt(mnext[0] * mnext[0] + mnext[1] * mnext[1] + mnext[2] * mnext[2]) *
          Ly.ms_scale[n] * Ly.vol[n];
  }
  *errmx_l = em;
  *errmx1_l = em1;
  *mmag1 = mm;
}

static void compute_stats(Sim* s, double errmx, double errmx1, double mmag, double energy,
                          const double* errmx1_l) {
  Stats& st = s->last;
  std::memset(&st, 0, sizeof(st));
  for (int l = 0; l < s->nl; ++l) st.errmx1_l[l] = errmx1_l[l];
  st.t = s->t;
  st.step = s->step;
  double vtot = 0.0;
  for (int l = 0; l < s->nl; ++l) {
    Layer& Ly = s->L[l];
    const double* m = Ly.m[s->in].data();
    double V = 0, Mw = 0, sm[3] = {0, 0, 0}, sh[3] = {0, 0, 0}, sms[3] = {0, 0, 0};
    long long nup = 0;
    double hd[3] = {Ly.hdir[0], Ly.hdir[1], Ly.hdir[2]};
    for (int n = 0; n < Ly.N; ++n) {
      double v = Ly.vol[n];
      V += v;
      double w = Ly.ms[n] * Ly.ms_scale[n] * v;
      Mw += w;
      for (int a = 0; a < 3; ++a) {
        sm[a] += v * m[3 * n + a];
        sh[a] += v * Ly.h[3 * n + a];
        sms[a] += w * m[3 * n + a];
      }
      if (m[3 * n] * hd[0] + m[3 * n + 1] * hd[1] + m[3 * n + 2] * hd[2] > 0.0) ++nup;
    }
    double mv[3] = {0, 0, 0};
    for (int n = 0; n < Ly.N; ++n)
      for (int a = 0; a < 3; ++a) {
        double dd = m[3 * n + a] - sm[a] / V;
        mv[a] += Ly.vol[n] * dd * dd;
      }
    for (int a = 0; a < 3; ++a) {
      st.mave_l[l][a] = sm[a] / V;
      st.mvar_l[l][a] = mv[a] / V;
      st.have_l[l][a] = sh[a] / V;
      st.mms_l[l][a] = sms[a] * Mw / (Mw * Mw + 1e-300);
    }
    st.vol_l[l] = V;
    st.msvol_l[l] = Mw;
    st.nup_l[l] = nup;
    vtot += V;
  }
  for (int l = 0; l < s->nl; ++l)
    for (int a = 0; a < 3; ++a) {
      st.mave[a] += st.vol_l[l] * st.mave_l[l][a] / vtot;
      st.mvar[a] += st.vol_l[l] * st.mvar_l[l][a] / vtot;
      st.have[a] += st.vol_l[l] * st.have_l[l][a] / vtot;
    }
  st.errmx = errmx;
  st.errmx1 = errmx1;
  st.mmag = mmag;
  st.energy = energy;
}

// push_m's passes (llg.f90:1207-1266) at step dt with the field and thermal
// draw at t already in place: the new state is left in the other buffer (the
// caller toggles `in`, llg.f90:1269); per-layer max |dm|^2 of the last pass in e1l.
static void push_passes(Sim* s, double dt, int type, double* errmx, double* errmx1, double* mmag, double* e1l,
                        double* energy) {
  const int nl = s->nl;
  double dt_s = 1.0;
  int iter = 1;
  if (type < 0) {
    iter = 2;
    if (type > -3) dt_s = 0.5;
  }
  while (iter > 0) {
    *errmx = 0; *errmx1 = 0; *mmag = 0;
    for (int l = 0; l < nl; ++l) {
      double e0, e1, m1;
      if (s->L[l].llb && s->L[l].mode == 1)
        push_mt(s, l, type, iter, dt * dt_s, dt, &e0, &e1, &m1);
      else if (s->L[l].llb && s->L[l].mode == 2)
        push_zhang(s, l, type, iter, dt * dt_s, dt, &e0, &e1, &m1);
      else if (s->L[l].llb)
        push_llb(s, l, type, iter, dt * dt_s, dt, &e0, &e1, &m1);
      else
        push_llg(s, l, type, iter, dt * dt_s, dt, &e0, &e1, &m1);
      double vs = 0;  // sum(grain_vol, mask=do_grain), llg.f90:1239
      for (int n = 0; n < s->L[l].N; ++n)
        if (s->L[l].do_grain[n]) vs += s->L[l].vol[n];
      *mmag += m1 / vs;
      *errmx = std::max(*errmx, std::sqrt(e0));
      *errmx1 = std::max(*errmx1, e1);
      e1l[l] = e1;
    }
    iter -= 1;
    if (iter > 0) {
      // llg.f90:1262-1266: field at t+dt*dt_s on the predicted state, thermal reused
      s->in = 1 - s->in;
      get_field(s, s->t + dt * dt_s, s->in, energy);
      s->in = 1 - s->in;
      dt_s = 1.0;
    }
  }
}

// update_do_grain (data.f90:120-157) with get_window (:52-64): the window
// origin at time t, the grains with a cell inside it and their index range,
// and the copy of every grain's state into the other buffer (:139).
// Without a window every grain is pushed.
static void update_do_grain(Sim* s, double t) {
  for (auto& Ly : s->L) {
    if (s->wnx == 0) {
      Ly.do_grain.assign(Ly.N, 1);
      Ly.min_n = 0;
      Ly.max_n = Ly.N - 1;
      continue;
    }
  }
  if (s->wnx == 0) return;
  // off = v t + offset rounded as two operations (no fused multiply-add), so
  // that a half-cell tie in nint falls the same way on every build
  volatile double vtx = s->wvx * t, vty = s->wvy * t;
  const double offx = vtx + s->wox, offy = vty + s->woy;
  s->wi0 = std::max(1, std::min(s->nx - s->wnx + 1, (int)std::lround((s->nx - s->wnx) * 0.5 + offx / s->dx))) - 1;
  s->wj0 = std::max(1, std::min(s->ny - s->wny + 1, (int)std::lround((s->ny - s->wny) * 0.5 + offy / s->dy))) - 1;
  for (auto& Ly : s->L) {
    Ly.do_grain.assign(Ly.N, 0);
    Ly.min_n = Ly.N;
    Ly.max_n = -1;
    Ly.m[1 - s->in] = Ly.m[s->in];
    for (int j = s->wj0; j < s->wj0 + s->wny; ++j)
      for (int i = s->wi0; i < s->wi0 + s->wnx; ++i) {
        const int g = Ly.c2g[(size_t)j * s->nx + i];
        if (g < 0) continue;
        Ly.do_grain[g] = 1;
        Ly.min_n = std::min(Ly.min_n, g);
        Ly.max_n = std::max(Ly.max_n, g);
      }
  }
}

// One pass of the llg() loop body (llg.f90:240-269) with push_m (llg.f90:1195-1271)
// at fixed dt (fixed_dt_p: max_dmdt = 1, no retries).
static void heun_or_boris_step(Sim* s, double dt, int type) {
  double energy = 0.0;
  // get_fields(t): field + thermal at the current state (llg.f90:363-365)
  get_field(s, s->t, s->in, &energy);
  get_thermal(s);
  double errmx = 0, errmx1 = 0, mmag = 0, e1l[8] = {0};
  push_passes(s, dt, type, &errmx, &errmx1, &mmag, e1l, &energy);
  s->in = 1 - s->in;  // llg.f90:1269
  s->t += dt;
  s->step += 1;
  compute_stats(s, errmx, errmx1, mmag, energy, e1l);
  update_do_grain(s, s->t);  // llg.f90:284
}

// The same with the adaptive time step (dt_frac != 0): get_fields picks dt from
// the largest |h + hthm/sqrt(dt*max_dmdt)| (llg.f90:369-387); push_m retries
// from the unchanged state with max_dmdt *= 0.9/rot_ratio while the first layer
// (in order) whose rot_ratio = acos(1 - |dm|^2/2)/max_dm exceeds 1 says so, and
// sets the next max_dmdt (llg.f90:1225-1253,1270); dt becomes the step taken
// and t advances by it (llg.f90:268-269).
static void adaptive_step(Sim* s, int type, double dt_frac, double dt_max, const double* max_dm, double* dt,
                          double* max_dmdt) {
  double energy = 0.0;
  get_field(s, s->t, s->in, &energy);
  get_thermal(s);
  const double dti = 1.0 / std::sqrt(*dt * *max_dmdt);
  double ndt = 1e22;
  for (int l = 0; l < s->nl; ++l) {
    const Layer& Ly = s->L[l];
    double hmag = 0.0;
    for (int n = 0; n < Ly.N; ++n) {
      double v2 = 0.0;
      for (int a = 0; a < 3; ++a) {
        const double v = Ly.h[3 * n + a] + Ly.hthm[3 * n + a] * dti;
        v2 += v * v;
      }
      hmag = std::max(hmag, v2);
    }
    hmag = std::sqrt(hmag);
    const double fact1 = (1.0 + Ly.alpha * Ly.alpha) / ((1.0 + Ly.alpha) * Ly.gamma) * dt_frac;
    const double fact0 = fact1 != 0.0 ? 0.0 : 1.0;
    ndt = std::min(std::min(ndt, dt_max), fact1 / std::max(1.0, hmag) + fact0 * ndt);
  }
  *dt = ndt;
  double errmx = 0, errmx1 = 0, mmag = 0, e1l[8] = {0}, next = 1e22;
  while (true) {
    push_passes(s, *dt * *max_dmdt, type, &errmx, &errmx1, &mmag, e1l, &energy);
    bool too_far = false;
    next = 1e22;
    for (int l = 0; l < s->nl; ++l) {
      const double r = std::acos(1.0 - 0.5 * e1l[l]) / max_dm[l];
      if (r > 1.0) {
        *max_dmdt = 0.9 * *max_dmdt / r;
        too_far = true;
        break;
      }
      next = std::min(next, r < 2.0 / 3.0 ? std::min(2.0, *max_dmdt / (r + 1e-200)) : *max_dmdt);
    }
    if (!too_far) break;
  }
  if (next > 1e20) next = *max_dmdt;
  s->in = 1 - s->in;
  *dt = *dt * *max_dmdt;
  *max_dmdt = next;
  s->t += *dt;
  s->step += 1;
  compute_stats(s, errmx, errmx1, mmag, energy, e1l);
}

}  // namespace orc

// ===========================================================================
// C ABI for ctypes (tests / bench cpu leg only)
// ===========================================================================
using namespace orc;

extern "C" {

void orc_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

int orc_get_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

// ---- RNG probes ----
void orc_mt_u32(int seed, int n, uint32_t* out) {
  MT s;
  mt_create(&s, seed);
  for (int i = 0; i < n; ++i) out[i] = mt_next_u32(&s);
}
void orc_mt_state(int seed, uint32_t* out624) {
  MT s;
  mt_create(&s, seed);
  std::memcpy(out624, s.mt, sizeof(s.mt));
}
void orc_mt_normals(int seed, int n, double* out) {
  MT s;
  mt_create(&s, seed);
  for (int i = 0; i < n; ++i) out[i] = mt_normal(&s);
}
void orc_philox4x64(const uint64_t* ctr, const uint64_t* key, uint64_t* out) {
  philox4x64(ctr, key, out);
}
void orc_philox_normal3(uint64_t seed, uint64_t stream, uint64_t step, uint64_t grain, double* out) {
  philox_normal3(seed, stream, step, grain, out);
}

// ---- tensor ----
void orc_volume_averaged_n(double rx, double ry, double rz, double xs, double ys, double zs,
                           double xo, double yo, double zo, double* n9) {
  volume_averaged_n(rx, ry, rz, xs, ys, zs, xo, yo, zo, n9);
}
// volume_averaged_n in quadruple precision at offsets (ix dx, iy dy, rz),
// summed over `count` offsets (ix[k], iy[k]) and scaled by `scale`, rounded to
// FP64: one FFT-grid slot of the tensor (several offsets where the grid wraps)
void orc_volume_averaged_n_q(int count, const int* ix, const int* iy, double dx, double dy, double rz,
                             double xs, double ys, double zs, double xo, double zo, double scale, double* n9) {
  q128 n[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int k = 0; k < count; ++k) volume_averaged_n_q(ix[k], iy[k], dx, dy, rz, xs, ys, zs, xo, zo, n);
  for (int k = 0; k < 9; ++k) n9[k] = (double)(n[k] * (q128)scale);
}
void orc_calculate_tensor(int nx, int ny, int nl, double dx, double dy, const double* dz,
                          const double* il_space, int imx, int imy, double space_to_sul,
                          double sul_mu, double head_mu, double fly_height, double* n2d) {
  calculate_tensor(nx, ny, nl, dx, dy, dz, il_space, imx, imy, space_to_sul, sul_mu, head_mu,
                   fly_height, n2d);
}

// ---- FFT probes (row-major [ny][nx] real, [ny][nx/2+1] complex interleaved) ----
void orc_fft_r2c(int nx, int ny, const double* r, double* c) {
  FFT2<double> f;
  f.init(nx, ny);
  f.r2c(r, reinterpret_cast<cd*>(c));
}
void orc_fft_c2r(int nx, int ny, const double* c_in, double* r) {
  FFT2<double> f;
  f.init(nx, ny);
  std::vector<cd> c(reinterpret_cast<const cd*>(c_in),
                    reinterpret_cast<const cd*>(c_in) + (size_t)ny * (nx / 2 + 1));
  f.c2r(c.data(), r);
}

// Direct FP64 circular convolution with the real-space tensor n2d (reference layout):
// H_a(o) = P * sum_s sum_b n2d[ks][ko][3a+b][(o-s) mod P] M_b(s), for a list of
// observation cells `obs` (pairs i,j) on layer ko.  M grids [nl][3][py][px].
void orc_demag_direct(int px, int py, int nl, const double* n2d, const double* mgrid, int nobs,
                      const int* obs_ij, int ko, double* hout) {
  const size_t plane = (size_t)px * py;
  const double P = (double)px * py;
#pragma omp parallel for schedule(static)
  for (int q = 0; q < nobs; ++q) {
    int oi = obs_ij[2 * q], oj = obs_ij[2 * q + 1];
    double h[3] = {0, 0, 0};
    for (int ks = 0; ks < nl; ++ks) {
      const double* N = n2d + ((size_t)ks * nl + ko) * 9 * plane;
      for (int sj = 0; sj < py; ++sj) {
        int dj = ((oj - sj) % py + py) % py;
        for (int si = 0; si < px; ++si) {
          size_t sc = (size_t)sj * px + si;
          double m0 = mgrid[((size_t)ks * 3 + 0) * plane + sc];
          double m1 = mgrid[((size_t)ks * 3 + 1) * plane + sc];
          double m2 = mgrid[((size_t)ks * 3 + 2) * plane + sc];
          if (m0 == 0.0 && m1 == 0.0 && m2 == 0.0) continue;
          int di = ((oi - si) % px + px) % px;
          size_t off = (size_t)dj * px + di;
          for (int a = 0; a < 3; ++a)
            h[a] += N[(3 * a + 0) * plane + off] * m0 + N[(3 * a + 1) * plane + off] * m1 +
                    N[(3 * a + 2) * plane + off] * m2;
        }
      }
    }
    for (int a = 0; a < 3; ++a) hout[3 * q + a] = h[a] * P;
  }
}

// ---- simulation handle ----
void* orc_create(int nx, int ny, int nl, int boundary, int images, double dx, double dy,
                 const double* dz, const double* il_space, double space_to_sul, double sul_mu,
                 double head_mu, double fly_height, int demag_on) {
  Sim* s = new Sim();
  s->nx = nx; s->ny = ny; s->nl = nl;
  s->boundary = boundary; s->images = images;
  s->dx = dx; s->dy = dy;
  s->dz.assign(dz, dz + nl);
  s->il_space.assign(il_space, il_space + nl);
  s->space_to_sul = space_to_sul; s->sul_mu = sul_mu; s->head_mu = head_mu;
  s->fly_height = fly_height;
  s->px = boundary == 1 ? 2 * nx : nx;
  s->py = boundary == 1 ? 2 * ny : ny;
  s->ph = s->px / 2 + 1;
  s->fft.init(s->px, s->py);
  s->fft32.init(s->px, s->py);
  s->demag_on = demag_on != 0;
  s->L.resize(nl);
  return s;
}

void orc_destroy(void* h) { delete static_cast<Sim*>(h); }

// FFT precision of the demag convolution: 64 (the FFTD=1 build) or 32 (the
// default single-precision FFTW build); the spectrum is re-formed from the
// real tensor if one is set
int orc_set_fft_precision(void* h, int bits) {
  Sim* s = static_cast<Sim*>(h);
  if (bits != 32 && bits != 64) return 1;
  s->fft_bits = bits;
  if (!s->n2d_real.empty()) {
    const std::vector<double> t = s->n2d_real;
    build_spectrum(s, t.data());
  }
  return 0;
}

// {window nx, ny, origin i0, j0} (the whole grid and 0, 0 without a window)
void orc_get_window(void* h, int* out4) {
  Sim* s = static_cast<Sim*>(h);
  out4[0] = s->wnx ? s->wnx : s->nx;
  out4[1] = s->wnx ? s->wny : s->ny;
  out4[2] = s->wi0;
  out4[3] = s->wj0;
}

// moving demag window (mrm_gpu_set_window's arguments): the FFT grid becomes
// the window's; the tensor must be built or set again
int orc_set_window(void* h, int nxw, int nyw, double vx, double vy, double ox, double oy) {
  Sim* s = static_cast<Sim*>(h);
  if (nxw < 2 || nyw < 2 || nxw > s->nx || nyw > s->ny) return 1;
  const bool none = nxw == s->nx && nyw == s->ny;
  s->wnx = none ? 0 : nxw;
  s->wny = none ? 0 : nyw;
  s->wvx = vx; s->wvy = vy; s->wox = ox; s->woy = oy;
  s->wi0 = s->wj0 = 0;
  const int fx = none ? s->nx : nxw, fy = none ? s->ny : nyw;
  s->px = s->boundary == 1 ? 2 * fx : fx;
  s->py = s->boundary == 1 ? 2 * fy : fy;
  s->ph = s->px / 2 + 1;
  s->fft.init(s->px, s->py);
  s->fft32.init(s->px, s->py);
  s->nhat.clear();
  s->nhat32.clear();
  s->n2d_real.clear();
  return 0;
}

// Real-space tensor of the FFT grid (reference layout, with normalisation), FP64.
// Periodic: calculate_tensor on (nx,ny) with the handle's images; open: on the
// padded grid (2nx,2ny) with no images.
void orc_build_tensor(void* h, double* n2d_out) {
  Sim* s = static_cast<Sim*>(h);
  int im = s->boundary == 1 ? 0 : s->images;
  std::vector<double> n2d((size_t)s->px * s->py * 9 * s->nl * s->nl);
  calculate_tensor(s->px, s->py, s->nl, s->dx, s->dy, s->dz.data(), s->il_space.data(), im, im,
                   s->space_to_sul, s->sul_mu, s->head_mu, s->fly_height, n2d.data());
  build_spectrum(s, n2d.data());
  if (n2d_out) std::memcpy(n2d_out, n2d.data(), n2d.size() * sizeof(double));
}

void orc_set_tensor(void* h, const double* n2d) {
  Sim* s = static_cast<Sim*>(h);
  build_spectrum(s, n2d);
}

int orc_upload_layer(void* h, int l, int N, const double* ms, const double* vol,
                     const double* axis, const double* hk, const double* hk_scale,
                     const double* ms_scale, const double* alpha_scale, double alpha, double gamma,
                     double floor_ms, const int* g2c_index, const int* g2c /* 2 per cell, 1-based */,
                     const int* hx_index, const int* hx_grain /*1-based*/, const double* hx) {
  Sim* s = static_cast<Sim*>(h);
  if (l < 0 || l >= s->nl) return 1;
  Layer& Ly = s->L[l];
  Ly.N = N;
  Ly.ms.assign(ms, ms + N);
  Ly.vol.assign(vol, vol + N);
  Ly.axis.assign(axis, axis + 3 * N);
  Ly.hk.assign(hk, hk + 2 * N);
  Ly.hk_scale.assign(hk_scale, hk_scale + N);
  Ly.ms_scale.assign(ms_scale, ms_scale + N);
  Ly.alpha_scale.assign(alpha_scale, alpha_scale + N);
  Ly.alpha = alpha; Ly.gamma = gamma; Ly.floor_ms = floor_ms;
  Ly.g2c_idx.assign(g2c_index, g2c_index + N + 1);
  int nc = g2c_index[N];
  Ly.g2c_i.resize(nc);
  Ly.g2c_j.resize(nc);
  for (int q = 0; q < nc; ++q) {
    Ly.g2c_i[q] = g2c[2 * q] - 1;
    Ly.g2c_j[q] = g2c[2 * q + 1] - 1;
  }
  if (hx_index) {
    Ly.hx_idx.assign(hx_index, hx_index + N + 1);
    int nnz = hx_index[N];
    Ly.hx_nbr.resize(nnz);
    for (int q = 0; q < nnz; ++q) Ly.hx_nbr[q] = hx_grain[q] - 1;
    Ly.hx.assign(hx, hx + nnz);
  } else {
    Ly.hx_idx.clear(); Ly.hx_nbr.clear(); Ly.hx.clear();
  }
  for (int b = 0; b < 2; ++b) Ly.m[b].assign(3 * N, 0.0);
  Ly.dm.assign(3 * N, 0.0);
  Ly.h.assign(3 * N, 0.0);
  Ly.hthm.assign(3 * N, 0.0);
  Ly.hdemag.assign(3 * N, 0.0);
  Ly.happ.assign(3 * N, 0.0);
  Ly.c2g.assign((size_t)s->nx * s->ny, -1);
  for (int n = 0; n < N; ++n)
    for (int q = Ly.g2c_idx[n]; q < Ly.g2c_idx[n + 1]; ++q) Ly.c2g[(size_t)Ly.g2c_j[q] * s->nx + Ly.g2c_i[q]] = n;
  Ly.do_grain.assign(N, 1);
  Ly.min_n = 0;
  Ly.max_n = N - 1;
  Ly.mag[0].assign(N, 1.0);
  Ly.mag[1].assign(N, 1.0);
  Ly.llb = false;
  return 0;
}

// side 0: upper (couples to layer l-1, uhx), side 1: lower (couples to layer l+1, lhx)
int orc_upload_interlayer(void* h, int l, int side, const int* index, const int* grain,
                          const double* coef) {
  Sim* s = static_cast<Sim*>(h);
  if (l < 0 || l >= s->nl) return 1;
  Layer& Ly = s->L[l];
  int N = Ly.N;
  std::vector<int>& idx = side == 0 ? Ly.uhx_idx : Ly.lhx_idx;
  std::vector<int>& nbr = side == 0 ? Ly.uhx_nbr : Ly.lhx_nbr;
  std::vector<double>& cf = side == 0 ? Ly.uhx : Ly.lhx;
  idx.assign(index, index + N + 1);
  int nnz = index[N];
  nbr.resize(nnz);
  for (int q = 0; q < nnz; ++q) nbr[q] = grain[q] - 1;
  cf.assign(coef, coef + nnz);
  return 0;
}

int orc_set_uniform_field(void* h, int l, const double* dir, double t_start, double t_end,
                          double s_start, double s_end, double scale) {
  Sim* s = static_cast<Sim*>(h);
  if (l < 0 || l >= s->nl) return 1;
  Layer& Ly = s->L[l];
  for (int a = 0; a < 3; ++a) Ly.hdir[a] = dir[a];
  Ly.t_start = t_start; Ly.t_end = t_end; Ly.s_start = s_start; Ly.s_end = s_end; Ly.scale = scale;
  // set_fld :309-312 folds a constant scale
  if (Ly.s_start == Ly.s_end) {
    Ly.scale *= Ly.s_start;
    Ly.s_start = 1.0; Ly.s_end = 1.0;
  }
  return 0;
}

// uniform field with a time function: scale(t) = (amp*funct(t)+dc)*scale (applied.f90:867-869)
int orc_set_field_function(void* h, int l, const double* dir, int func, double amp, double g,
                           double phase, double param, double duty, double moddepth, double dc,
                           double scale) {
  Sim* s = static_cast<Sim*>(h);
  if (l < 0 || l >= s->nl) return 1;
  Layer& Ly = s->L[l];
  for (int a = 0; a < 3; ++a) Ly.hdir[a] = dir[a];
  Ly.func = func; Ly.amp = amp; Ly.fgamma = g; Ly.phase = phase; Ly.param = param;
  Ly.duty = std::max(0.0, std::min(1.0, duty)); Ly.moddepth = std::max(0.0, std::min(1.0, moddepth));
  Ly.dc = dc; Ly.scale = scale;
  return 0;
}

// cubic axes of layer l (NULL: back to uniaxial); layout of Layer::cax
int orc_set_cubic_axes(void* h, int l, const double* cax) {
  Sim* s = static_cast<Sim*>(h);
  if (l < 0 || l >= s->nl) return 1;
  Layer& Ly = s->L[l];
  if (!cax) Ly.cax.clear();
  else Ly.cax.assign(cax, cax + 9 * (size_t)Ly.N);
  return 0;
}

int orc_set_head_field(void* h, int l, double gap, double z, double hg, double v, double x0, double t0,
                       double tbit, uint64_t bits, int nbits) {
  Sim* s = static_cast<Sim*>(h);
  if (l < 0 || l >= s->nl || !(gap > 0 && z > 0 && tbit > 0) || nbits < 1 || nbits > 64) return 1;
  Layer& Ly = s->L[l];
  Ly.head = true;
  Ly.tab = false;
  Ly.hd_gap = gap; Ly.hd_z = z; Ly.hd_hg = hg; Ly.hd_v = v; Ly.hd_x0 = x0; Ly.hd_t0 = t0;
  Ly.hd_tbit = tbit; Ly.hd_bits = bits; Ly.hd_nbits = nbits;
  return 0;
}

// tabulated field profile (mrm_gpu_set_field_table's arguments; nfx = nfy = 0 removes it)
int orc_set_field_table(void* h, int l, int nfx, int nfy, const double* xpos, const double* ypos,
                        const double* vfld, double vx, double vy, double ox, double oy, double rx, double ry,
                        double t0) {
  Sim* s = static_cast<Sim*>(h);
  if (l < 0 || l >= s->nl) return 1;
  Layer& Ly = s->L[l];
  Ly.tab = false;
  if (nfx == 0 && nfy == 0) return 0;
  if (nfx < 2 || nfy < 2) return 1;
  Ly.head = false;
  Ly.tnx = nfx;
  Ly.tny = nfy;
  Ly.tab_x.assign(xpos, xpos + nfx);
  Ly.tab_y.assign(ypos, ypos + nfy);
  Ly.tab_v.assign(vfld, vfld + 3 * (size_t)nfx * nfy);
  Ly.tox = ox < -1e200 ? s->dx * s->nx * 0.5 : ox;  // applied.f90:804-805
  Ly.toy = oy < -1e200 ? s->dy * s->ny * 0.5 : oy;
  Ly.tvx = vx; Ly.tvy = vy; Ly.trx = rx; Ly.try_ = ry; Ly.tt0 = t0;
  Ly.tab = true;
  return 0;
}

// rng_mode 0: MT19937 per layer seeded like input.f90:190-206 / field.f90:712-733;
// rng_mode 1: Philox stream (seed) shared with the GPU path.
int orc_set_thermal(void* h, int l, int on, double temperature, int rng_mode, long long seed) {
  Sim* s = static_cast<Sim*>(h);
  if (l < 0 || l >= s->nl) return 1;
  Layer& Ly = s->L[l];
  Ly.thermal = on != 0;
  Ly.temperature = temperature;
  s->rng_mode = rng_mode;
  if (rng_mode == 0) mt_create(&Ly.rng, (int)seed);
  else s->seed = (uint64_t)seed;
  return 0;
}

int orc_set_state(void* h, int l, const double* m) {
  Sim* s = static_cast<Sim*>(h);
  if (l < 0 || l >= s->nl) return 1;
  Layer& Ly = s->L[l];
  std::memcpy(Ly.m[s->in].data(), m, sizeof(double) * 3 * Ly.N);
  std::memcpy(Ly.m[1 - s->in].data(), m, sizeof(double) * 3 * Ly.N);
  Ly.mag[0].assign(Ly.N, 1.0);  // a new state starts at |m| = 1 (data.f90:202)
  Ly.mag[1].assign(Ly.N, 1.0);
  return 0;
}

// grain temperatures of the last field evaluation (field(k)%temp)
int orc_get_temp(void* h, int l, double* out) {
  Sim* s = static_cast<Sim*>(h);
  if (l < 0 || l >= s->nl || (int)s->L[l].temp.size() != s->L[l].N) return 1;
  std::memcpy(out, s->L[l].temp.data(), sizeof(double) * s->L[l].N);
  return 0;
}

// temperature profile (mrm_gpu_set_temp_profile's arguments; expn < 0: off)
int orc_set_temp_profile(void* h, int l, double bg, double dtemp, double sx, double sy, int expn, double vx,
                         double vy, double ox, double oy, double rx, double ry, double t0) {
  Sim* s = static_cast<Sim*>(h);
  if (l < 0 || l >= s->nl) return 1;
  Layer& Ly = s->L[l];
  if (expn < 0) {
    Ly.tprof = false;
    return 0;
  }
  if (!Ly.tprof) {
    Ly.tp_func = 0; Ly.tp_t_start = -1e22; Ly.tp_t_end = 1e22; Ly.tp_s_start = Ly.tp_s_end = 1.0; Ly.tp_scale = 1.0;
  }
  Ly.tprof = true;
  Ly.tp_bg = bg; Ly.tp_dtemp = dtemp;
  Ly.tp_isx = sx != 0.0 ? 1.0 / sx : 0.0;  // applied.f90:476-477
  Ly.tp_isy = sy != 0.0 ? 1.0 / sy : 0.0;
  Ly.tp_expn = 2 * expn;
  Ly.tp_vx = vx; Ly.tp_vy = vy;
  Ly.tp_ox = ox < -1e200 ? s->dx * s->nx * 0.5 : ox;
  Ly.tp_oy = oy < -1e200 ? s->dy * s->ny * 0.5 : oy;
  Ly.tp_rx = rx; Ly.tp_ry = ry; Ly.tp_t0 = t0;
  return 0;
}

int orc_set_temp_function(void* h, int l, int func, double t_start, double t_end, double s_start, double s_end,
                          double amp, double g, double phase, double param, double duty, double moddepth, double dc,
                          double scale) {
  Sim* s = static_cast<Sim*>(h);
  if (l < 0 || l >= s->nl || !s->L[l].tprof) return 1;
  Layer& Ly = s->L[l];
  Ly.tp_func = func; Ly.tp_t_start = t_start; Ly.tp_t_end = t_end; Ly.tp_s_start = s_start; Ly.tp_s_end = s_end;
  Ly.tp_amp = amp; Ly.tp_fgamma = g; Ly.tp_phase = phase; Ly.tp_param = param;
  Ly.tp_duty = std::max(0.0, std::min(1.0, duty)); Ly.tp_moddepth = std::max(0.0, std::min(1.0, moddepth));
  Ly.tp_dc = dc; Ly.tp_scale = scale;
  return 0;
}

// MT (mode 1) or Zhang (mode 2) on layer l (mrm_gpu_set_mt's arguments; lam_ms NULL: off)
int orc_set_mt(void* h, int l, double spin, const double* lam_ms, int meq_bs, int garanin_tau, int mode) {
  Sim* s = static_cast<Sim*>(h);
  if (l < 0 || l >= s->nl) return 1;
  Layer& Ly = s->L[l];
  Ly.llb = lam_ms != nullptr;
  Ly.mode = mode;
  if (!lam_ms) return 0;
  Ly.spin = spin;
  Ly.meq_bs = meq_bs;
  Ly.garanin_tau = garanin_tau;
  Ly.tc.assign(Ly.N, 0.0);
  Ly.lam_ms.assign(lam_ms, lam_ms + Ly.N);
  return 0;
}

// LLB on layer l (mrm_gpu_set_llb's arguments; tc NULL: off)
// set_temp_scaling (temp_scaling.f90:37-50) with the grains' Tc: msexp / hkexp
// < 0 leave those power laws off; tc null switches the scaling off
int orc_set_temp_scaling(void* h, int l, const double* tc, double msexp, double hkexp, int use_mag) {
  Sim* s = static_cast<Sim*>(h);
  if (l < 0 || l >= s->nl) return 1;
  Layer& Ly = s->L[l];
  Ly.tsc = tc != nullptr;
  if (!tc) return 0;
  Ly.tsc_tc.assign(tc, tc + Ly.N);
  Ly.tsc_msexp = msexp;
  Ly.tsc_hkexp = hkexp;
  Ly.tsc_mag = use_mag != 0;
  return 0;
}

// file_temp_scaling's table which (1 Ms, 2 alpha, 3 Hk, 4 Hx) as read; n = 0 removes it
int orc_set_temp_scaling_table(void* h, int l, int which, int n, const double* temp, const double* scaling) {
  Sim* s = static_cast<Sim*>(h);
  if (l < 0 || l >= s->nl || which < 1 || which > 4 || n < 0) return 1;
  Layer& Ly = s->L[l];
  if (n == 0) {
    Ly.tsc_t[which - 1].clear();
    Ly.tsc_v[which - 1].clear();
    return 0;
  }
  reduce_scaling_table(n, temp, scaling, Ly.tsc_t[which - 1], Ly.tsc_v[which - 1]);
  return 0;
}

// the reduced table (for tests): *n on input the room, on output the nodes
int orc_get_temp_scaling_table(void* h, int l, int which, int* n, double* temp, double* scaling) {
  Sim* s = static_cast<Sim*>(h);
  if (l < 0 || l >= s->nl || which < 1 || which > 4) return 1;
  const Layer& Ly = s->L[l];
  const int m = (int)Ly.tsc_t[which - 1].size();
  if (*n < m) return 2;
  for (int i = 0; i < m; ++i) {
    temp[i] = Ly.tsc_t[which - 1][i];
    scaling[i] = Ly.tsc_v[which - 1][i];
  }
  *n = m;
  return 0;
}

// the layer's scales after the last field evaluation (for tests): ms, alpha, hk per grain
int orc_get_scales(void* h, int l, double* ms_scale, double* alpha_scale, double* hk_scale) {
  Sim* s = static_cast<Sim*>(h);
  if (l < 0 || l >= s->nl) return 1;
  const Layer& Ly = s->L[l];
  std::copy(Ly.ms_scale.begin(), Ly.ms_scale.end(), ms_scale);
  std::copy(Ly.alpha_scale.begin(), Ly.alpha_scale.end(), alpha_scale);
  std::copy(Ly.hk_scale.begin(), Ly.hk_scale.end(), hk_scale);
  return 0;
}

int orc_set_llb(void* h, int l, double spin, const double* tc, const double* lam_ms) {
  Sim* s = static_cast<Sim*>(h);
  if (l < 0 || l >= s->nl) return 1;
  Layer& Ly = s->L[l];
  Ly.llb = tc != nullptr;
  Ly.mode = 0;
  if (!tc) return 0;
  Ly.spin = spin;
  Ly.tc.assign(tc, tc + Ly.N);
  Ly.lam_ms.assign(lam_ms, lam_ms + Ly.N);
  return 0;
}

int orc_set_mag(void* h, int l, const double* mag) {
  Sim* s = static_cast<Sim*>(h);
  if (l < 0 || l >= s->nl) return 1;
  Layer& Ly = s->L[l];
  Ly.mag[s->in].assign(mag, mag + Ly.N);
  Ly.mag[1 - s->in].assign(mag, mag + Ly.N);
  return 0;
}

int orc_get_mag(void* h, int l, double* mag) {
  Sim* s = static_cast<Sim*>(h);
  if (l < 0 || l >= s->nl) return 1;
  std::memcpy(mag, s->L[l].mag[s->in].data(), sizeof(double) * s->L[l].N);
  return 0;
}

int orc_get_state(void* h, int l, double* m) {
  Sim* s = static_cast<Sim*>(h);
  if (l < 0 || l >= s->nl) return 1;
  std::memcpy(m, s->L[l].m[s->in].data(), sizeof(double) * 3 * s->L[l].N);
  return 0;
}

int orc_get_field(void* h, int l, double* out) {
  Sim* s = static_cast<Sim*>(h);
  if (l < 0 || l >= s->nl) return 1;
  std::memcpy(out, s->L[l].h.data(), sizeof(double) * 3 * s->L[l].N);
  return 0;
}

int orc_get_demag(void* h, int l, double* out) {
  Sim* s = static_cast<Sim*>(h);
  if (l < 0 || l >= s->nl) return 1;
  std::memcpy(out, s->L[l].hdemag.data(), sizeof(double) * 3 * s->L[l].N);
  return 0;
}

// applied field per grain of the last field evaluation (field(k)%h_app)
int orc_get_applied(void* h, int l, double* out) {
  Sim* s = static_cast<Sim*>(h);
  if (l < 0 || l >= s->nl) return 1;
  std::memcpy(out, s->L[l].happ.data(), sizeof(double) * 3 * s->L[l].N);
  return 0;
}

void orc_set_time(void* h, double t, long long step) {
  Sim* s = static_cast<Sim*>(h);
  s->t = t;
  s->step = step;
}

// evaluate the (non-thermal) field of the current state at time t (get_field)
void orc_eval_field(void* h, double t) {
  Sim* s = static_cast<Sim*>(h);
  double e;
  update_do_grain(s, t);
  get_field(s, t, s->in, &e);
}

// nsteps fixed-dt steps of llg type (-3 Heun, 2 Boris, -2 Boris midpoint).
// stats_out: mirrors mrm_gpu_stats (see include/mrm_gpu.h) for the last step.
// traj: optional [nsteps][nl][3] vol-weighted <m> after each step.
int orc_step(void* h, int nsteps, double dt, int type, double* stats_out, double* traj) {
  Sim* s = static_cast<Sim*>(h);
  if (!(type == -3 || type == 2 || type == -2 || type == 1 || type == -1)) return 2;
  for (const Layer& Ly : s->L)
    if (Ly.llb && std::abs(type) == 1) return 2;  // push_llb has no analytic rotation here
  update_do_grain(s, s->t);  // llg.f90:138
  for (int k = 0; k < nsteps; ++k) {
    heun_or_boris_step(s, dt, type);
    if (traj)
      for (int l = 0; l < s->nl; ++l)
        for (int a = 0; a < 3; ++a) traj[((size_t)k * s->nl + l) * 3 + a] = s->last.mave_l[l][a];
  }
  if (stats_out) std::memcpy(stats_out, &s->last, sizeof(Stats));
  return 0;
}

// nsteps adaptive steps (see adaptive_step); dt and max_dmdt carry llgp%dt and
// llgp%max_dmdt from call to call; max_dm per layer in radians.
int orc_step_adaptive(void* h, int nsteps, int type, double dt_frac, double dt_max, const double* max_dm, double* dt,
                      double* max_dmdt, double* stats_out) {
  Sim* s = static_cast<Sim*>(h);
  if (!(type == -3 || type == 2 || type == -2 || type == 1 || type == -1)) return 2;
  if (s->wnx) return 3;  // fixed dt only with a moving window
  for (int k = 0; k < nsteps; ++k) adaptive_step(s, type, dt_frac, dt_max, max_dm, dt, max_dmdt);
  if (stats_out) std::memcpy(stats_out, &s->last, sizeof(Stats));
  return 0;
}

// calculate_off_field_tensor (off_field.f90:216-320) and get_off_field
// (:55-108) on the nx x ny data grid: out[(c*ny + j)*nx + i] = H_c at the
// observation slab (bottom zoff above the top layer, thickness dzobs)
int orc_off_field(void* h, double zoff, double dzobs, double head_mu, double fly_height, double sul_mu,
                  double space_to_sul, int nimg, double* out) {
  Sim* s = static_cast<Sim*>(h);
  const int nx = s->nx, ny = s->ny, nl = s->nl;
  const size_t plane = (size_t)nx * ny, hplane = (size_t)(nx / 2 + 1) * ny;
  const bool sul_p = sul_mu > 1.0, head_p = head_mu > 1.0;  // off_field.f90:191,251-256
  const double mus = sul_p ? std::max(0.0, (std::max(1.0, sul_mu) - 1.0) / (std::max(1.0, sul_mu) + 1.0)) : 0.0;
  const double mush = head_p ? std::max(0.0, (std::max(1.0, head_mu) - 1.0) / (std::max(1.0, head_mu) + 1.0)) : 0.0;
  std::vector<double> hdz(nl);
  hdz[0] = fly_height;
  for (int k = 1; k < nl; ++k) hdz[k] = hdz[k - 1] + s->dz[k - 1] + s->il_space[k];
  for (int k = 0; k < nl; ++k) hdz[k] += 0.5 * s->dz[k];
  double zob = space_to_sul + zoff;
  for (int k = 0; k < nl; ++k) {
    zob += s->dz[k];
    if (k != nl - 1) zob += s->il_space[k];
  }
  const double zot = zob + dzobs;
  FFT2<double> f;
  f.init(nx, ny);
  std::vector<double> nn(9 * plane), t(9 * plane), grid(3 * plane);
  std::vector<cd> T(9 * hplane), X(3 * hplane), H(3 * hplane, cd(0, 0));
  double zsb = space_to_sul;
  for (int ks = nl - 1; ks >= 0; --ks) {
    const double zst = zsb + s->dz[ks];
    std::fill(t.begin(), t.end(), 0.0);
    auto add = [&](double rz, double fxy, double fz) {
      plane_to_plane(nx, ny, s->dx, s->dy, s->dz[ks], dzobs, rz, nimg, nimg, nn.data());
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b)
          for (size_t p = 0; p < plane; ++p)
            t[(3 * b + a) * plane + p] += (a < 2 ? fxy : fz) * nn[(a * 3 + b) * plane + p];
    };
    add(0.5 * (zst - zot + zsb - zob), 1.0, 1.0);
    if (sul_p) add(0.5 * (-zst - zot - zsb - zob), -mus, mus);
    if (head_p) add(hdz[ks] + fly_height - (zoff + 0.5 * dzobs), -mush, mush);
    const double norm = 1.0 / (s->dx * s->dy * dzobs * (double)nx * (double)ny);
    for (auto& v : t) v *= norm;
    // get_mag of layer ks on the data grid
    std::fill(grid.begin(), grid.end(), 0.0);
    const Layer& Ly = s->L[ks];
    const double* m = Ly.m[s->in].data();
    for (int n = 0; n < Ly.N; ++n) {
      const double fm = Ly.ms[n] * Ly.ms_scale[n];
      for (int q = Ly.g2c_idx[n]; q < Ly.g2c_idx[n + 1]; ++q) {
        const size_t cell = (size_t)Ly.g2c_j[q] * nx + Ly.g2c_i[q];
        for (int a = 0; a < 3; ++a) grid[a * plane + cell] = fm * m[3 * n + a];
      }
    }
    for (int c = 0; c < 9; ++c) f.r2c(&t[c * plane], &T[c * hplane]);
    for (int b = 0; b < 3; ++b) f.r2c(&grid[b * plane], &X[b * hplane]);
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b)
        for (size_t q = 0; q < hplane; ++q) H[a * hplane + q] += T[(3 * a + b) * hplane + q] * X[b * hplane + q];
    zsb = zst + s->il_space[ks];
  }
  for (int a = 0; a < 3; ++a) f.c2r(&H[a * hplane], out + a * plane);
  return 0;
}

int orc_stats_size(void) { return (int)sizeof(Stats); }

}  // extern "C"
