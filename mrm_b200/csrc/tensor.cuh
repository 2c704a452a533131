// tensor.cuh -- FP64 magnetostatic tensor and its spectrum, once per run.
//
// Device restatement of volume_averaged_n / plane_to_plane
// (src/tensor_element.f90:13-102, :219-261) and calculate_tensor
// (src/tensor.f90:82-216): one thread per FFT-grid slot sums, in the
// reference's order, every in-plane offset that wraps onto that slot and all
// its periodic images.  The FP64 real tensor is then transformed in FP64
// (demag.f90:259-267 does this once per run) and packed: each of the 9
// components of a layer pair has a purely real (xx, yy, zz, xy, yx) or purely
// imaginary (xz, zx, yz, zy) spectrum, even or odd in ky, so one real number
// per (kx, 0 <= ky <= py/2) is kept.
#pragma once
#include "common.cuh"
#include "fft.cuh"

namespace mrm {

struct PairGeom {
  double dz_s, dz_o;  // source / observation layer thickness
  double rz;          // centre-to-centre z offset, source - observation
  double rz_sul, f_sul;    // SUL image term (f_sul = 0: none), tensor.f90:162-171
  double rz_head, f_head;  // head image term, tensor.f90:172-181
  double norm;        // 1/(dx dy dz_o px py), tensor.f90:183
};

__device__ __forceinline__ double fsign_d(double a, double b) { return copysign(fabs(a), b); }

__device__ __forceinline__ double tg1(double x, double y, double z, double d) {
  double r = x * y * z * atan(y * z / fsign_d(fmax(1.0e-300, fabs(x) * d), x));
  r += 0.5 * y * (z * z - x * x) * log(fmax(1.0e-300, d - y));
  r += 0.5 * z * (y * y - x * x) * log(fmax(1.0e-300, d - z));
  r += (y * y + z * z - 2.0 * x * x) * d / 6.0;
  return r;
}

__device__ __forceinline__ double tg2(double z, double x, double y, double d) {
  double r = -x * y * z * log(fmax(1.0e-300, d + z));
  r += y * (y * y - 3.0 * z * z) * log(fmax(1.0e-300, d + x)) / 6.0;
  r += x * (x * x - 3.0 * z * z) * log(fmax(1.0e-300, d + y)) / 6.0;
  r += 0.5 * x * x * z * atan(y * z / fsign_d(fmax(1.0e-300, fabs(x) * d), x));
  r += 0.5 * y * y * z * atan(x * z / fsign_d(fmax(1.0e-300, fabs(y) * d), y));
  r += z * z * z * atan(x * y / fsign_d(fmax(1.0e-300, fabs(z) * d), z)) / 6.0;
  r += x * y * d / 3.0;
  return r;
}

// n -= t over the 64 corner combinations; n[a*3+b] = reference n(a,b)
__device__ void vol_avg_n(double rx, double ry, double rz, double xs, double ys, double zs,
                          double xo, double zo, double* n) {
  const double dxo[2] = {-0.5 * xo, 0.5 * xo}, dyo[2] = {-0.5 * xo, 0.5 * xo},
               dzo[2] = {-0.5 * zo, 0.5 * zo};
  const double dxs[2] = {-0.5 * xs, 0.5 * xs}, dys[2] = {-0.5 * ys, 0.5 * ys},
               dzs[2] = {-0.5 * zs, 0.5 * zs};
  double t[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int i6 = 1; i6 <= 2; ++i6)
    for (int i5 = 1; i5 <= 2; ++i5)
      for (int i4 = 1; i4 <= 2; ++i4)
        for (int i3 = 1; i3 <= 2; ++i3) {
          const double dx = -rx + dxo[i3 - 1] - dxs[i6 - 1];
          for (int i2 = 1; i2 <= 2; ++i2) {
            const double dy = -ry + dyo[i2 - 1] - dys[i5 - 1];
            for (int i1 = 1; i1 <= 2; ++i1) {
              const double dz = -rz + dzo[i1 - 1] - dzs[i4 - 1];
              const double d = sqrt(dx * dx + dy * dy + dz * dz);
              if (d != 0.0) {
                const double sg = ((i1 + i2 + i3 + i4 + i5 + i6 - 1) & 1) ? -1.0 : 1.0;
                t[0] += sg * tg1(dx, dy, dz, d);
                t[4] += sg * tg1(dy, dz, dx, d);
                t[8] += sg * tg1(dz, dx, dy, d);
                double x = sg * tg2(dx, dy, dz, d);
                t[7] += x;
                t[5] += x;
                x = sg * tg2(dy, dz, dx, d);
                t[6] += x;
                t[2] += x;
                x = sg * tg2(dz, dx, dy, d);
                t[3] += x;
                t[1] += x;
              }
            }
          }
        }
  for (int k = 0; k < 9; ++k) n[k] -= t[k];
}

// offsets i in [-n/2, n/2] with (n - i) mod n == f, ascending
__device__ __forceinline__ int slot_offsets(int f, int n, int* out) {
  if ((n & 1) == 0 && f == n / 2) {
    out[0] = -n / 2;
    out[1] = n / 2;
    return 2;
  }
  out[0] = (f == 0) ? 0 : (f <= n / 2 ? -f : n - f);
  return 1;
}

// plane_to_plane for one slot (tensor_element.f90:233-257); acc[a*3+b]
__device__ void slot_plane(int fi, int fj, int nx, int ny, double dx, double dy, double dz,
                           double dzo, double rz, int nimg, double* acc) {
  int il[2], jl[2];
  const int ni = slot_offsets(fi, nx, il), nj = slot_offsets(fj, ny, jl);
  for (int k = 0; k < 9; ++k) acc[k] = 0.0;
  for (int qj = 0; qj < nj; ++qj) {
    const int j = jl[qj];
    const int yp0 = -nimg * (1 - max(0, j / ((ny + 1) / 2)));
    const int yp1 = nimg * (1 + min(0, j / ((ny + 1) / 2)));
    for (int qi = 0; qi < ni; ++qi) {
      const int i = il[qi];
      const int xp0 = -nimg * (1 - max(0, i / ((nx + 1) / 2)));
      const int xp1 = nimg * (1 + min(0, i / ((nx + 1) / 2)));
      double t[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
      for (int iy = yp0; iy <= yp1; ++iy)
        for (int ix = xp0; ix <= xp1; ++ix) {
          const double rx = (double)i * dx + (double)ix * dx * (double)nx;
          const double ry = (double)j * dy + (double)iy * dy * (double)ny;
          vol_avg_n(rx, ry, rz, dx, dy, dz, dx, dzo, t);
        }
      for (int k = 0; k < 9; ++k) acc[k] += t[k];
    }
  }
}

// n2d[((pair*9 + c)*py + fj)*px + fi], c = 3*b + a holds t(a,b) (Fortran n2d layout)
__global__ void tensor_real_kernel(double* __restrict__ n2d, const PairGeom* __restrict__ pg,
                                   int npair, int px, int py, double dx, double dy, int nimg) {
  const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long plane = (long long)px * py;
  if (gid >= plane * npair) return;
  const int pair = (int)(gid / plane);
  const int rem = (int)(gid - (long long)pair * plane);
  const int fj = rem / px, fi = rem - fj * px;
  const PairGeom g = pg[pair];
  double acc[9], tot[9];
  slot_plane(fi, fj, px, py, dx, dy, g.dz_s, g.dz_o, g.rz, nimg, acc);
  for (int k = 0; k < 9; ++k) tot[k] = acc[k];
  if (g.f_sul != 0.0) {
    slot_plane(fi, fj, px, py, dx, dy, g.dz_s, g.dz_o, g.rz_sul, nimg, acc);
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) tot[a * 3 + b] += (a < 2 ? -g.f_sul : g.f_sul) * acc[a * 3 + b];
  }
  if (g.f_head != 0.0) {
    slot_plane(fi, fj, px, py, dx, dy, g.dz_s, g.dz_o, g.rz_head, nimg, acc);
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) tot[a * 3 + b] += (a < 2 ? -g.f_head : g.f_head) * acc[a * 3 + b];
  }
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b)
      n2d[(((long long)pair * 9 + 3 * b + a) * py + fj) * px + fi] = tot[a * 3 + b] * g.norm;
}

// FP64 r2c along x of `planes` real planes [p][py][px] -> [p][py][px/2+1]
__global__ void __launch_bounds__(256) r2c_rows_f64(const double* __restrict__ in,
                                                    Cx<double>* __restrict__ out, int lgpx,
                                                    int py, const Cx<double>* __restrict__ tw) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lgM = lgpx - 1, M = 1 << lgM, ph = M + 1, px = 2 * M;
  const long long row = blockIdx.x;  // p*py + j
  const int cs = pad_stride(M);
  Cx<double>* A = reinterpret_cast<Cx<double>*>(smem_raw);
  Cx<double>* B = A + cs;
  const double* src = in + row * px;
  for (int k = threadIdx.x; k < M; k += blockDim.x) A[k] = Cx<double>{src[2 * k], src[2 * k + 1]};
  __syncthreads();
  Cx<double>* Y = block_fft<double, -1>(A, B, lgM, 1, cs, tw, kTwLog);
  for (int k = threadIdx.x; k < ph; k += blockDim.x) {
    const Cx<double> yk = Y[k & (M - 1)], ymk = cconj(Y[(M - k) & (M - 1)]);
    const Cx<double> e = cscale(cadd(yk, ymk), 0.5), o = cscale(csub(yk, ymk), 0.5);
    const Cx<double> wo = cmul(twiddle(tw, k & (px - 1), lgpx), o);
    out[row * ph + k] = csub(e, cmul_i(wo, 1.0));
  }
}

// FP64 complex FFT along y of [p][py][ph], in place; one block per (p, column)
__global__ void __launch_bounds__(256) c2c_cols_f64(Cx<double>* __restrict__ data, int lgpy, int ph,
                                                    const Cx<double>* __restrict__ tw) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int py = 1 << lgpy;
  const long long p = blockIdx.x / ph;
  const int k = blockIdx.x - (int)(p * ph);
  const int cs = pad_stride(py);
  Cx<double>* A = reinterpret_cast<Cx<double>*>(smem_raw);
  Cx<double>* B = A + cs;
  Cx<double>* base = data + p * (long long)py * ph + k;
  for (int j = threadIdx.x; j < py; j += blockDim.x) A[j] = base[(long long)j * ph];
  __syncthreads();
  Cx<double>* Y = block_fft<double, -1>(A, B, lgpy, 1, cs, tw, kTwLog);
  for (int j = threadIdx.x; j < py; j += blockDim.x) base[(long long)j * ph] = Y[j];
}

// inverse FP64 complex FFT along y of [p][py][ph], in place (unnormalised)
__global__ void __launch_bounds__(256) c2c_cols_f64_inv(Cx<double>* __restrict__ data, int lgpy, int ph,
                                                        const Cx<double>* __restrict__ tw) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int py = 1 << lgpy;
  const long long p = blockIdx.x / ph;
  const int k = blockIdx.x - (int)(p * ph);
  const int cs = pad_stride(py);
  Cx<double>* A = reinterpret_cast<Cx<double>*>(smem_raw);
  Cx<double>* B = A + cs;
  Cx<double>* base = data + p * (long long)py * ph + k;
  for (int j = threadIdx.x; j < py; j += blockDim.x) A[j] = base[(long long)j * ph];
  __syncthreads();
  Cx<double>* Y = block_fft<double, +1>(A, B, lgpy, 1, cs, tw, kTwLog);
  for (int j = threadIdx.x; j < py; j += blockDim.x) base[(long long)j * ph] = Y[j];
}

// FP64 c2r along x (FFTW's unnormalised c2r): rows [p][py][px/2+1] -> real
// [p][py][px] through the half-length complex transform (imaginary parts of
// the k = 0 and k = px/2 bins ignored)
__global__ void __launch_bounds__(256) c2r_rows_f64(const Cx<double>* __restrict__ in, double* __restrict__ out,
                                                    int lgpx, const Cx<double>* __restrict__ tw) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lgM = lgpx - 1, M = 1 << lgM, ph = M + 1, px = 2 * M;
  const long long row = blockIdx.x;  // p*py + j
  const int cs = pad_stride(M);
  Cx<double>* A = reinterpret_cast<Cx<double>*>(smem_raw);
  Cx<double>* B = A + cs;
  const Cx<double>* X = in + row * ph;
  for (int k = threadIdx.x; k < M; k += blockDim.x) {
    Cx<double> a = X[k], b = X[M - k];
    if (k == 0) {
      a.y = 0.0;
      b.y = 0.0;
    }
    const Cx<double> e = cadd(a, cconj(b)), o = csub(a, cconj(b));
    const Cx<double> w = cconj(twiddle(tw, k, lgpx));  // e^{+2 pi i k / px}
    A[k] = cadd(e, cmul_i(cmul(o, w), 1.0));
  }
  __syncthreads();
  Cx<double>* Z = block_fft<double, +1>(A, B, lgM, 1, cs, tw, kTwLog);
  double* dst = out + row * px;
  for (int n = threadIdx.x; n < M; n += blockDim.x) {
    dst[2 * n] = Z[n].x;
    dst[2 * n + 1] = Z[n].y;
  }
}

// block-wide max of two non-negative doubles, one atomicMax per block
__device__ __forceinline__ void block_max2(double a, double b, unsigned long long* ga,
                                           unsigned long long* gb) {
  __shared__ double sa[32], sb[32];
  for (int o = 16; o > 0; o >>= 1) {
    a = fmax(a, __shfl_xor_sync(0xffffffffu, a, o));
    b = fmax(b, __shfl_xor_sync(0xffffffffu, b, o));
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) { sa[warp] = a; sb[warp] = b; }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x + 31) / 32; ++w) { a = fmax(a, sa[w]); b = fmax(b, sb[w]); }
    atomicMax(ga, (unsigned long long)__double_as_longlong(a));
    atomicMax(gb, (unsigned long long)__double_as_longlong(b));
  }
}

// parity-violating part of one spectral value (and its ky mirror) and the kept part
__device__ __forceinline__ void parity_parts(const Cx<double>* S, int c, int kyh, int k, int py, int ph,
                                             double* keep, double* disc) {
  const Cx<double> v = S[(long long)kyh * ph + k];
  const bool imag = (kImagMask >> c) & 1;
  const bool odd = (kOddMask >> c) & 1;
  *keep = imag ? v.y : v.x;
  double d = imag ? fabs(v.x) : fabs(v.y);
  if (kyh > 0 && kyh < py - kyh) {
    const Cx<double> u = S[(long long)(py - kyh) * ph + k];
    const double um = imag ? u.y : u.x;
    d = fmax(d, fabs(um - (odd ? -*keep : *keep)));
  }
  *disc = d;
}

// spectrum [pair][9][py][ph] (FP64) -> tens[k][pair][c][kyh] (R, rows of pyhs
// reals): one real per component and 0 <= ky <= py/2 (FP32 runs); tracks the
// dropped residue.
template <typename R>
__global__ void pack_tensor_kernel(const Cx<double>* __restrict__ spec, R* __restrict__ tens,
                                   int npair, int py, int ph, int pyhs, unsigned long long* resid,
                                   unsigned long long* kept) {
  const int pyh = py / 2 + 1;
  const long long total = (long long)ph * npair * 9 * pyh;
  const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  double keep = 0.0, disc = 0.0;
  if (gid < total) {
    const int kyh = (int)(gid % pyh);
    long long r = gid / pyh;
    const int c = (int)(r % 9);
    r /= 9;
    const int pair = (int)(r % npair);
    const int k = (int)(r / npair);
    parity_parts(spec + ((long long)pair * 9 + c) * py * ph, c, kyh, k, py, ph, &keep, &disc);
    tens[(gid / pyh) * pyhs + kyh] = (R)keep;
  }
  block_max2(disc, fabs(keep), resid, kept);
}

// spectrum [pair][9][py][ph] -> tens[k][pair][c][ky] complex, unchanged (FP64 runs)
__global__ void pack_tensor_full_kernel(const Cx<double>* __restrict__ spec, Cx<double>* __restrict__ tens,
                                        int npair, int py, int ph, unsigned long long* resid,
                                        unsigned long long* kept) {
  const long long total = (long long)ph * npair * 9 * py;
  const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  double keep = 0.0, disc = 0.0;
  if (gid < total) {
    const int ky = (int)(gid % py);
    long long r = gid / py;
    const int c = (int)(r % 9);
    r /= 9;
    const int pair = (int)(r % npair);
    const int k = (int)(r / npair);
    const Cx<double>* S = spec + ((long long)pair * 9 + c) * py * ph;
    tens[gid] = S[(long long)ky * ph + k];
    if (ky <= py / 2) parity_parts(S, c, ky, k, py, ph, &keep, &disc);
  }
  block_max2(disc, fabs(keep), resid, kept);
}

}  // namespace mrm
