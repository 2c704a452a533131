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
#include "dd.cuh"
#include "fft.cuh"

namespace mrm {

struct PairGeom {
  double dz_s, dz_o;  // source / observation layer thickness
  double rz;          // centre-to-centre z offset, source - observation
  double rz_sul, f_sul;    // SUL image term (f_sul = 0: none), tensor.f90:162-171
  double rz_head, f_head;  // head image term, tensor.f90:172-181
  double norm;        // 1/(dx dy dz_o px py), tensor.f90:183
};

// One corner combination of volume_averaged_n (tensor_element.f90:39-72) in
// double-double: the corner offsets (x, y, z), d = |(x, y, z)|, the three
// arctangents and six logarithms that g1 and g2 (:78-100) share, and the
// six distinct elements.  g1(x,y,z,d) and g2(z,x,y,d) are the reference's
// closed forms with their max(1e-300, .) guards and Fortran sign(); the
// arctangent arguments y z / sign(max(1e-300, |x| d), x) and their
// permutations are A_x, A_y, A_z.
struct TensCorner {
  dd t00, t11, t22, t12, t02, t01;  // g1(x,y,z), g1(y,z,x), g1(z,x,y), g2(x,y,z), g2(y,z,x), g2(z,x,y)
};

__device__ __forceinline__ dd tens_den(dd v, dd d) {
  // sign(max(1e-300, |v| d), v)
  const dd a = dd_max_d(dd_mul(dd_abs(v), d), 1.0e-300);
  return signbit(v.hi) ? dd_neg(a) : a;
}
__device__ __forceinline__ dd tens_log(dd v) { return dd_log(dd_max_d(v, 1.0e-300)); }

__device__ __noinline__ TensCorner tens_corner(dd x, dd y, dd z) {
  const dd x2 = dd_mul(x, x), y2 = dd_mul(y, y), z2 = dd_mul(z, z);
  const dd d = dd_sqrt(dd_add(dd_add(x2, y2), z2));
  const dd xyz = dd_mul(dd_mul(x, y), z);
  const dd ax = dd_atan(dd_div(dd_mul(y, z), tens_den(x, d)));
  const dd ay = dd_atan(dd_div(dd_mul(z, x), tens_den(y, d)));
  const dd az = dd_atan(dd_div(dd_mul(x, y), tens_den(z, d)));
  const dd lmx = tens_log(dd_sub(d, x)), lmy = tens_log(dd_sub(d, y)), lmz = tens_log(dd_sub(d, z));
  const dd lpx = tens_log(dd_add(d, x)), lpy = tens_log(dd_add(d, y)), lpz = tens_log(dd_add(d, z));
  const dd sixth = dd_recip_int(6), third = dd_recip_int(3);
  auto half = [](dd v) { return dd_ldexp(v, -1); };
  TensCorner c;
  // g1(x, y, z, d)
  c.t00 = dd_add(dd_add(dd_mul(xyz, ax), half(dd_mul(dd_mul(y, dd_sub(z2, x2)), lmy))),
                 dd_add(half(dd_mul(dd_mul(z, dd_sub(y2, x2)), lmz)),
                        dd_mul(dd_mul(dd_sub(dd_add(y2, z2), dd_ldexp(x2, 1)), d), sixth)));
  // g1(y, z, x, d)
  c.t11 = dd_add(dd_add(dd_mul(xyz, ay), half(dd_mul(dd_mul(z, dd_sub(x2, y2)), lmz))),
                 dd_add(half(dd_mul(dd_mul(x, dd_sub(z2, y2)), lmx)),
                        dd_mul(dd_mul(dd_sub(dd_add(z2, x2), dd_ldexp(y2, 1)), d), sixth)));
  // g1(z, x, y, d)
  c.t22 = dd_add(dd_add(dd_mul(xyz, az), half(dd_mul(dd_mul(x, dd_sub(y2, z2)), lmx))),
                 dd_add(half(dd_mul(dd_mul(y, dd_sub(x2, z2)), lmy)),
                        dd_mul(dd_mul(dd_sub(dd_add(x2, y2), dd_ldexp(z2, 1)), d), sixth)));
  // g2(x, y, z, d): -x y z log(d+x) + z (z^2 - 3x^2) log(d+y)/6 + y (y^2 - 3x^2) log(d+z)/6
  //   + y^2 x A_y / 2 + z^2 x A_z / 2 + x^3 A_x / 6 + y z d / 3
  c.t12 = dd_add(dd_add(dd_neg(dd_mul(xyz, lpx)),
                        dd_mul(dd_add(dd_mul(dd_mul(z, dd_sub(z2, dd_mul_d(x2, 3.0))), lpy),
                                      dd_mul(dd_mul(y, dd_sub(y2, dd_mul_d(x2, 3.0))), lpz)),
                               sixth)),
                 dd_add(dd_add(half(dd_mul(dd_mul(y2, x), ay)), half(dd_mul(dd_mul(z2, x), az))),
                        dd_add(dd_mul(dd_mul(dd_mul(x2, x), ax), sixth), dd_mul(dd_mul(dd_mul(y, z), d), third))));
  // g2(y, z, x, d)
  c.t02 = dd_add(dd_add(dd_neg(dd_mul(xyz, lpy)),
                        dd_mul(dd_add(dd_mul(dd_mul(x, dd_sub(x2, dd_mul_d(y2, 3.0))), lpz),
                                      dd_mul(dd_mul(z, dd_sub(z2, dd_mul_d(y2, 3.0))), lpx)),
                               sixth)),
                 dd_add(dd_add(half(dd_mul(dd_mul(z2, y), az)), half(dd_mul(dd_mul(x2, y), ax))),
                        dd_add(dd_mul(dd_mul(dd_mul(y2, y), ay), sixth), dd_mul(dd_mul(dd_mul(z, x), d), third))));
  // g2(z, x, y, d)
  c.t01 = dd_add(dd_add(dd_neg(dd_mul(xyz, lpz)),
                        dd_mul(dd_add(dd_mul(dd_mul(y, dd_sub(y2, dd_mul_d(z2, 3.0))), lpx),
                                      dd_mul(dd_mul(x, dd_sub(x2, dd_mul_d(z2, 3.0))), lpy)),
                               sixth)),
                 dd_add(dd_add(half(dd_mul(dd_mul(x2, z), ax)), half(dd_mul(dd_mul(y2, z), ay))),
                        dd_add(dd_mul(dd_mul(dd_mul(z2, z), az), sixth), dd_mul(dd_mul(dd_mul(x, y), d), third))));
  return c;
}

// volume_averaged_n (tensor_element.f90:13-102) in double-double: t over the
// 64 corner combinations with the reference's signs; the source offset
// (rx, ry) is (ix dx, iy dy) for integers ix, iy, exactly; rz as given.
// n[a*3+b] -= t(a,b).  The reference's quirk dyo = xo (:31) is kept.
__device__ void vol_avg_n(double ix, double iy, double dxc, double dyc, double rz, double xs, double ys,
                          double zs, double xo, double zo, dd* n) {
  const dd rx = two_prod(ix, dxc), ry = two_prod(iy, dyc);
  dd t00 = dd_from(0), t11 = dd_from(0), t22 = dd_from(0), t12 = dd_from(0), t02 = dd_from(0), t01 = dd_from(0);
#pragma unroll 1
  for (int c = 0; c < 64; ++c) {
    const int i1 = 1 + (c & 1), i2 = 1 + ((c >> 1) & 1), i3 = 1 + ((c >> 2) & 1);
    const int i4 = 1 + ((c >> 3) & 1), i5 = 1 + ((c >> 4) & 1), i6 = 1 + ((c >> 5) & 1);
    // dx = -rx + dxo(i3) - dxs(i6), dxo = xo (-1/2, 1/2), dxs = xs (-1/2, 1/2)
    const dd dx = dd_add_d(dd_add_d(dd_neg(rx), (i3 == 1 ? -0.5 : 0.5) * xo), -((i6 == 1 ? -0.5 : 0.5) * xs));
    const dd dy = dd_add_d(dd_add_d(dd_neg(ry), (i2 == 1 ? -0.5 : 0.5) * xo), -((i5 == 1 ? -0.5 : 0.5) * ys));
    const dd dz = dd_add_d(dd_add_d(dd_from(-rz), (i1 == 1 ? -0.5 : 0.5) * zo), -((i4 == 1 ? -0.5 : 0.5) * zs));
    if (dx.hi == 0.0 && dy.hi == 0.0 && dz.hi == 0.0) continue;  // d = 0
    const TensCorner k = tens_corner(dx, dy, dz);
    const bool minus = ((i1 + i2 + i3 + i4 + i5 + i6 - 1) & 1) != 0;
    auto acc = [&](dd& a, dd v) { a = minus ? dd_sub(a, v) : dd_add(a, v); };
    acc(t00, k.t00);
    acc(t11, k.t11);
    acc(t22, k.t22);
    acc(t12, k.t12);
    acc(t02, k.t02);
    acc(t01, k.t01);
  }
  // t(1,1), t(2,2), t(3,3); t(2,3) = t(3,2) = g2(x,y,z); t(1,3) = t(3,1) = g2(y,z,x); t(1,2) = t(2,1) = g2(z,x,y)
  n[0] = dd_sub(n[0], t00);
  n[4] = dd_sub(n[4], t11);
  n[8] = dd_sub(n[8], t22);
  n[5] = dd_sub(n[5], t12);
  n[7] = dd_sub(n[7], t12);
  n[2] = dd_sub(n[2], t02);
  n[6] = dd_sub(n[6], t02);
  n[1] = dd_sub(n[1], t01);
  n[3] = dd_sub(n[3], t01);
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
                           double dzo, double rz, int nimg, dd* acc) {
  int il[2], jl[2];
  const int ni = slot_offsets(fi, nx, il), nj = slot_offsets(fj, ny, jl);
  for (int k = 0; k < 9; ++k) acc[k] = dd_from(0.0);
  for (int qj = 0; qj < nj; ++qj) {
    const int j = jl[qj];
    const int yp0 = -nimg * (1 - max(0, j / ((ny + 1) / 2)));
    const int yp1 = nimg * (1 + min(0, j / ((ny + 1) / 2)));
    for (int qi = 0; qi < ni; ++qi) {
      const int i = il[qi];
      const int xp0 = -nimg * (1 - max(0, i / ((nx + 1) / 2)));
      const int xp1 = nimg * (1 + min(0, i / ((nx + 1) / 2)));
      dd t[9];
      for (int k = 0; k < 9; ++k) t[k] = dd_from(0.0);
      for (int iy = yp0; iy <= yp1; ++iy)
        for (int ix = xp0; ix <= xp1; ++ix)
          vol_avg_n((double)i + (double)ix * (double)nx, (double)j + (double)iy * (double)ny, dx, dy, rz, dx, dy,
                    dz, dx, dzo, t);
      for (int k = 0; k < 9; ++k) acc[k] = dd_add(acc[k], t[k]);
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
  dd acc[9], tot[9];
  slot_plane(fi, fj, px, py, dx, dy, g.dz_s, g.dz_o, g.rz, nimg, acc);
  for (int k = 0; k < 9; ++k) tot[k] = acc[k];
  if (g.f_sul != 0.0) {
    slot_plane(fi, fj, px, py, dx, dy, g.dz_s, g.dz_o, g.rz_sul, nimg, acc);
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) tot[a * 3 + b] = dd_add(tot[a * 3 + b], dd_mul_d(acc[a * 3 + b], a < 2 ? -g.f_sul : g.f_sul));
  }
  if (g.f_head != 0.0) {
    slot_plane(fi, fj, px, py, dx, dy, g.dz_s, g.dz_o, g.rz_head, nimg, acc);
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b)
        tot[a * 3 + b] = dd_add(tot[a * 3 + b], dd_mul_d(acc[a * 3 + b], a < 2 ? -g.f_head : g.f_head));
  }
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b)
      n2d[(((long long)pair * 9 + 3 * b + a) * py + fj) * px + fi] = dd_mul_d(tot[a * 3 + b], g.norm).hi;
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

// spectrum [0][9][py][ph] (FP64, one layer) -> tens[k][6][py] floats for the
// register column kernel (colreg.cuh): components xx, yy, zz, xy, xz, yz (the
// tensor is symmetric: yx, zx, zy are xy, xz, yz) at the positions of the
// column transform's digit-reversed order (element p holds k_y = ip_freq(p)),
// the sign of the odd components for k_y > py/2 folded in.  The residue adds
// any difference between a component and its transpose.
__global__ void pack_tensor_creg_kernel(const Cx<double>* __restrict__ spec, float* __restrict__ tens, int lgpy,
                                        int ph, unsigned long long* resid, unsigned long long* kept) {
  const int py = 1 << lgpy;
  const long long total = (long long)ph * 6 * py;
  const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  double keep = 0.0, disc = 0.0;
  if (gid < total) {
    const int p = (int)(gid % py);
    const int c6 = (int)((gid / py) % 6);
    const int k = (int)(gid / ((long long)6 * py));
    const int ky = ip_freq(p, lgpy);
    const bool upper = ky > py / 2;
    const int kyh = upper ? py - ky : ky;
    constexpr int kComp[6] = {0, 4, 8, 1, 2, 5};   // xx yy zz xy xz yz
    constexpr int kTrans[6] = {0, 4, 8, 3, 6, 7};  // their transposes
    const int c = kComp[c6];
    parity_parts(spec + (long long)c * py * ph, c, kyh, k, py, ph, &keep, &disc);
    if (kTrans[c6] != c) {
      double kt, dt;
      parity_parts(spec + (long long)kTrans[c6] * py * ph, kTrans[c6], kyh, k, py, ph, &kt, &dt);
      disc = fmax(disc, fmax(dt, fabs(kt - keep)));
    }
    const bool odd = (kOddMask >> c) & 1;
    tens[gid] = (float)((odd && upper) ? -keep : keep);
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
