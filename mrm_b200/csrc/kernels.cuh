// kernels.cuh -- fused per-step kernels of the grain-dynamics path (sm_100a).
//
// One Heun step (src/llg.f90:1195-1271, llg_type = -3) is four launches:
//   row<PRED>  : inverse row FFT of H^(m_n) -> H_demag, field assembly
//                (field.f90:197-225), Philox thermal field (field.f90:397-436),
//                Heun predictor (llg.f90:1122-1139, iter = 2), forward row FFT
//                of Ms*m* (data.f90:322-390 scatter + demag.f90:113-116)
//   col        : column FFT, tensor multiply (demag.f90:117-121), inverse
//                column FFT, all in shared memory
//   row<CORR>  : same with the corrector (iter = 1) at t+dt on m*, thermal
//                regenerated from the same counter; optional FP64 reductions
//                (llg.f90:217-237, push_llg errmx/errmx1/mmag)
//   col
// The spectrum buffer always holds H^(m) of the state it follows, so a step
// starts from it without a separate demag pass.
//
// Latency layout: every per-grain global load (state, parameters, lattice
// neighbours, columnar interlayer partner) is issued at the top of the row
// kernel, before the inverse FFT, so its latency overlaps the shared-memory
// passes; the column kernel batches its strided loads the same way.
#pragma once
#include "common.cuh"
#include "fft.cuh"
#include "regfft.cuh"
#include "philox.cuh"
#include "tma.cuh"

namespace mrm {

enum Stage { kInit = 0, kPred = 1, kCorr = 2, kEval = 3 };
enum Flags {
  kFlagStats = 1, kFlagForce = 2, kFlagStoreField = 4, kFlagBoris = 8, kFlagMid = 16, kFlagStoredField = 32,
  kFlagMapped = 64, kFlagDemagOnly = 128, kFlagCorrTime = 256, kFlagProbeTimeout = 512, kFlagRot = 1024
};
// kFlagRot (with kFlagBoris): the analytic-rotation push of llg_type 1 / -1
// in place of the semi-implicit one (push_llg, llg.f90:1093-1107).
// kFlagProbeTimeout (row kernel): the grain-row barrier expects 16 bytes that
// no copy sends, so every block's bounded wait runs out and the block takes the
// failure path a lost bulk copy would (error flag, second bounded wait,
// return) -- the device failure test of mrm_gpu_selftest_timeout.
// kFlagMapped (kPred, kCorr, kEval): the demag field comes from an earlier
// evaluation's per-cell values averaged over each grain's cells (L.hdm; L.hd
// with one grain per cell), not from this launch's inverse row transform.
// kFlagDemagOnly (kEval): the inverse transforms' demag per cell (L.hd) only.
// kFlagCorrTime (gather_demag_kernel): the applied field at the corrector's time.
// kFlagStoredField (kPred): the push uses the stored field L.hf instead of the
// field of m_n -- push_m's retry after a rejected adaptive step, whose field
// is still the one of the rejected predicted state (llg.f90:1205-1266)
// llg_type -3 (Heun): kPred + kCorr.  llg_type -2: kPred with kFlagBoris |
// kFlagMid (semi-implicit push over dt/2) then kCorr with the same flags (field
// at t+dt/2 on the predicted state, push of m_n over dt).  llg_type 2: kPred
// with kFlagBoris alone (one push over dt into the predictor buffer; the
// commit kernel copies it to the state).

template <typename R>
MRM_D void cross3(R ax, R ay, R az, R bx, R by, R bz, R& cx, R& cy, R& cz) {
  cx = ay * bz - az * by;
  cy = az * bx - ax * bz;
  cz = ax * by - ay * bx;
}

// rotate_q (transform.f90:65-74): m -> w ** (0, m) ** w* for the quaternion w
MRM_D void rotate_q(const double* w, const double* m, double* t) {
  const double w1 = w[0] * w[0], w2 = w[1] * w[1], w3 = w[2] * w[2], w4 = w[3] * w[3];
  t[0] = 2.0 * (m[2] * (w[0] * w[2] + w[1] * w[3]) + m[1] * (w[1] * w[2] - w[0] * w[3])) + m[0] * (w1 + w2 - w3 - w4);
  t[1] = 2.0 * (m[0] * (w[0] * w[3] + w[1] * w[2]) + m[2] * (w[2] * w[3] - w[0] * w[1])) + m[1] * (w1 + w3 - w2 - w4);
  t[2] = 2.0 * (m[1] * (w[0] * w[1] + w[2] * w[3]) + m[0] * (w[1] * w[3] - w[0] * w[2])) + m[2] * (w1 + w4 - w3 - w2);
}

// rotate_2 (transform.f90:97-115) with norm0 given and norm1 absent: m
// rotated about u0 (normalised; (0,0,1) and no turn if it is zero) by th0,
// then about u1 (as given) by th1
MRM_D void rotate_2(double th0, const double* u0, double th1, const double* u1, const double* m, double* t) {
  double st1 = 0.5 * th1, st0 = 0.5 * th0;
  double t0[3] = {u0[0], u0[1], u0[2]};
  const double n0 = sqrt(t0[0] * t0[0] + t0[1] * t0[1] + t0[2] * t0[2]);
  if (n0 != 0.0) {
    t0[0] /= n0;
    t0[1] /= n0;
    t0[2] /= n0;
  } else {
    t0[0] = 0.0;
    t0[1] = 0.0;
    t0[2] = 1.0;
    st0 = 0.0;
  }
  if (st0 == 0.0 && st0 == st1) {
    t[0] = m[0];
    t[1] = m[1];
    t[2] = m[2];
    return;
  }
  const double ct1 = cos(st1);
  st1 = sin(st1);
  const double ct0 = cos(st0);
  st0 = sin(st0);
  const double* t1 = u1;
  const double q[4] = {ct0 * ct1 - (t0[0] * t1[0] + t0[1] * t1[1] + t0[2] * t1[2]) * st0 * st1,
                       t0[0] * ct1 * st0 + (t1[0] * ct0 + (t1[1] * t0[2] - t0[1] * t1[2]) * st0) * st1,
                       t0[1] * ct1 * st0 + (t1[1] * ct0 + (t1[2] * t0[0] - t0[2] * t1[0]) * st0) * st1,
                       t0[2] * ct1 * st0 + (t1[2] * ct0 + (t1[0] * t0[1] - t0[0] * t1[1]) * st0) * st1};
  rotate_q(q, m, t);
}

// Analytic-rotation push of llg_type 1 / -1 (llg.f90:1093-1107), FP64: the
// precession |s11| about h and the damping turn th0 - 2 atan(e^(s11 a) tan(th0/2))
// about m x h, s11 = 2 s1 |h| / (1 + a^2), s1 = -gamma dt / 2; d = m' - m
MRM_D void rot_push(const double* m, const double* h, double s1, double a, double* d) {
  double y = h[0] * h[0] + h[1] * h[1] + h[2] * h[2];
  if (!(y > 0.0)) {
    d[0] = d[1] = d[2] = 0.0;
    return;
  }
  y = sqrt(y);
  const double s11 = 2.0 * s1 * y / (1.0 + a * a);
  const double o[3] = {h[0] / y, h[1] / y, h[2] / y};
  const double th0 = acos(fmin(1.0, fmax(-1.0, o[0] * m[0] + o[1] * m[1] + o[2] * m[2])));
  const double u0[3] = {m[1] * o[2] - m[2] * o[1], m[2] * o[0] - m[0] * o[2], m[0] * o[1] - m[1] * o[0]};
  double t[3];
  rotate_2(th0 - 2.0 * atan(exp(s11 * a) * tan(0.5 * th0)), u0, fabs(s11), o, m, t);
  d[0] = t[0] - m[0];
  d[1] = t[1] - m[1];
  d[2] = t[2] - m[2];
}

// funct (applied.f90:328-377); Fortran mod(x,g) = x - int(x/g)*g = fmod.
// f = 7 (ROT) is its branch with the rotation angles present and |gamma| != 1:
// magnitude 1 along the rotating direction of rot_dir
MRM_D double funct(int f, double t, double g, double phase, double param, double duty,
                   double moddepth) {
  if (f == 7) return 1.0;
  if (f == 1) return sin(t * g + phase);
  if (f == 2) return cos(t * g + phase);
  if (f == 3) return exp(t * g + phase);
  if (f == 5) {  // NEW
    double x = g / param;
    const double y = exp(duty * x), w = exp(x);
    x = t + phase;
    if (x < 0.0) x = x + g * (1.0 + (double)(long long)fabs(x / g));
    x = fmod(x, g);
    if (x > duty * g) {
      x = exp((g - x) / param);
      return 1.0 - moddepth + x * (y - 1.0) * moddepth / (w - 1.0);
    }
    x = exp(-x / param);
    return 1.0 + x * (y - w) * moddepth / (w - 1.0);
  }
  if (f == 4) {  // STE: trapezoidal square wave of period g, rise time param
    double x = t + phase;
    if (x < 0.0) x = x + g * (1.0 + (double)(long long)fabs(x / g));
    x = fmod(x, g);
    if (x < 0.5 * param) return 2.0 * x / param;
    if (x < 0.5 * (g - param)) return 1.0;
    if (x < 0.5 * (g + param)) return (g - 2.0 * x) / param;
    if (x < g - 0.5 * param) return -1.0;
    return 2.0 * (x - g) / param;
  }
  return 0.0;
}

// direction of a ROT field at time t (applied.f90:382-383, rot_fld :398-416):
// (cos((2 gamma t + phase) pi), sin((2 gamma t + phase) pi), 0)
MRM_D void rot_dir(double g, double phase, double t, double* d) {
  const double th = (2.0 * g * t + phase) * 3.14159265358979323846;
  d[0] = cos(th);
  d[1] = sin(th);
  d[2] = 0.0;
}

// time scale of a layer's uniform field (applied.f90:866-883; set_fld folds
// a constant ramp into `scale`, :309-312)
template <typename R>
MRM_D double ramp(const LayerDev<R>& L, double t) {
  if (L.func != 0)
    return (L.amp * funct(L.func, t, L.fgamma, L.phase, L.param, L.duty, L.moddepth) + L.dc) * L.scale;
  double u = (t - L.t_start) / (L.t_end - L.t_start);
  u = fmax(0.0, fmin(1.0, u));
  return ((L.s_end - L.s_start) * u + L.s_start) * L.scale;
}

// Temperature profile (TempDev): x**n for an integer n >= 0 by squaring (the
// reference's real**integer), the profile's time scale and a cell's temperature
MRM_HD double powi(double x, int n) {
  double r = 1.0;
  while (n > 0) {
    if (n & 1) r *= x;
    x *= x;
    n >>= 1;
  }
  return r;
}
MRM_D double temp_scale(const TempDev& P, double t) {
  if (P.func != 0) return (P.amp * funct(P.func, t, P.fgamma, P.phase, P.param, P.duty, P.moddepth) + P.dc) * P.scale;
  double u = (t - P.t_start) / (P.t_end - P.t_start);
  u = fmax(0.0, fmin(1.0, u));
  return ((P.s_end - P.s_start) * u + P.s_start) * P.scale;
}
// set_sg (applied.f90:1778-1790) and get_sg (:1792-1809) at grid cell (i, j);
// s = dtemp times the time scale
MRM_D double temp_cell(const TempDev& P, double s, double t, int i, int j) {
  const double delx = P.rx - P.vx * (t - P.t0) - P.ox, dely = P.ry - P.vy * (t - P.t0) - P.oy;
  const double fx = exp(-powi((P.dx * ((double)i + 0.5) + delx) * P.isx, P.expn));
  const double fy = exp(-powi((P.dy * ((double)j + 0.5) + dely) * P.isy, P.expn));
  return P.bg + s * fy * fx;
}

// find_temp_scaling (temp_scaling.f90:365-430) for one cell.  A table at
// x = T/Tc: its first scale at or below the first node, its last at or above
// the last, linear in between (bisection on the nodes, :397-414).
MRM_D double tsc_table(const double* tt, const double* tv, int n, double x) {
  int k1 = 0, k2 = n - 1;
  double y;
  if (x <= tt[0]) {
    y = 0.0;
  } else if (x >= tt[k2]) {
    y = 0.0;
    k1 = k2;
  } else {
    while (k2 - k1 > 1) {
      const int k = (k2 + k1 + 2) / 2 - 1;  // the midpoint of the 1-based indices
      if (x < tt[k]) k2 = k;
      else k1 = k;
    }
    y = fmax(0.0, fmin(1.0, (x - tt[k1]) / (tt[k2] - tt[k1])));
  }
  return tv[k1] + y * (tv[k2] - tv[k1]);
}
// Ms scale of cell n at temperature T (|m| = mag): |m| itself (use_mag_p),
// the power law, the table, or 1
MRM_D double tsc_ms(const TscDev& S, int n, double T, double mag) {
  if (S.mag) return fmin(1.0, fmax(0.0, fabs(mag)));
  if (S.msexp >= 0.0) return pow(fmin(1.0, fmax(0.0, 1.0 - T / S.tc[n])), S.msexp);
  if (S.nt[0] > 1) return tsc_table(S.tt + S.off[0], S.tv + S.off[0], S.nt[0], T / S.tc[n]);
  return 1.0;
}
MRM_D double tsc_alpha(const TscDev& S, int n, double T) {
  return S.nt[1] > 1 ? tsc_table(S.tt + S.off[1], S.tv + S.off[1], S.nt[1], T / S.tc[n]) : 1.0;
}
MRM_D double tsc_hk(const TscDev& S, int n, double T) {
  if (S.hkexp >= 0.0) return pow(fmin(1.0, fmax(0.0, 1.0 - T / S.tc[n])), S.hkexp);
  if (S.nt[2] > 1) return tsc_table(S.tt + S.off[2], S.tv + S.off[2], S.nt[2], T / S.tc[n]);
  return 1.0;
}
// temperature of cell (i, j) of a layer at time t: its profile's, or the uniform one
template <typename R>
MRM_D double layer_temp(const LayerDev<R>& L, double t, int i, int j) {
  if (!L.tprof) return L.temperature;
  const TempDev& P = *L.tprof;
  return temp_cell(P, P.dtemp * temp_scale(P, t), t, i, j);
}

// Write head (func 6): gap-centre position and write polarity at time t
template <typename R>
MRM_D void head_state(const LayerDev<R>& L, double t, double* xh, double* pol) {
  *xh = L.hd_x0 + L.hd_v * (t - L.hd_t0);
  long long k = (long long)floor((t - L.hd_t0) / L.hd_tbit);
  const long long nb = L.hd_nbits > 0 ? L.hd_nbits : 1;
  k %= nb;
  if (k < 0) k += nb;
  *pol = ((L.hd_bits >> k) & 1ull) ? 1.0 : -1.0;
}

// Karlqvist field at down-track offset u from the gap centre:
//   h_x = Hg/pi (atan((u + g/2)/z) - atan((u - g/2)/z))
//   h_z = Hg/(2 pi) ln(((u - g/2)^2 + z^2) / ((u + g/2)^2 + z^2))
template <typename R>
MRM_D void karlqvist(R u, R g, R z, R hg, R& hx, R& hz) {
  const R a = u + (R)0.5 * g, b = u - (R)0.5 * g;
  const R pi = (R)3.14159265358979323846;
  hx = hg / pi * (atan(a / z) - atan(b / z));
  hz = hg / ((R)2 * pi) * log((b * b + z * z) / (a * a + z * z));
}

// Interpolation weights of a tabulated field profile: the table interval
// [k, k+1] and the weight f of node k for one mesh coordinate.
struct TabW {
  int k, pad;
  double f;
};

// set (applied.f90:1757-1776) for one mesh coordinate x over the n >= 2
// ascending nodes pos[]: the first node above x, searched from the second
// node on and capped at the last, closes the interval; the lower node's
// weight is clamped to [0, 1].  (A bisection: the reference's sweep gives the
// same node on ascending positions.)
MRM_D TabW tab_weight(const double* __restrict__ pos, int n, double x) {
  int lo = 1, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (pos[mid] > x) hi = mid;
    else lo = mid + 1;
  }
  TabW w;
  w.k = lo - 1;
  w.pad = 0;
  w.f = fmax(0.0, fmin(1.0, (pos[lo] - x) / (pos[lo] - pos[lo - 1])));
  return w;
}

// interpolate (applied.f90:1471-1520): s-scaled bilinear value of the vector
// profile at one cell from its column and row weights
MRM_D void tab_value(const double* __restrict__ v, int tnx, TabW wx, TabW wy, double s, double& vx, double& vy,
                     double& vz) {
  const double yf = s * wy.f, yfc = s * (1.0 - wy.f);
  const double w00 = wx.f * yf, w10 = (1.0 - wx.f) * yf, w01 = wx.f * yfc, w11 = (1.0 - wx.f) * yfc;
  const double* __restrict__ a = v + 3 * ((size_t)wy.k * tnx + wx.k);
  const double* __restrict__ c = a + 3 * (size_t)tnx;
  vx = w00 * a[0] + w10 * a[3] + w01 * c[0] + w11 * c[3];
  vy = w00 * a[1] + w10 * a[4] + w01 * c[1] + w11 * c[4];
  vz = w00 * a[2] + w10 * a[5] + w01 * c[2] + w11 * c[5];
}

// ---------------- LLB integrator (llgp%llb) ----------------
// (The integrators below are calls, not inlined: their FP64 state would
// otherwise share the general row kernel's register budget and spill on its
// common paths.)
constexpr double kGmubKb = 1.343427768e-4;  // g mu_B / k_B (llg.f90:924)
constexpr double kBoltz = 1.380662e-16;     // field.f90:407

// lv(x) = coth x - 1/x and dlv = d lv/dx = 1/x^2 - csch^2 x with the
// reference's small-argument forms (llg.f90:704-710,727-733)
MRM_D double llb_lv(double x) { return fabs(x) > 1e-2 ? 1.0 / tanh(x) - 1.0 / x : x / 3.0; }
MRM_D double llb_dlv(double x) {
  if (fabs(x) > 4e-3) {
    const double s = sinh(x);
    return 1.0 / (x * x) - 1.0 / (s * s);
  }
  return 1.0 / 3.0;
}

// One grain of push_llb (llg.f90:916-1064), Heun (llg_type -3):
//   mc, magc: the current state and magnitude; mpr, magp: the predicted ones
//   (second pass); h: the field without thermal; ht: thermal field / sqrt(dt);
//   d1: the first pass's increment (second pass); ab = alpha alpha_scale;
//   tc, lam = Tc and lambdaMs (spin + 1)/spin; T the temperature; dt the step.
// Out: the new direction and magnitude, the increment d (the first pass
// stores it), |d|^2 (errmx1: the squared magnitude change on the |m| = 0
// branch) and |m x (h + h_perp)|^2 (errmx).
struct LlbStep {
  double m[3], mag, d[3], d2, tq2;
};
static __device__ __noinline__ LlbStep llb_heun(bool corr, const double* mc, double magc, const double* mpr, double magp, const double* h,
                       const double* ht, const double* d1, double ab, double tc, double lam, const LlbDev& P,
                       double T, double gamma, double dt) {
  LlbStep o;
  const double scale1 = -0.5 * gamma * dt;
  o.tq2 = 0.0;
  if (!(magc > 0.0)) {
    // |m| = 0 (llg.f90:1048-1060): m along h, |m| relaxed towards its equilibrium
    const double y = sqrt(h[0] * h[0] + h[1] * h[1] + h[2] * h[2]);
    if (y > 0.0) {
      for (int a = 0; a < 3; ++a) o.m[a] = h[a] / y;
      const double meq = kGmubKb * P.spin * y / T;
      const double scale2 = lam * T / (3.0 * llb_dlv(meq) * tc);
      o.mag = (y / scale2 + llb_lv(meq)) * (1.0 - exp(2.0 * scale1 * scale2 * 2.0 * T * P.alpha / (3.0 * tc)));
    } else {
      for (int a = 0; a < 3; ++a) o.m[a] = mc[a];
      o.mag = magc;
    }
    for (int a = 0; a < 3; ++a) o.d[a] = 0.0;
    o.d2 = (o.mag - magc) * (o.mag - magc);
    return o;
  }
  double m[3], mag;
  if (corr) {  // llg.f90:1002-1004
    for (int a = 0; a < 3; ++a) m[a] = mpr[a];
    mag = magp;
    if (mag <= 0.0) {
      mag = 0.0;
      const double y = sqrt(h[0] * h[0] + h[1] * h[1] + h[2] * h[2]);
      if (y != 0.0)
        for (int a = 0; a < 3; ++a) m[a] = h[a] / y;
    }
  } else {
    for (int a = 0; a < 3; ++a) m[a] = mc[a];
    mag = magc;
  }
  double ht3[3];
  for (int a = 0; a < 3; ++a) ht3[a] = h[a] + lam * mag * m[a];
  const double mh = sqrt(ht3[0] * ht3[0] + ht3[1] * ht3[1] + ht3[2] * ht3[2]);
  if (mh != 0.0)
    for (int a = 0; a < 3; ++a) ht3[a] /= mh;
  const double meq = kGmubKb * P.spin * mh / T;
  const double lvm = llb_lv(meq);
  const double aperp = P.alpha * (1.0 - lam * lvm * T / (3.0 * mh * tc));
  const double apar = P.alpha * 2.0 * T / (3.0 * tc);
  // thermal field hthm / sqrt(alpha alpha_scale dt0), split along m (llg.f90:1016-1026)
  const double rs = 1.0 / sqrt(ab);
  double th[3], hpar[3], hperp[3];
  for (int a = 0; a < 3; ++a) th[a] = ht[a] * rs;
  const double tp = th[0] * m[0] + th[1] * m[1] + th[2] * m[2];
  const double fpar = sqrt(apar), fperp = sqrt(fmax(0.0, aperp - apar) / (aperp * aperp));
  for (int a = 0; a < 3; ++a) {
    hpar[a] = tp * m[a];
    hperp[a] = (th[a] - hpar[a]) * fperp;
    hpar[a] *= fpar;
  }
  const double scale11 = 2.0 * scale1;
  const double mht = m[0] * ht3[0] + m[1] * ht3[1] + m[2] * ht3[2];
  const double mq = apar * (lam / mh) * lam * 2.0 * scale1 * T * lvm / (3.0 * llb_dlv(meq) * tc) * (mag - lvm * mht);
  double hh[3] = {h[0] + hperp[0], h[1] + hperp[1], h[2] + hperp[2]}, t[3], mxh[3], mxt[3];
  cross3(m[0], m[1], m[2], hh[0], hh[1], hh[2], t[0], t[1], t[2]);
  cross3(m[0], m[1], m[2], h[0], h[1], h[2], mxh[0], mxh[1], mxh[2]);
  cross3(m[0], m[1], m[2], t[0], t[1], t[2], mxt[0], mxt[1], mxt[2]);
  const double sm = copysign(fmin(0.5, fabs(mq)), mq);
  for (int a = 0; a < 3; ++a) o.d[a] = scale11 * (mag * mxh[a] + aperp * mxt[a] + hpar[a]) + sm * m[a];
  if (corr)
    for (int a = 0; a < 3; ++a) o.d[a] = 0.5 * (o.d[a] + d1[a]);
  o.tq2 = t[0] * t[0] + t[1] * t[1] + t[2] * t[2];
  o.d2 = o.d[0] * o.d[0] + o.d[1] * o.d[1] + o.d[2] * o.d[2];
  // m(t+dt) = m |m| + d (llg.f90:1039-1047)
  double w[3];
  for (int a = 0; a < 3; ++a) w[a] = mc[a] * magc + o.d[a];
  const double y = sqrt(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]);
  if (y > 0.0) {
    for (int a = 0; a < 3; ++a) o.m[a] = w[a] / y;
    o.mag = y;
  } else {
    for (int a = 0; a < 3; ++a) o.m[a] = -mc[a];
    o.mag = 0.0;
  }
  return o;
}

// One grain of push_llb's semi-implicit branch (llg.f90:935-999), |type| = 2:
// first = the first or only pass (llg_type 2, or the first pass of -2, which
// relaxes |m| from the current state), else the second pass of -2 (from the
// predicted state mpr, magp).  dt is the pass's step (dt/2 for the first pass
// of -2).  Out: the new direction and magnitude, |dm|^2 as errmx1 forms it,
// |m x h|^2.  (|m| = 0: llb_heun's branch, the same for both pushes.)
static __device__ __noinline__ LlbStep llb_boris(bool first, const double* mc, double magc, const double* mpr, double magp, const double* h,
                        const double* ht, double ab, double tc, double lam, const LlbDev& P, double T, double gamma,
                        double dt) {
  LlbStep o;
  const double scale1 = -0.5 * gamma * dt, scale11 = scale1;
  const double a = P.alpha;
  double m[3], mag, ht3[3], mh, meq;
  auto field_tot = [&](const double* mm, double mg) {
    for (int c = 0; c < 3; ++c) ht3[c] = h[c] + lam * mg * mm[c];
    mh = sqrt(ht3[0] * ht3[0] + ht3[1] * ht3[1] + ht3[2] * ht3[2]);
    if (mh != 0.0)
      for (int c = 0; c < 3; ++c) ht3[c] /= mh;
    meq = kGmubKb * P.spin * mh / T;
  };
  if (first) {  // :940-947
    for (int c = 0; c < 3; ++c) m[c] = mc[c];
    field_tot(m, magc);
    const double lvm = llb_lv(meq);
    mag = lvm * (m[0] * ht3[0] + m[1] * ht3[1] + m[2] * ht3[2]);
    mag = mag + (magc - mag) * exp(scale1 * 2.0 * a * lam * lam * T * T * lvm /
                                   (3.0 * tc * tc * llb_dlv(meq) * (mh + 1e-20)));
  } else {
    for (int c = 0; c < 3; ++c) m[c] = mpr[c];
    mag = magp;
  }
  field_tot(m, mag);  // :952-954
  const double aperp = a * (1.0 - lam * llb_lv(meq) * T / (3.0 * mh * tc));
  const double apar = a * 2.0 * T / (3.0 * tc);
  const double scale2 = -aperp / (fabs(mag) + 1e-20);
  // h + hthm sqrt(|scale2 / (alpha alpha_scale dt0 (|mag| + 1e-20))|), hthm / sqrt(dt0) = ht
  const double fth = sqrt(fabs(scale2 / (ab * (fabs(mag) + 1e-20))));
  double hb[3], t[3], om[3], tt[3], d[3];
  for (int c = 0; c < 3; ++c) hb[c] = h[c] + ht[c] * fth;
  cross3(mc[0], mc[1], mc[2], hb[0], hb[1], hb[2], t[0], t[1], t[2]);
  o.tq2 = t[0] * t[0] + t[1] * t[1] + t[2] * t[2];
  for (int c = 0; c < 3; ++c) om[c] = scale11 * hb[c] + scale2 * mc[c];  // |type| = 2 (:971)
  cross3(mc[0], mc[1], mc[2], om[0], om[1], om[2], tt[0], tt[1], tt[2]);
  for (int c = 0; c < 3; ++c) tt[c] += mc[c];
  const double y = 2.0 / (1.0 + om[0] * om[0] + om[1] * om[1] + om[2] * om[2]);
  cross3(tt[0], tt[1], tt[2], om[0], om[1], om[2], d[0], d[1], d[2]);
  for (int c = 0; c < 3; ++c) {
    d[c] *= y;
    o.m[c] = mc[c] + d[c];
  }
  // the magnitude at the midpoint direction (:978-986)
  double mid[3];
  for (int c = 0; c < 3; ++c) mid[c] = mc[c] + 0.5 * d[c];
  field_tot(mid, mag);
  const double lvm = llb_lv(meq);
  const double sg = copysign(1.0, mag);
  double mg2 = lvm * sg * (mid[0] * ht3[0] + mid[1] * ht3[1] + mid[2] * ht3[2]);
  double q = mg2 + (magc - mg2) * exp(scale1 * 4.0 * a * lam * lam * T * T * lvm /
                                      (3.0 * tc * tc * llb_dlv(meq) * (mh + 1e-20)));
  const double fpar = sqrt(fabs(apar / ab));
  q = q - 2.0 * scale11 * (ht[0] * fpar * mid[0] + ht[1] * fpar * mid[1] + ht[2] * fpar * mid[2]);
  o.mag = fabs(q);
  if (q < 0.0) {  // :988-991
    const double r = sqrt(mid[0] * mid[0] + mid[1] * mid[1] + mid[2] * mid[2]);
    for (int c = 0; c < 3; ++c) {
      o.m[c] = -mid[c] / r;
      d[c] = o.m[c] - mc[c];
    }
  }
  const double ya = 0.5 * (o.mag + magc);
  double e[3];
  for (int c = 0; c < 3; ++c) {
    o.d[c] = d[c];
    e[c] = d[c] * ya + mc[c] * (o.mag - magc);
  }
  o.d2 = e[0] * e[0] + e[1] * e[1] + e[2] * e[2];
  return o;
}

// Brillouin function B_S and its derivative as bs / dbs write them (llg.f90:390-408)
MRM_D double mt_bs(double x, double sp) {
  double b = x / (2.0 * sp);
  if (b != 0.0) b = ((2.0 * sp + 1.0) / tanh((2.0 * sp + 1.0) * b) - 1.0 / tanh(b)) / (2.0 * sp);
  return b;
}
MRM_D double mt_dbs(double x, double sp) {
  double b = (1.0 + sp) / (3.0 * sp);
  if (x != 0.0) {
    b = x / (2.0 * sp);
    const double b1 = sinh(b);
    b = sinh(x + b);
    b = (1.0 / (b1 * b1) - (1.0 + 2.0 * sp) * (1.0 + 2.0 * sp) / (b * b)) / (4.0 * sp * sp);
  }
  return b;
}

// One grain of push_mt (llg.f90:735-915), dm/dt = -gamma m x H - (m - meq)/tau + eta:
// the Heun branch (:843-906; corr: the second pass) or the semi-implicit
// |type| = 2 branch (:757-842; first: the first or only pass).  mc, magc: the
// current state; mpr, magp: the predicted (second pass); h the field without
// thermal; ht the thermal field / sqrt(dt); d1 the first pass's increment
// (Heun); ab = alpha alpha_scale; lam = lambdaMs; T the temperature; dt the
// pass's step.  Out as llb_heun.
static __device__ __noinline__ LlbStep mt_step(bool boris, bool first, bool corr, const double* mc, double magc, const double* mpr, double magp,
                      const double* h, const double* ht, const double* d1, double ab, double lam0, const LlbDev& P,
                      double T, double gamma, double dt, double dt0) {
  LlbStep o;
  const double sp = P.spin;
  const double lam = P.meq_bs ? lam0 : lam0 * (sp + 1.0) / sp;
  const double y0 = kGmubKb * sp / T;
  const double scale1 = -0.5 * gamma * dt, scale11 = 2.0 * scale1;
  const double hth[3] = {ht[0] * sqrt(dt0), ht[1] * sqrt(dt0), ht[2] * sqrt(dt0)};  // hthm
  double m[3], mag, htot[3], mhtot;
  auto tot = [&](const double* v, double mg) {  // htot = h + lam mg v, normalised
    for (int c = 0; c < 3; ++c) htot[c] = h[c] + lam * mg * v[c];
    mhtot = sqrt(htot[0] * htot[0] + htot[1] * htot[1] + htot[2] * htot[2]);
    if (mhtot != 0.0)
      for (int c = 0; c < 3; ++c) htot[c] /= mhtot;
  };
  // eta, the stochastic increment with its parallel part scaled (:820-826, :874-884)
  auto noise = [&](double meq, double sig_p, double sig_l, double* eta) {
    double e[3];
    for (int c = 0; c < 3; ++c)
      e[c] = P.garanin_tau ? dt * hth[c] * gamma * sig_p * sqrt(2.0 / ((sig_l + (boris ? 1e-80 : 1e-22)) * dt0))
                           : dt * hth[c] * gamma * sqrt(lam * meq / ((mhtot + (boris ? 1e-80 : 1e-22)) * dt0));
    const double pe = htot[0] * e[0] + htot[1] * e[1] + htot[2] * e[2], r = sqrt(sig_l / sig_p);
    double x1[3], x2[3];
    cross3(htot[0], htot[1], htot[2], e[0], e[1], e[2], x1[0], x1[1], x1[2]);
    cross3(htot[0], htot[1], htot[2], x1[0], x1[1], x1[2], x2[0], x2[1], x2[2]);
    for (int c = 0; c < 3; ++c) eta[c] = r * pe * htot[c] - x2[c];
  };
  double d[3], t[3], eta[3];
  if (boris) {
    for (int c = 0; c < 3; ++c) m[c] = first ? mc[c] : mpr[c];
    mag = first ? magc : magp;
    tot(m, mag);
    const double yh = y0 * mhtot;
    double meq = P.meq_bs ? mt_bs(yh, sp) : llb_lv(yh);
    double scale2;
    if (P.garanin_tau) {
      const double sg = meq / (yh * (P.meq_bs ? mt_dbs(yh, sp) : llb_dlv(yh)) + 1e-80);
      scale2 = 2.0 * ab * sg / y0;
    } else {
      scale2 = ab * lam;
    }
    for (int c = 0; c < 3; ++c) m[c] = mc[c];
    mag = magc;
    cross3(m[0], m[1], m[2], h[0], h[1], h[2], t[0], t[1], t[2]);
    o.tq2 = t[0] * t[0] + t[1] * t[1] + t[2] * t[2];
    const double dec = 1.0 - exp(scale1 * scale2);
    double w[3], x[3];
    for (int c = 0; c < 3; ++c) d[c] = (meq * htot[c] - mag * m[c]) * dec;  // half decay (:802)
    for (int c = 0; c < 3; ++c) w[c] = mag * m[c] + d[c];
    cross3(w[0], w[1], w[2], h[0], h[1], h[2], x[0], x[1], x[2]);
    for (int c = 0; c < 3; ++c) d[c] += scale11 * x[c];  // full rotation (:803)
    for (int c = 0; c < 3; ++c) w[c] = mag * m[c] + d[c];
    for (int c = 0; c < 3; ++c) htot[c] = h[c] + lam * w[c];
    mhtot = sqrt(htot[0] * htot[0] + htot[1] * htot[1] + htot[2] * htot[2]);
    if (mhtot != 0.0)
      for (int c = 0; c < 3; ++c) htot[c] /= mhtot;
    const double y2 = y0 * mhtot;
    meq = P.meq_bs ? mt_bs(y2, sp) : llb_lv(y2);
    const double sig_p = meq / (y2 + 1e-80), sig_l = P.meq_bs ? mt_dbs(y2, sp) : llb_dlv(y2);
    if (P.garanin_tau) scale2 = 2.0 * ab * sig_p / (y0 * (sig_l + 1e-80));
    noise(meq, sig_p, sig_l, eta);
    const double dec2 = 1.0 - exp(scale1 * scale2);
    for (int c = 0; c < 3; ++c) d[c] = d[c] + (meq * htot[c] - w[c]) * dec2 + eta[c];  // :833
  } else {
    for (int c = 0; c < 3; ++c) m[c] = mc[c];
    mag = magc;
    if (corr) {  // :844-847
      for (int c = 0; c < 3; ++c) m[c] = mpr[c];
      mag = magp;
      if (mag <= 0.0) {
        mag = 0.0;
        const double e = sqrt(h[0] * h[0] + h[1] * h[1] + h[2] * h[2]);
        if (e != 0.0)
          for (int c = 0; c < 3; ++c) m[c] = h[c] / e;
      }
    }
    tot(m, mag);
    const double y = y0 * mhtot;
    const double meq = P.meq_bs ? mt_bs(y, sp) : llb_lv(y);
    const double sig_l = P.meq_bs ? mt_dbs(y, sp) : llb_dlv(y), sig_p = meq / (y + 1e-22);
    noise(meq, sig_p, sig_l, eta);
    const double scale2 = P.garanin_tau ? 2.0 * T * sig_p / (kGmubKb * sp * (sig_l + 1e-22)) : lam;
    double mm[3], x[3];
    for (int c = 0; c < 3; ++c) mm[c] = m[c] * mag;
    cross3(mm[0], mm[1], mm[2], h[0], h[1], h[2], x[0], x[1], x[2]);
    for (int c = 0; c < 3; ++c) d[c] = scale11 * (x[c] + (mm[c] - meq * htot[c]) * scale2 * ab) + eta[c];
    if (corr)
      for (int c = 0; c < 3; ++c) d[c] = 0.5 * (d[c] + d1[c]);
    cross3(m[0], m[1], m[2], h[0], h[1], h[2], t[0], t[1], t[2]);
    o.tq2 = t[0] * t[0] + t[1] * t[1] + t[2] * t[2];
  }
  for (int c = 0; c < 3; ++c) o.d[c] = d[c];
  o.d2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
  double w[3];
  for (int c = 0; c < 3; ++c) w[c] = mc[c] * magc + d[c];
  const double e = sqrt(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]);
  if (e > 0.0) {
    for (int c = 0; c < 3; ++c) o.m[c] = w[c] / e;
    o.mag = e;
  } else {
    for (int c = 0; c < 3; ++c) o.m[c] = -mc[c];
    o.mag = 0.0;
  }
  return o;
}

// One grain of push_zhang (llg.f90:410-703): the Heun branch (:633-700) or
// the semi-implicit |type| = 2 branch (:428-510), arguments as mt_step.  The
// thermal field joins the precession with the variance scale2 meq/(|H| |m|)
// (no separate eta).
static __device__ __noinline__ LlbStep zhang_step(bool boris, bool first, bool corr, const double* mc, double magc, const double* mpr,
                         double magp, const double* h, const double* ht, const double* d1, double ab, double lam0,
                         const LlbDev& P, double T, double gamma, double dt, double dt0) {
  LlbStep o;
  const double sp = P.spin;
  const double lam = P.meq_bs ? lam0 : lam0 * (sp + 1.0) / sp;
  double y = kGmubKb * sp / T;
  const double scale1 = -0.5 * gamma * dt;
  const double sq = sqrt(dt0);
  double m[3], mag, htot[3], mhtot, d[3], t[3];
  auto tot = [&](const double* v, double mg) {
    for (int c = 0; c < 3; ++c) htot[c] = h[c] + lam * mg * v[c];
    mhtot = sqrt(htot[0] * htot[0] + htot[1] * htot[1] + htot[2] * htot[2]);
    if (mhtot != 0.0)
      for (int c = 0; c < 3; ++c) htot[c] /= mhtot;
  };
  auto meq_of = [&](double x) { return P.meq_bs ? mt_bs(x, sp) : llb_lv(x); };
  auto dmeq_of = [&](double x) { return P.meq_bs ? mt_dbs(x, sp) : llb_dlv(x); };
  if (boris) {
    for (int c = 0; c < 3; ++c) m[c] = first ? mc[c] : mpr[c];
    mag = first ? magc : magp;
    tot(m, mag);
    double meq = meq_of(y * mhtot);
    double scale2 = P.garanin_tau ? 2.0 * (meq / (y * mhtot * dmeq_of(y * mhtot) + 1e-80)) / y : lam;
    // hthm sqrt(|scale2 meq / (|H| |m| dt0)|), hthm = ht sqrt(dt0)
    const double fth = sqrt(fabs(scale2 * meq / (mhtot * mag * dt0 + 1e-80))) * sq;
    scale2 = ab * scale2;
    for (int c = 0; c < 3; ++c) m[c] = mc[c];
    mag = magc;
    double hb[3], w[3], x[3];
    for (int c = 0; c < 3; ++c) hb[c] = h[c] + ht[c] * fth;
    cross3(m[0], m[1], m[2], hb[0], hb[1], hb[2], t[0], t[1], t[2]);
    o.tq2 = t[0] * t[0] + t[1] * t[1] + t[2] * t[2];
    const double dec = 1.0 - exp(scale1 * scale2);
    for (int c = 0; c < 3; ++c) d[c] = (meq * htot[c] - mag * m[c]) * dec;
    for (int c = 0; c < 3; ++c) w[c] = mag * m[c] + d[c];
    cross3(w[0], w[1], w[2], hb[0], hb[1], hb[2], x[0], x[1], x[2]);
    for (int c = 0; c < 3; ++c) d[c] += 2.0 * scale1 * x[c];  // :472
    for (int c = 0; c < 3; ++c) w[c] = mag * m[c] + d[c];
    tot(w, 1.0);
    meq = meq_of(y * mhtot);
    scale2 = ab * (P.garanin_tau ? 2.0 * (meq / (y * mhtot * dmeq_of(y * mhtot) + 1e-80)) / y : lam);
    const double dec2 = 1.0 - exp(scale1 * scale2);
    for (int c = 0; c < 3; ++c) d[c] = d[c] + (meq * htot[c] - w[c]) * dec2;  // :500
  } else {
    const double scale11 = 2.0 * scale1;
    for (int c = 0; c < 3; ++c) m[c] = mc[c];
    mag = magc;
    if (corr) {  // :635-638 (y becomes |h| when |m| <= 0, as there)
      for (int c = 0; c < 3; ++c) m[c] = mpr[c];
      mag = magp;
      if (mag <= 0.0) {
        mag = 0.0;
        y = sqrt(h[0] * h[0] + h[1] * h[1] + h[2] * h[2]);
        if (y != 0.0)
          for (int c = 0; c < 3; ++c) m[c] = h[c] / y;
      }
    }
    tot(m, mag);
    y = y * mhtot;
    const double meq = meq_of(y);
    double scale2;
    if (P.garanin_tau) {
      y = meq / (y * dmeq_of(y) + 1e-66);
      scale2 = 2.0 * T * y / (kGmubKb * sp);
    } else {
      scale2 = lam;
    }
    y = fabs(scale2 * meq / (mhtot * mag + 1e-66));
    double hb[3], mm[3], x[3];
    for (int c = 0; c < 3; ++c) hb[c] = h[c] + ht[c] * sq * sqrt(fabs(y / dt0));
    scale2 = scale2 * ab;
    for (int c = 0; c < 3; ++c) mm[c] = m[c] * mag;
    cross3(mm[0], mm[1], mm[2], hb[0], hb[1], hb[2], x[0], x[1], x[2]);
    for (int c = 0; c < 3; ++c) d[c] = scale11 * (x[c] + (mm[c] - meq * htot[c]) * scale2);
    if (corr)
      for (int c = 0; c < 3; ++c) d[c] = 0.5 * (d[c] + d1[c]);
    cross3(m[0], m[1], m[2], hb[0], hb[1], hb[2], t[0], t[1], t[2]);
    o.tq2 = t[0] * t[0] + t[1] * t[1] + t[2] * t[2];
  }
  for (int c = 0; c < 3; ++c) o.d[c] = d[c];
  o.d2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
  double w[3];
  for (int c = 0; c < 3; ++c) w[c] = mc[c] * magc + d[c];
  const double e = sqrt(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]);
  if (e > 0.0) {
    for (int c = 0; c < 3; ++c) o.m[c] = w[c] / e;
    o.mag = e;
  } else {
    for (int c = 0; c < 3; ++c) o.m[c] = -mc[c];
    o.mag = 0.0;
  }
  return o;
}

// shared memory of a row block's table weights (grid columns, then the
// block's rows; at most 8 rows per block)
MRM_HD int field_table_bytes(int nx) { return (nx + 8) * (int)sizeof(TabW); }

// shared memory of a row block's head-field table (one (h_x, h_z) per grid column)
template <typename R>
MRM_HD int head_table_bytes(int nx) {
  return (nx * (int)sizeof(Cx<R>) + 15) & ~15;
}

// CSR neighbour sum  sum_j c_j m_j  (field.f90:350-363 / :326-348)
// The FP32 stepping arithmetic uses the hardware reciprocal and reciprocal
// square root (a couple of ulp) where FP64 runs keep the correctly rounded forms.
MRM_D float fast_div(float a, float b) { return __fdividef(a, b); }
MRM_D double fast_div(double a, double b) { return a / b; }
MRM_D float fast_rsqrt(float x) { return rsqrtf(x); }
MRM_D double fast_rsqrt(double x) { return 1.0 / sqrt(x); }

template <typename R>
MRM_D void csr_sum(const int* __restrict__ idx, const int* __restrict__ nbr,
                   const R* __restrict__ cf, const V4<R>* __restrict__ mb, int n, R& hx, R& hy,
                   R& hz) {
  const int q0 = __ldg(idx + n), q1 = __ldg(idx + n + 1);
  for (int q = q0; q < q1; ++q) {
    const int j = __ldg(nbr + q);
    const R c = __ldg(cf + q);
    const V4<R> mj = mb[j];
    hx += c * mj.x;
    hy += c * mj.y;
    hz += c * mj.z;
  }
}

// csr_sum with each neighbour's coefficient times scale(j, m_j) (temperature
// scaling: the neighbour's ms_scale at this evaluation)
template <typename R, class SCALE>
MRM_D void csr_sum_scaled(const int* __restrict__ idx, const int* __restrict__ nbr, const R* __restrict__ cf,
                          const V4<R>* __restrict__ mb, int n, const SCALE& scale, R& hx, R& hy, R& hz) {
  const int q0 = __ldg(idx + n), q1 = __ldg(idx + n + 1);
  for (int q = q0; q < q1; ++q) {
    const int j = __ldg(nbr + q);
    const V4<R> mj = mb[j];
    const R c = (R)((double)__ldg(cf + q) * scale(j, mj));
    hx += c * mj.x;
    hy += c * mj.y;
    hz += c * mj.z;
  }
}

// stats record slots (sums except the two maxima)
constexpr int kSlotV = 0, kSlotM = 1, kSlotM2 = 4, kSlotH = 7, kSlotWM = 10, kSlotW = 13,
              kSlotNup = 14, kSlotMaxTq = 15, kSlotMaxD2 = 16, kSlotMmag = 17, kSlotE = 18, kSlotVA = 19;
MRM_HD constexpr bool slot_is_max(int s) { return s == kSlotMaxTq || s == kSlotMaxD2; }

MRM_D void block_reduce_record(double* rec, double* sred /* [32][kNPart] */, double* out) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int s = 0; s < kNPart; ++s) {
    double v = rec[s];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      double w = __shfl_xor_sync(0xffffffffu, v, o);
      v = slot_is_max(s) ? fmax(v, w) : v + w;
    }
    if (lane == 0) sred[warp * kNPart + s] = v;
  }
  __syncthreads();
  if (threadIdx.x < kNPart) {
    const int s = threadIdx.x;
    double v = sred[s];
    for (int w = 1; w < nw; ++w) v = slot_is_max(s) ? fmax(v, sred[w * kNPart + s]) : v + sred[w * kNPart + s];
    out[s] = v;
  }
}

template <int STAGE, bool STATS>
__host__ __device__ constexpr int stats_slots() { return ((STAGE == kCorr || STAGE == kPred) && STATS) ? 32 * kNPart : 1; }

// ---------------- grain-row staging plan ----------------
//
// The row kernel copies the grain rows it works on into shared memory with
// bulk copies issued by one thread: static rows (parameters, lattice
// coefficients) before the dependency wait, the state rows after it.  The
// field's rows carry a one-row halo on each side for the lattice stencil.
// Everything is staged when it fits in the launch's staging capacity,
// otherwise the block reads the same arrays from global memory.
struct RowStage {
  int pb, pa, xst, ucol, lcol;  // static rows (byte offsets, -1: not used)
  int mf, m0, dm, ht, vu, vl;   // dynamic rows
  int halo;                     // rows of halo on each side of mf (0 or 1)
  int bytes;                    // total
};

// Loads from shared memory through a generic pointer that is known to point
// there (ld.shared: the compiler need not prove the address space).
MRM_D V4<float> lds_v4(const V4<float>* p) {
  V4<float> v;
  asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];"
               : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
               : "r"(smem_u32(p)));
  return v;
}
MRM_D V4<double> lds_v4(const V4<double>* p) {
  V4<double> v;
  asm volatile("ld.shared.v2.f64 {%0, %1}, [%2];" : "=d"(v.x), "=d"(v.y) : "r"(smem_u32(p)));
  asm volatile("ld.shared.v2.f64 {%0, %1}, [%2 + 16];" : "=d"(v.z), "=d"(v.w) : "r"(smem_u32(p)));
  return v;
}
MRM_D float lds_r(const float* p) {
  float v;
  asm volatile("ld.shared.f32 %0, [%1];" : "=f"(v) : "r"(smem_u32(p)));
  return v;
}
MRM_D double lds_r(const double* p) {
  double v;
  asm volatile("ld.shared.f64 %0, [%1];" : "=d"(v) : "r"(smem_u32(p)));
  return v;
}

// compile-time value selecting a generic lambda's instantiation
template <int V>
struct IntC {
  static constexpr int value = V;
};

// R-valued rows can be staged when a row is a whole number of 16-byte units
template <typename R>
MRM_HD bool rows_16b(int nx) { return ((long long)nx * (long long)sizeof(R)) % 16 == 0; }

template <typename R>
MRM_HD RowStage row_stage_plan(int stage, int nx, int nrows, bool stencil, bool ucol, bool lcol,
                               bool thermal) {
  RowStage p{-1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, 0, 0};
  const int v4row = nx * (int)sizeof(V4<R>);
  const int rrow = nx * (int)sizeof(R);
  int off = 0;
  auto take = [&](int bytes) {
    const int at = off;
    off += bytes;
    return at;
  };
  p.pb = take(nrows * v4row);
  if (stage != kInit) {
    p.pa = take(nrows * v4row);
    if (stencil) p.xst = take(nrows * v4row);
    if (ucol && rows_16b<R>(nx)) p.ucol = take(nrows * rrow);
    if (lcol && rows_16b<R>(nx)) p.lcol = take(nrows * rrow);
  }
  p.halo = (stage != kInit && stencil) ? 1 : 0;
  p.mf = take((nrows + 2 * p.halo) * v4row);
  if (stage == kCorr) {
    p.m0 = take(nrows * v4row);
    p.dm = take(nrows * v4row);
    if (thermal) p.ht = take(nrows * v4row);
  }
  if (stage != kInit) {
    if (ucol) p.vu = take(nrows * v4row);
    if (lcol) p.vl = take(nrows * v4row);
  }
  p.bytes = off;
  return p;
}

// shared memory of the row kernel ahead of the grain staging area: twiddles
// and the two FFT buffers sized for RPB rows
template <typename R>
MRM_HD int row_fft_smem(int lgpx, int rpb) {
  const int M = 1 << (lgpx - 1);
  return (row_tw_count(lgpx) + 2 * rpb * 3 * seq_stride(M)) * (int)sizeof(Cx<R>);
}

// Register row transforms of a block's sequences (FP32 runs, 16 <= M <= 1024
// points): sequence s (= 3 row + component) at s * cs in each buffer, one group
// of M/8 threads per sequence, group g taking sequences g, g + G, ...
// (G = BLOCK / (M/8)).  The choice depends on M alone, so every row shape
// computes the same transform.
MRM_HD constexpr bool rrow_len_ok(int lgM) { return lgM >= 4 && lgM <= 10; }

template <int LGM, int BLOCK>
MRM_D void rrow_inverse_block(const Cx<float>* X, Cx<float>* xb, Cx<float>* out, int cs, int nseq, int nz,
                              const Cx<float>* __restrict__ twpost, const Cx<float>* __restrict__ twpass) {
  constexpr int NT = 1 << (LGM - 3), G = BLOCK / NT;
  static_assert(G >= 1 && BLOCK % NT == 0, "whole groups per block");
  static_assert(NT <= 32 || G <= 4, "named barriers 1..4");
  const int g = threadIdx.x / NT, t = threadIdx.x % NT;
#pragma unroll 1
  for (int s0 = 0; s0 < nseq; s0 += G) {
    const int s = s0 + g;
    if (s < nseq) rrow_inverse<LGM>(X + s * cs, xb + s * cs, out + s * cs, t, g, nz, twpost, twpass);
  }
}

// POST(s, t, nt, Y): the group's spectrum post-processing of sequence s from
// its natural-order Y (the group is synchronised before and after the call's
// reads through the next sequence's barriers; Y is not written again).
template <int LGM, bool HALF, int BLOCK, class POST>
MRM_D void rrow_forward_block(Cx<float>* in, Cx<float>* xb, int cs, int nseq, const Cx<float>* __restrict__ twpass,
                              const POST& post) {
  constexpr int NT = 1 << (LGM - 3), G = BLOCK / NT;
  static_assert(G >= 1 && BLOCK % NT == 0, "whole groups per block");
  static_assert(NT <= 32 || G <= 4, "named barriers 1..4");
  const int g = threadIdx.x / NT, t = threadIdx.x % NT;
#pragma unroll 1
  for (int s0 = 0; s0 < nseq; s0 += G) {
    const int s = s0 + g;
    if (s < nseq) {
      rrow_forward<LGM, HALF>(in + s * cs, xb + s * cs, in + s * cs, t, g, twpass);
      post(s, t, NT, in + s * cs);
    }
  }
}

template <int BLOCK, int LGMAX>
MRM_D void rrow_inverse_any(int lgM, const Cx<float>* X, Cx<float>* xb, Cx<float>* out, int cs, int nseq, int nz,
                            const Cx<float>* twpost, const Cx<float>* twpass) {
  switch (lgM) {
    case 4: rrow_inverse_block<4, BLOCK>(X, xb, out, cs, nseq, nz, twpost, twpass); break;
    case 5: rrow_inverse_block<5, BLOCK>(X, xb, out, cs, nseq, nz, twpost, twpass); break;
    case 6: rrow_inverse_block<6, BLOCK>(X, xb, out, cs, nseq, nz, twpost, twpass); break;
    case 7: if constexpr (LGMAX >= 8) rrow_inverse_block<7, BLOCK>(X, xb, out, cs, nseq, nz, twpost, twpass); break;
    case 8: if constexpr (LGMAX >= 9) rrow_inverse_block<8, BLOCK>(X, xb, out, cs, nseq, nz, twpost, twpass); break;
    case 9: if constexpr (LGMAX >= 10) rrow_inverse_block<9, BLOCK>(X, xb, out, cs, nseq, nz, twpost, twpass); break;
    default: if constexpr (LGMAX >= 11) rrow_inverse_block<10, BLOCK>(X, xb, out, cs, nseq, nz, twpost, twpass); break;
  }
}

template <int BLOCK, int LGMAX, bool HALF, class POST>
MRM_D void rrow_forward_any(int lgM, Cx<float>* in, Cx<float>* xb, int cs, int nseq, const Cx<float>* twpass,
                            const POST& post) {
  switch (lgM) {
    case 4: rrow_forward_block<4, HALF, BLOCK>(in, xb, cs, nseq, twpass, post); break;
    case 5: rrow_forward_block<5, HALF, BLOCK>(in, xb, cs, nseq, twpass, post); break;
    case 6: rrow_forward_block<6, HALF, BLOCK>(in, xb, cs, nseq, twpass, post); break;
    case 7: if constexpr (LGMAX >= 8) rrow_forward_block<7, HALF, BLOCK>(in, xb, cs, nseq, twpass, post); break;
    case 8: if constexpr (LGMAX >= 9) rrow_forward_block<8, HALF, BLOCK>(in, xb, cs, nseq, twpass, post); break;
    case 9: if constexpr (LGMAX >= 10) rrow_forward_block<9, HALF, BLOCK>(in, xb, cs, nseq, twpass, post); break;
    default: if constexpr (LGMAX >= 11) rrow_forward_block<10, HALF, BLOCK>(in, xb, cs, nseq, twpass, post); break;
  }
}

// Row kernel: one task = up to RPB grid rows of one layer of one run (more for
// a run of short FP32 rows, packed by the host).
//   kInit: forward row FFT of Ms*m (spectrum of the current state)
//   kPred / kCorr: inverse row FFT of H^ -> H_demag, field assembly, Heun
//                  stage, forward row FFT of Ms*m* / Ms*m_{n+1}
//   kEval: inverse row FFT and field assembly only (H_demag and h stored)
// stage_cap: bytes of dynamic shared memory available for grain staging.
// GEN: 0 Heun without a head (the general paths compiled out); 1 the general
// instantiation (semi-implicit pushes, write heads, field tables, cubic
// anisotropy, windows); 2 the general one with the LLB / MT / Zhang
// integrators and temperature profiles as well (kept apart: their FP64 code
// would share level 1's register budget and spill on its paths).
template <typename R, int STAGE, bool STATS, int RPB, int BLOCK, int MINB, int LGMAX, int GEN>
__global__ void __launch_bounds__(BLOCK, MINB) row_kernel(const RunDev<R>* __restrict__ runs,
                                                          const Task* __restrict__ tasks,
                                                          const Cx<R>* __restrict__ twg, int istep,
                                                          int flags, double* __restrict__ part,
                                                          int* __restrict__ err, int stage_cap) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ uint64_t bars[3];
  __shared__ double sred[stats_slots<STAGE, STATS>()];
  pdl_launch_dependents();
  const Task tk = tasks[blockIdx.x];
  const RunDev<R>& rd = runs[tk.x];
  if (!rd.active) return;  // host-set, constant within a captured graph
  if (rd.lgpx > LGMAX) {  // shape not compiled into this variant (the host never picks it)
    if (threadIdx.x == 0) atomicOr(err, kErrShape);
    return;
  }

  const int l = tk.y, row0 = tk.z, nrows = tk.w;
  const int nx = rd.nx, ny = rd.ny;
  // moving demag window (general kernels, one row per task): the task's row is
  // grid row wj0 + row0, its cells grid columns wi0 .. wi0 + nx - 1 of the full
  // gnx x gny grid that the per-grain arrays cover
  const bool win = GEN && rd.gnx > 0;
  if (win && nrows != 1) {
    if (threadIdx.x == 0) atomicOr(err, kErrShape);
    return;
  }
  const int gnx = win ? rd.gnx : nx, gny = win ? rd.gny : ny, wi0 = win ? rd.wi0 : 0, wj0 = win ? rd.wj0 : 0;
  const int lgpx = rd.lgpx, lgM = lgpx - 1, M = 1 << lgM, ph = M + 1;
  const int cs = seq_stride(M);  // complex stride of one sequence in shared memory
  // FP32 rows of 16..1024 complex points: the register transforms, whose
  // loops take any number of rows; a run of rows shorter than the launch's
  // longest may then have more than RPB rows per task (the host packs them
  // into the FFT buffers sized for the longest rows; not in level-2 batches)
  constexpr bool kRegRowType = sizeof(R) == sizeof(float);
  const bool regrow = kRegRowType && rrow_len_ok(lgM);
  const int rcap = (GEN < 2 && regrow && !win) ? max(RPB, nrows) : RPB;
  const int nseq = nrows * 3;
  const int ngr = nrows * nx;
  const LayerDev<R>& L = rd.L[l];
  const bool demag = rd.demag != 0;
  constexpr bool stats = (STAGE == kCorr || STAGE == kPred) && STATS;
  constexpr int NBMAX = 3 * RPB;
  const bool boris = GEN && (flags & kFlagBoris) != 0, mid = GEN && (flags & kFlagMid) != 0;

  Cx<R>* tws = reinterpret_cast<Cx<R>*>(smem_raw);  // post twiddles | pass tables
  const int ntw = row_tw_count(lgpx);
  if (nrows > rcap || (long long)(ntw + 2 * rcap * 3 * cs) * (long long)sizeof(Cx<R>) >
                          (long long)dynamic_smem_bytes()) {  // host bug: a task the buffers do not hold
    if (threadIdx.x == 0) atomicOr(err, kErrShape);
    return;
  }
  Cx<R>* bufA = tws + ntw;
  Cx<R>* bufB = bufA + rcap * 3 * cs;
  // a layer under the moving write head gets its head field per grid column in
  // a table after the FFT buffers (the host reserves it), then the staging area
  // (its byte offset; 0: no head)
  // (a tabulated field profile gets its interpolation weights there instead)
  const bool ftab = GEN && STAGE != kInit && rd.L[tk.y].tab != nullptr;
  const int htab_off = GEN && (rd.L[tk.y].func == kFuncHead || ftab)
                           ? (int)(reinterpret_cast<unsigned char*>(bufB + rcap * 3 * cs) - smem_raw)
                           : 0;
  unsigned char* stg = reinterpret_cast<unsigned char*>(bufB + rcap * 3 * cs) +
                       (ftab ? field_table_bytes(rd.nx) : htab_off ? head_table_bytes<R>(rd.nx) : 0);
  if (htab_off && (long long)(stg - smem_raw) > (long long)dynamic_smem_bytes()) {  // host bug: no room reserved
    if (threadIdx.x == 0) atomicOr(err, kErrShape);
    return;
  }
  const Cx<R>* twpost = tws;
  const Cx<R>* twpass = tws + row_tw_post(lgpx);

  const LayerDev<R>* Lu = (l > 0) ? &rd.L[l - 1] : nullptr;
  const LayerDev<R>* Ll = (l + 1 < rd.nl) ? &rd.L[l + 1] : nullptr;
  const bool stencil = L.xst != nullptr;
  const bool ucol = L.ucol && Lu, lcol = L.lcol && Ll;
  const bool thermal = (STAGE == kPred || STAGE == kCorr) && L.thermal;
  const V4<R>* __restrict__ mfield = (STAGE == kCorr) ? L.mp : L.m;
  const V4<R>* __restrict__ mother_u = Lu ? ((STAGE == kCorr) ? Lu->mp : Lu->m) : nullptr;
  const V4<R>* __restrict__ mother_l = Ll ? ((STAGE == kCorr) ? Ll->mp : Ll->m) : nullptr;
  const RowStage sp = row_stage_plan<R>(STAGE, nx, nrows, stencil, ucol, lcol, thermal);
  // staged when the plan fits both the launch's staging capacity and the
  // shared memory actually allocated behind the FFT buffers
  const bool staged = !win && sp.bytes <= stage_cap &&
                      (long long)(stg - smem_raw) + sp.bytes <= (long long)dynamic_smem_bytes();
  const int base = win ? (wj0 + row0) * gnx + wi0 : row0 * nx;
  const int v4row = nx * (int)sizeof(V4<R>);
  const int rrow = nx * (int)sizeof(R);
  const bool mapped = (STAGE != kInit) && (flags & kFlagMapped);
  const bool inverse = (STAGE != kInit) && demag && !mapped;

  // bulk copy with the self-checks of the MRM_CHECKS build (source offset
  // within its array, destination within the dynamic shared memory, 16-byte
  // alignment)
  auto copy = [&](uint64_t* bar, void* dst, const void* src, long long src_off_bytes, long long src_len_bytes,
                  int bytes, int code) {
#ifdef MRM_CHECKS
    uint32_t dyn;
    asm volatile("mov.u32 %0, %%dynamic_smem_size;" : "=r"(dyn));
    const long long doff = (long long)smem_u32(dst) - (long long)smem_u32(smem_raw);
    if (!MRM_CHECK(src_off_bytes >= 0 && src_off_bytes + bytes <= src_len_bytes, code, src_off_bytes)) return;
    if (!MRM_CHECK(doff >= 0 && doff + bytes <= (long long)dyn, code + 1, doff)) return;
    if (!MRM_CHECK(((((uintptr_t)src) | (uintptr_t)doff | (uintptr_t)bytes) & 15) == 0, code + 2,
                   (long long)(uintptr_t)src))
      return;
#endif
    bulk_copy(bar, dst, src, (uint32_t)bytes);
  };
  const long long nlay = (long long)gnx * gny;  // grains per layer
  const long long v4b = (long long)sizeof(V4<R>), rb = (long long)sizeof(R), cb = (long long)sizeof(Cx<R>);
  MRM_CHECK(l >= 0 && l < rd.nl && row0 >= 0 && nrows >= 1 && row0 + nrows <= ny, 900, row0);

  // ---------------- static inputs: twiddles, parameter rows ----------------
  if (threadIdx.x == 0) {
    mbar_init(&bars[0], 1);
    mbar_init(&bars[1], 1);
    mbar_init(&bars[2], 1);
    mbar_fence_init();
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    if (demag)
      copy(&bars[0], tws, twg + rd.tw_row, rd.tw_row * cb, (long long)tw_table_size() * cb, ntw * (int)cb, 100);
    if (staged) {
      copy(&bars[0], stg + sp.pb, L.pb + base, base * v4b, nlay * v4b, nrows * v4row, 110);
      if (sp.pa >= 0) copy(&bars[0], stg + sp.pa, L.pa + base, base * v4b, nlay * v4b, nrows * v4row, 120);
      if (sp.xst >= 0) copy(&bars[0], stg + sp.xst, L.xst + base, base * v4b, nlay * v4b, nrows * v4row, 130);
      if (sp.ucol >= 0) copy(&bars[0], stg + sp.ucol, L.ucol + base, base * rb, nlay * rb, nrows * rrow, 140);
      if (sp.lcol >= 0) copy(&bars[0], stg + sp.lcol, L.lcol + base, base * rb, nlay * rb, nrows * rrow, 150);
    } else if (!win && v4row % 16 == 0) {
      // rows read at use: their parameter rows start for L2 now, and arrive
      // while the inverse row transforms run
      bulk_prefetch_l2(L.pb + base, (uint32_t)(nrows * v4row));
      if (STAGE != kInit) {
        bulk_prefetch_l2(L.pa + base, (uint32_t)(nrows * v4row));
        if (stencil) bulk_prefetch_l2(L.xst + base, (uint32_t)(nrows * v4row));
      }
    }
    mbar_arrive(&bars[0]);
  }

  // ---------------- wait for the previous kernel's results ----------------
  pdl_wait();
  const long long step = *reinterpret_cast<const volatile long long*>(&rd.step) + istep;
  const bool run_it = (flags & kFlagForce) || step_due(rd, step);
  if (threadIdx.x == 0) {
    if (run_it && inverse)
      for (int s = 0; s < nseq; ++s) {
        const int row = s / 3, comp = s - 3 * row;
        const long long off = ((long long)(l * 3 + comp) * ny + row0 + row) * rd.phs;
        copy(&bars[1], bufB + s * cs, rd.spech + off, off * cb, (long long)rd.nl * 3 * ny * rd.phs * cb,
             rd.phs * (int)cb, 200);
      }
    mbar_arrive(&bars[1]);
    if (run_it && !staged && !win && v4row % 16 == 0) {
      // the state rows of this stage (with the lattice neighbours' rows) for L2
      bulk_prefetch_l2(mfield + base, (uint32_t)(nrows * v4row));
      if (STAGE != kInit && stencil) {
        const int jm = row0 == 0 ? ny - 1 : row0 - 1, jp = row0 + nrows == ny ? 0 : row0 + nrows;
        bulk_prefetch_l2(mfield + (size_t)jm * nx, (uint32_t)v4row);
        bulk_prefetch_l2(mfield + (size_t)jp * nx, (uint32_t)v4row);
      }
      if (STAGE == kCorr) {
        bulk_prefetch_l2(L.m + base, (uint32_t)(nrows * v4row));
        bulk_prefetch_l2(L.dm + base, (uint32_t)(nrows * v4row));
        if (thermal) bulk_prefetch_l2(L.ht + base, (uint32_t)(nrows * v4row));
      }
    }
    if (run_it && staged) {
      if (sp.halo) {
        const int jm = row0 == 0 ? ny - 1 : row0 - 1, jp = row0 + nrows == ny ? 0 : row0 + nrows;
        copy(&bars[2], stg + sp.mf, mfield + (size_t)jm * nx, (long long)jm * nx * v4b, nlay * v4b, v4row, 210);
        copy(&bars[2], stg + sp.mf + v4row, mfield + base, base * v4b, nlay * v4b, nrows * v4row, 220);
        copy(&bars[2], stg + sp.mf + (nrows + 1) * v4row, mfield + (size_t)jp * nx, (long long)jp * nx * v4b,
             nlay * v4b, v4row, 230);
      } else {
        copy(&bars[2], stg + sp.mf, mfield + base, base * v4b, nlay * v4b, nrows * v4row, 240);
      }
      if (sp.m0 >= 0) copy(&bars[2], stg + sp.m0, L.m + base, base * v4b, nlay * v4b, nrows * v4row, 250);
      if (sp.dm >= 0) copy(&bars[2], stg + sp.dm, L.dm + base, base * v4b, nlay * v4b, nrows * v4row, 260);
      if (sp.ht >= 0) copy(&bars[2], stg + sp.ht, L.ht + base, base * v4b, nlay * v4b, nrows * v4row, 270);
      if (sp.vu >= 0) copy(&bars[2], stg + sp.vu, mother_u + base, base * v4b, nlay * v4b, nrows * v4row, 280);
      if (sp.vl >= 0) copy(&bars[2], stg + sp.vl, mother_l + base, base * v4b, nlay * v4b, nrows * v4row, 290);
    }
    if (flags & kFlagProbeTimeout) mbar_expect_tx(&bars[2], 16);  // bytes that never come
    mbar_arrive(&bars[2]);
  }
  // every barrier completes (an unused one on the arrive alone); a block whose
  // copies do not land in time raises the error flag and leaves
  auto leave_on_timeout = [&](bool ok) -> bool {
    if (!__syncthreads_or(!ok)) return false;
    if (threadIdx.x == 0) atomicOr(err, kErrBarrierTimeout);
    for (int b = 0; b < 3; ++b) mbar_wait(&bars[b], 0);
    return true;
  };
  if (!run_it) {
    // nothing to do at this step: let the static copies land before leaving
    leave_on_timeout(mbar_wait(&bars[0], 0) & mbar_wait(&bars[1], 0) & mbar_wait(&bars[2], 0));
    return;
  }

  // ---------------- inverse row transform: H^ rows -> H_demag ----------------
  Cx<R>* Z = bufA;  // after the inverse: z[n] = x[2n] + i x[2n+1] per sequence
  if (inverse && regrow) {
    if (leave_on_timeout(mbar_wait(&bars[0], 0) & mbar_wait(&bars[1], 0))) return;
    if constexpr (kRegRowType)
      rrow_inverse_any<BLOCK, LGMAX>(lgM, bufB, bufA, bufB, cs, nseq, (nx + 1) >> 1, twpost, twpass);
    __syncthreads();
    Z = bufB;
  } else if (inverse) {
    if (leave_on_timeout(mbar_wait(&bars[0], 0) & mbar_wait(&bars[1], 0))) return;
    const int tot = nseq * M;
    for (int idx = threadIdx.x; idx < tot; idx += BLOCK) {
      const int s = idx >> lgM, k = idx & (M - 1);
      const Cx<R>* X = bufB + s * cs;
      Cx<R> a = X[k], b = X[M - k];
      if (k == 0) { a.y = 0; b.y = 0; }  // self-conjugate bins: imaginary parts ignored (c2r)
      const Cx<R> e = cadd(a, cconj(b));
      const Cx<R> o = csub(a, cconj(b));
      const Cx<R> w = cconj(twpost[k]);  // e^{+2 pi i k / px}
      bufA[s * cs + k] = cadd(e, cmul_i(cmul(o, w), (R)1));
    }
    __syncthreads();
    Z = block_fft_c<R, +1, NBMAX, BLOCK, LGMAX - 1>(bufA, bufB, lgM, nseq, twpass);
  }
  Cx<R>* W = (Z == bufA) ? bufB : bufA;  // real outputs of this stage (forward input)
  const R* hdr = reinterpret_cast<const R*>(Z);
  R* outr = reinterpret_cast<R*>(W);
  const int rs = 2 * cs;  // real stride of one sequence
  if (leave_on_timeout(mbar_wait(&bars[0], 0) & mbar_wait(&bars[2], 0))) return;

  // ---------------- per-grain field + integrator stage ----------------
  const double t_now = rd.t_base + (double)(step - rd.step_base) * rd.dt;
  const double t_stage = (STAGE == kCorr) ? t_now + (mid ? 0.5 * rd.dt : rd.dt) : t_now;
  const double sc = ramp(L, t_stage);
  const double tps = (GEN == 2 && L.tprof) ? L.tprof->dtemp * temp_scale(*L.tprof, t_stage) : 0.0;
  // a layer's field is its uniform direction or its tabulated profile, scaled
  double hd3[3] = {L.hdir[0], L.hdir[1], L.hdir[2]};
  if (L.func == kFuncRot) rot_dir(L.fgamma, L.phase, t_stage, hd3);
  const R hax = ftab ? (R)0 : (R)(sc * hd3[0]), hay = ftab ? (R)0 : (R)(sc * hd3[1]),
          haz = ftab ? (R)0 : (R)(sc * hd3[2]);
  const R dt = (R)rd.dt;
  const R gamma = (R)L.gamma;
  const R tfac = thermal ? (R)sqrt(L.temperature / rd.dt) : (R)0;  // sqrt(T/dt)
  // (a demag-only evaluation leaves L.hf alone: it holds the last stepping
  // stage's field, which a retried adaptive step reads)
  const bool store_field = (flags & kFlagStoreField) || (STAGE == kEval && !(flags & kFlagDemagOnly));
  // Write head: its field depends on the column and the time only.  The
  // stepping stages add it to the block's demag values in shared memory (zero
  // when demag is off), so their per-grain loop is the same with or without a
  // head; the evaluation stage keeps demag apart and reads a per-column table.
  const bool fold_head = (STAGE == kPred || STAGE == kCorr) && htab_off && !ftab;
  const bool use_hdr = !mapped && (demag || fold_head);
  if (ftab) {
    // set (applied.f90:896-902) for the grid columns and the block's rows
    TabW* tw = reinterpret_cast<TabW*>(smem_raw + htab_off);
    const TabDev& T = *L.tab;
    const double ox = T.ox + T.vx * (t_stage - T.t0) - T.rx;
    const double oy = T.oy + T.vy * (t_stage - T.t0) - T.ry;
    for (int c = threadIdx.x; c < nx + nrows; c += BLOCK)
      tw[c] = c < nx ? tab_weight(T.pos, T.nx, ((double)(wi0 + c) + 0.5) * T.dx - ox)
                     : tab_weight(T.pos + T.nx, T.ny, ((double)(wj0 + row0 + c - nx) + 0.5) * T.dy - oy);
    __syncthreads();
  } else if (STAGE != kInit && htab_off) {
    double xh, pol;
    head_state(L, t_stage, &xh, &pol);
    R* hw = reinterpret_cast<R*>(Z);
    for (int c = threadIdx.x; c < nx; c += BLOCK) {
      R khx, khz;
      karlqvist<R>((R)(((double)(wi0 + c) + 0.5) * L.hd_dx - xh), (R)L.hd_gap, (R)L.hd_z, (R)(pol * L.hd_hg), khx,
                   khz);
      if (STAGE == kEval) {
        reinterpret_cast<Cx<R>*>(smem_raw + htab_off)[c] = Cx<R>{khx, khz};
      } else {
        for (int r = 0; r < nrows; ++r) {
          R* w = hw + (size_t)(r * 3) * rs + c;
          if (demag) {
            w[0] += khx;
            w[2 * rs] += khz;
          } else {
            w[0] = khx;
            w[rs] = (R)0;
            w[2 * rs] = khz;
          }
        }
      }
    }
    __syncthreads();
  }
  const bool pow2x = (nx & (nx - 1)) == 0;
  const int lgnx = __ffs(nx) - 1;
  const bool cubic = GEN && L.cax != nullptr;

  double rec[stats ? kNPart : 1];
#pragma unroll
  for (int s = 0; s < (stats ? kNPart : 1); ++s) rec[s] = 0.0;

  // The per-grain loop, compiled twice in the fast kernels without
  // reductions: staged (the
  // block's rows in shared memory: every row view is a shared-memory address
  // known as such, and no global fallback is loaded) and unstaged.  Staged, the plan
  // holds every row the loop reads: pa and the row field outside kInit, xst
  // with the stencil, m0 and dm in kCorr, ht in kCorr with a thermal field,
  // vu / vl with the columnar couplings (row_stage_plan); ucol / lcol rows
  // are staged when a row is a whole number of 16-byte units.
  auto grain_loop = [&](auto mode_c) {
  // mode 1: staged, 0: unstaged, 2: decided at run time (the general kernels,
  // whose larger loop bodies would spill more as two copies)
  constexpr int MODE = decltype(mode_c)::value;
  const bool ST = MODE == 2 ? staged : MODE == 1;
  auto srow = [&](int off) { return reinterpret_cast<const V4<R>*>(stg + off); };
  const V4<R>* PB = ST ? srow(sp.pb) : L.pb + base;
  const V4<R>* PA = ST ? srow(sp.pa) : L.pa + base;
  const V4<R>* XS = ST ? srow(sp.xst) : L.xst + base;
  const R* UC = (ST && sp.ucol >= 0) ? reinterpret_cast<const R*>(stg + sp.ucol) : (ucol ? L.ucol + base : nullptr);
  const R* LC = (ST && sp.lcol >= 0) ? reinterpret_cast<const R*>(stg + sp.lcol) : (lcol ? L.lcol + base : nullptr);
  const V4<R>* MF = ST ? srow(sp.mf) + sp.halo * nx : mfield + base;
  const V4<R>* M0 = ST ? srow(sp.m0) : L.m + base;
  const V4<R>* DM = ST ? srow(sp.dm) : L.dm + base;
  const V4<R>* HT = ST ? srow(sp.ht) : L.ht + base;
  const V4<R>* VU = ST ? srow(sp.vu) : (ucol ? mother_u + base : nullptr);
  const V4<R>* VL = ST ? srow(sp.vl) : (lcol ? mother_l + base : nullptr);
  if (ST) {
    MRM_CHECK(STAGE == kInit || sp.pa >= 0, 950, sp.pa);
    MRM_CHECK(STAGE == kInit || !stencil || sp.xst >= 0, 951, sp.xst);
    MRM_CHECK(STAGE != kCorr || (sp.m0 >= 0 && sp.dm >= 0 && (!thermal || sp.ht >= 0)), 952, sp.m0);
    MRM_CHECK(STAGE == kInit || ((!ucol || sp.vu >= 0) && (!lcol || sp.vl >= 0)), 953, sp.vu);
  }
  // field row rr in [-1, nrows] (lattice neighbours wrap periodically)
  auto mf_row = [&](int rr) -> const V4<R>* {
    if (ST) return MF + rr * nx;
    if (win) {
      int j = wj0 + row0 + rr;
      j = j < 0 ? j + gny : (j >= gny ? j - gny : j);
      return mfield + (size_t)j * gnx;
    }
    int j = row0 + rr;
    j = j < 0 ? j + ny : (j >= ny ? j - ny : j);
    return mfield + (size_t)j * nx;
  };
  // row-view loads: explicit shared-memory loads when staged
  auto at4 = [&](const V4<R>* p, int i) -> V4<R> {
    if constexpr (MODE == 1) return lds_v4(p + i);
    else return p[i];
  };
  auto at1 = [&](const R* p, int i) -> R {
    if constexpr (MODE == 1) return lds_r(p + i);
    else return p[i];
  };
  for (int idx = threadIdx.x; idx < ngr; idx += BLOCK) {
    const int rr = pow2x ? (idx >> lgnx) : idx / nx;
    const int i = idx - rr * nx;
    const int q = idx;                // index within the task's rows
    const int n = base + idx;         // grain index within the layer
    V4<R> pb = at4(PB, q);
    // (temperature scaling, level 2: the grain's grid cell)
    const int gi = wi0 + i, gj = wj0 + row0 + rr;
    if (STAGE == kInit) {
      const V4<R> mf = at4(MF, q);
      R ms0 = pb.x;  // Ms * ms_scale
      if constexpr (GEN == 2)
        if (L.tsc) ms0 = (R)((double)pb.x * tsc_ms(*L.tsc, n, layer_temp(L, t_stage, gi, gj), (double)mf.w));
      outr[(rr * 3 + 0) * rs + i] = ms0 * mf.x;
      outr[(rr * 3 + 1) * rs + i] = ms0 * mf.y;
      outr[(rr * 3 + 2) * rs + i] = ms0 * mf.z;
      continue;
    }
    const V4<R> mf = at4(MF, q);
    V4<R> pa = at4(PA, q);
    // Temperature scaling (find_temp_scaling at this stage's field evaluation,
    // temp_scaling.f90:365-430): the grain's Ms, alpha and Hk scales replace
    // the unit scales the layer was uploaded with (in Ms * ms_scale, Hk *
    // hk_scale, alpha * alpha_scale, and the thermal variance's
    // alpha_scale / max(floor_ms, ms_scale), field.f90:418-421)
    double sc_ms = 1.0, sc_al = 1.0;
    if constexpr (GEN == 2) {
      if (L.tsc) {
        const TscDev& S = *L.tsc;
        const double Tn = layer_temp(L, t_stage, gi, gj);
        sc_ms = tsc_ms(S, n, Tn, (double)mf.w);
        sc_al = tsc_alpha(S, n, Tn);
        const double sh = tsc_hk(S, n, Tn);
        pb.x = (R)((double)pb.x * sc_ms);
        pb.y = (R)((double)pb.y * sh);
        pa.w = (R)((double)pa.w * sh);
        pb.z = (R)((double)pb.z * sc_al);
        pb.w = sc_ms > 0.0 ? (R)((double)pb.w * sqrt(sc_al * fmax(S.floor_ms, 1.0) / fmax(S.floor_ms, sc_ms)))
                           : (R)0;
      }
    }
    const R mse = pb.x;  // Ms * ms_scale
    R hdx = 0, hdy = 0, hdz = 0;
    if (mapped) {
      const V4<R> g = L.cgrain ? L.hdm[n] : L.hd[n];
      hdx = g.x;
      hdy = g.y;
      hdz = g.z;
    } else if (use_hdr) {
      hdx = at1(hdr, (rr * 3 + 0) * rs + i);
      hdy = at1(hdr, (rr * 3 + 1) * rs + i);
      hdz = at1(hdr, (rr * 3 + 2) * rs + i);
    }
    // applied field of this grain: the uniform part (plus the write head's in
    // the evaluation stage; the stepping stages carry it in hdx, hdz)
    R apx = hax, apy = hay, apz = haz;
    if (ftab) {
      // the profile at the cell; a grain of several cells takes the average
      // over its cells that the gather kernel formed (get_applied,
      // field.f90:546-560)
      if (mapped && L.cgrain) {
        const V4<R> a = L.hapm[n];
        apx += a.x;
        apy += a.y;
        apz += a.z;
      } else if (!(STAGE == kEval && (flags & kFlagDemagOnly))) {
        const TabW* tw = reinterpret_cast<const TabW*>(smem_raw + htab_off);
        double vx, vy, vz;
        tab_value(L.tab->v, L.tab->nx, tw[i], tw[nx + rr], sc, vx, vy, vz);
        apx += (R)vx;
        apy += (R)vy;
        apz += (R)vz;
      }
    } else if (STAGE == kEval) {
      if (htab_off) {
        const Cx<R> kh = reinterpret_cast<const Cx<R>*>(smem_raw + htab_off)[i];
        apx += kh.x;
        apz += kh.y;
      }
    }
    // h = h_app + h_demag + H_uni + H_ex (+ interlayer)   (field.f90:201,211-220)
    R hx = apx + hdx, hy = apy + hdy, hz = apz + hdz;
    R e_k;
    if (GEN && cubic) {
      // get_cubic_hk (field.f90:377-395): a_i = m . e_i,
      // h = -sum_i e_i a_i (K1 (a_j^2 + a_k^2) + K2 a_j^2 a_k^2) with K = pa.w, pb.y
      // (hk_scale folded in); the energy keeps the reference's factors (:392-394)
      const V4<R> c1 = L.cax[3 * n], c2 = L.cax[3 * n + 1], c3 = L.cax[3 * n + 2];
      const R a1 = c1.x * mf.x + c1.y * mf.y + c1.z * mf.z;
      const R a2 = c2.x * mf.x + c2.y * mf.y + c2.z * mf.z;
      const R a3 = c3.x * mf.x + c3.y * mf.y + c3.z * mf.z;
      const R s1 = a1 * a1, s2 = a2 * a2, s3 = a3 * a3;
      const R k1 = pa.w, k2 = pb.y;
      const R d1 = a1 * (k1 * (s2 + s3) + k2 * s2 * s3);
      const R d2 = a2 * (k1 * (s1 + s3) + k2 * s1 * s3);
      const R d3 = a3 * (k1 * (s1 + s2) + k2 * s1 * s2);
      hx -= c1.x * d1 + c2.x * d2 + c3.x * d3;
      hy -= c1.y * d1 + c2.y * d2 + c3.y * d3;
      hz -= c1.z * d1 + c2.z * d2 + c3.z * d3;
      e_k = (R)0.5 * (k1 * (s1 * s2 + s1 * s3 + s2 * s3) + k2 * s1 * s2 * s3) * c1.w * mse;
    } else {
      // get_uni_hk (field.f90:366-375); pa.w = Hk1*hk_scale, pb.y = Hk2*hk_scale
      const R hks = mf.x * pa.x + mf.y * pa.y + mf.z * pa.z;
      const R yy = (R)1 - hks * hks;
      const R f = hks * (pa.w + pb.y * yy);
      hx += f * pa.x;
      hy += f * pa.y;
      hz += f * pa.z;
      e_k = (R)0.5 * yy * (pa.w + (R)0.5 * pb.y * yy) * mse;
    }
    R ex = 0, ey = 0, ez = 0;
    if (stencil) {
      V4<R> c = at4(XS, q);
      const V4<R>* rowc = mf_row(rr);
      // (in a window the neighbours are the full grid's: row pointers at the
      // full rows' starts, the grid column wi0 + i)
      const int ci = wi0 + i;
      const int im = (ci == 0 ? gnx - 1 : ci - 1), ip = (ci == gnx - 1 ? 0 : ci + 1);
      const V4<R> n0 = at4(mf_row(rr - 1), ci), n1 = at4(rowc, im), n2 = at4(rowc, ip), n3 = at4(mf_row(rr + 1), ci);
      if constexpr (GEN == 2) {
        if (L.tsc) {
          // hx(j) ms_scale(j) m(j) (get_intralayer_hx, field.f90:350-363) with the
          // neighbours' scales at this evaluation (one grain per cell, no window)
          const TscDev& S = *L.tsc;
          const int jm = gj == 0 ? gny - 1 : gj - 1, jp = gj == gny - 1 ? 0 : gj + 1;
          c.x = (R)((double)c.x * tsc_ms(S, jm * gnx + ci, layer_temp(L, t_stage, ci, jm), (double)n0.w));
          c.y = (R)((double)c.y * tsc_ms(S, gj * gnx + im, layer_temp(L, t_stage, im, gj), (double)n1.w));
          c.z = (R)((double)c.z * tsc_ms(S, gj * gnx + ip, layer_temp(L, t_stage, ip, gj), (double)n2.w));
          c.w = (R)((double)c.w * tsc_ms(S, jp * gnx + ci, layer_temp(L, t_stage, ci, jp), (double)n3.w));
        }
      }
      ex = c.x * n0.x + c.y * n1.x + c.z * n2.x + c.w * n3.x;
      ey = c.x * n0.y + c.y * n1.y + c.z * n2.y + c.w * n3.y;
      ez = c.x * n0.z + c.y * n1.z + c.z * n2.z + c.w * n3.z;
    } else if (L.xidx) {
      bool done = false;
      if constexpr (GEN == 2) {
        if (L.tsc) {
          // hx(j) ms_scale(j) m(j) with the neighbours' scales (one grain per cell: j is a cell)
          csr_sum_scaled<R>(L.xidx, L.xnbr, L.xcoef, mfield, n, [&](int j, const V4<R>& mj) {
            return tsc_ms(*L.tsc, j, layer_temp(L, t_stage, j % nx, j / nx), (double)mj.w);
          }, ex, ey, ez);
          done = true;
        }
      }
      if (!done) csr_sum<R>(L.xidx, L.xnbr, L.xcoef, mfield, n, ex, ey, ez);
    }
    R vx = 0, vy = 0, vz = 0;
    // (an interlayer partner with temperature scaling: its grains' ms_scale at
    // this evaluation, get_interlayer_hx field.f90:326-348)
    auto csr_pair = [&](const LayerDev<R>* Lo, const int* idx, const int* nbr, const R* cf, const V4<R>* mo, R& ox,
                        R& oy, R& oz) {
      if constexpr (GEN == 2) {
        if (Lo->tsc) {
          csr_sum_scaled<R>(idx, nbr, cf, mo, n, [&](int j, const V4<R>& mj) {
            return tsc_ms(*Lo->tsc, j, layer_temp(*Lo, t_stage, j % nx, j / nx), (double)mj.w);
          }, ox, oy, oz);
          return;
        }
      }
      csr_sum<R>(idx, nbr, cf, mo, n, ox, oy, oz);
    };
    auto col_scale = [&](const LayerDev<R>* Lo, R cf, R mag) -> R {
      if constexpr (GEN == 2)
        if (Lo->tsc) return (R)((double)cf * tsc_ms(*Lo->tsc, n, layer_temp(*Lo, t_stage, gi, gj), (double)mag));
      return cf;
    };
    if (ucol) {
      const V4<R> vu = VU[q];
      const R cu = col_scale(Lu, UC[q], vu.w);
      vx += cu * vu.x; vy += cu * vu.y; vz += cu * vu.z;
    } else if (L.uidx && Lu) {
      csr_pair(Lu, L.uidx, L.unbr, L.ucoef, mother_u, vx, vy, vz);
    }
    if (lcol) {
      const V4<R> vl = VL[q];
      const R cl = col_scale(Ll, LC[q], vl.w);
      vx += cl * vl.x; vy += cl * vl.y; vz += cl * vl.z;
    } else if (L.lidx && Ll) {
      csr_pair(Ll, L.lidx, L.lnbr, L.lcoef, mother_l, vx, vy, vz);
    }
    hx += ex + vx;
    hy += ey + vy;
    hz += ez + vz;
    if (STAGE == kPred && (flags & kFlagStoredField)) {
      const V4<R> hs = L.hf[n];
      hx = hs.x;
      hy = hs.y;
      hz = hs.z;
    }
    if (store_field) L.hf[n] = V4<R>{hx, hy, hz, (R)0};
    if (STAGE == kEval) {
      L.hd[n] = V4<R>{hdx, hdy, hdz, (R)0};
      continue;
    }

    // the grain's temperature: the layer's, or its profile's at the stage's time
    const double Tg = (GEN == 2 && L.tprof) ? temp_cell(*L.tprof, tps, t_stage, wi0 + i, wj0 + row0 + rr) : L.temperature;
    // thermal field / sqrt(dt) (llg.f90:1083): drawn by the predictor from the
    // step counter, reused by the corrector (:1262-1266)
    R htx = 0, hty = 0, htz = 0;
    if (thermal) {
      if (STAGE == kPred) {
        R gn[3];
        // the grain's stream (one per grain, shared by its cells)
        const int nt = L.cgrain ? max(0, L.cgrain[n]) : n;
        thermal_normals(rd.seed, (unsigned long long)l, (unsigned long long)step, (unsigned long long)nt, gn);
        R s = (GEN == 2 && L.tprof) ? (R)((double)pb.w * sqrt(Tg / rd.dt)) : pb.w * tfac;
        if (GEN == 2 && L.llb) {
          const LlbDev& P = *L.llb;
          if (P.mode != 2) {
            // LLB and MT runs: get_thermal with no_ms_p (get_fields, llg.f90:363-365;
            // field.f90:414-415): alpha_scale T / (Ms V)
            s = (R)sqrt(P.p[n].z * sc_al * Tg / rd.dt);
          } else if ((double)mf.w != 1.0) {
            // Zhang with |m| != 1 (field.f90:416-417): the variance over
            // max(floor_ms, |m|) instead of max(floor_ms, ms_scale)
            s = (R)sqrt(P.p[n].z * sc_al * Tg / (fmax(P.floor_ms, fabs((double)mf.w)) * rd.dt));
          }
        }
        htx = s * gn[0];
        hty = s * gn[1];
        htz = s * gn[2];
        L.ht[n] = V4<R>{htx, hty, htz, (R)0};
      } else {
        const V4<R> ht = at4(HT, q);
        htx = ht.x;
        hty = ht.y;
        htz = ht.z;
      }
    }
    const R fx = hx + htx, fy = hy + hty, fz = hz + htz;
    V4<R> mn;
    R dx = 0, dy = 0, dz = 0, tq2 = 0;
    double d2x = -1.0;  // errmx1's |dm|^2 where it is not |d|^2 (LLB)
    const bool llb = GEN == 2 && L.llb != nullptr;
    if (llb) {
      // push_llb (llg.f90:916-1064), Heun, in FP64; |m| in the w lane
      const LlbDev& P = *L.llb;
      const V4<double> gp = P.p[n];
      const V4<R> m0 = (STAGE == kCorr) ? M0[q] : mf;
      const double mc[3] = {(double)m0.x, (double)m0.y, (double)m0.z};
      const double mpr[3] = {(double)mf.x, (double)mf.y, (double)mf.z};
      const double hh[3] = {(double)hx, (double)hy, (double)hz}, th[3] = {(double)htx, (double)hty, (double)htz};
      double d1[3] = {0.0, 0.0, 0.0};
      if (STAGE == kCorr) {
        const V4<R> dd = DM[q];
        d1[0] = dd.x;
        d1[1] = dd.y;
        d1[2] = dd.z;
      }
      // (semi-implicit: push_llb's |type| = 2 branch, its first pass over dt/2 for -2;
      // mode 1: push_mt)
      const double pdt = (STAGE == kPred && mid) ? 0.5 * rd.dt : rd.dt;
      const LlbStep st =
          P.mode == 1
              ? mt_step(boris, STAGE == kPred, STAGE == kCorr, mc, (double)m0.w, mpr, (double)mf.w, hh, th, d1,
                        (double)pb.z, gp.y, P, Tg, L.gamma, pdt, rd.dt)
          : P.mode == 2
              ? zhang_step(boris, STAGE == kPred, STAGE == kCorr, mc, (double)m0.w, mpr, (double)mf.w, hh, th, d1,
                           (double)pb.z, gp.y, P, Tg, L.gamma, pdt, rd.dt)
          : (boris && (double)m0.w > 0.0)
              ? llb_boris(STAGE == kPred, mc, (double)m0.w, mpr, (double)mf.w, hh, th, (double)pb.z, gp.x, gp.y, P,
                          Tg, L.gamma, pdt)
              : llb_heun(STAGE == kCorr, mc, (double)m0.w, mpr, (double)mf.w, hh, th, d1, (double)pb.z, gp.x, gp.y, P,
                         Tg, L.gamma, pdt);
      if (STAGE == kPred && !boris) L.dm[n] = V4<R>{(R)st.d[0], (R)st.d[1], (R)st.d[2], (R)0};
      mn = V4<R>{(R)st.m[0], (R)st.m[1], (R)st.m[2], (R)st.mag};
      tq2 = (R)st.tq2;
      d2x = st.d2;
    } else if (mse > (R)0 && boris && (flags & kFlagRot)) {
      // analytic rotations (llg.f90:1093-1107), m_n in both stages
      const V4<R> m0 = (STAGE == kCorr) ? M0[q] : mf;
      const double s1 = -0.5 * (double)gamma * ((STAGE == kPred && mid) ? 0.5 * rd.dt : rd.dt);
      R tx, ty, tz;
      cross3(m0.x, m0.y, m0.z, fx, fy, fz, tx, ty, tz);
      tq2 = tx * tx + ty * ty + tz * tz;
      const double mm[3] = {(double)m0.x, (double)m0.y, (double)m0.z}, hh[3] = {(double)fx, (double)fy, (double)fz};
      double d[3];
      rot_push(mm, hh, s1, (double)pb.z, d);
      dx = (R)d[0];
      dy = (R)d[1];
      dz = (R)d[2];
      mn.x = (R)(mm[0] + d[0]);
      mn.y = (R)(mm[1] + d[1]);
      mn.z = (R)(mm[2] + d[2]);
    } else if (mse > (R)0 && boris) {
      // semi-implicit push (llg.f90:1109-1118): o = -g dt/2 h - alpha m,
      // d = 2/(1+|o|^2) (m + m x o) x o, m' = m + d (norm preserved, no renormalisation);
      // m is m_n in both stages, h the field of this stage
      const V4<R> m0 = (STAGE == kCorr) ? M0[q] : mf;
      const R a = pb.z;  // alpha * alpha_scale
      const R s1 = (R)(-0.5) * gamma * ((STAGE == kPred && mid) ? (R)0.5 * dt : dt);
      R tx, ty, tz;
      cross3(m0.x, m0.y, m0.z, fx, fy, fz, tx, ty, tz);
      tq2 = tx * tx + ty * ty + tz * tz;
      const R ox = s1 * fx - a * m0.x, oy = s1 * fy - a * m0.y, oz = s1 * fz - a * m0.z;
      R px, py, pz;
      cross3(m0.x, m0.y, m0.z, ox, oy, oz, px, py, pz);
      px += m0.x;
      py += m0.y;
      pz += m0.z;
      const R y = (R)2 / ((R)1 + ox * ox + oy * oy + oz * oz);
      cross3(px, py, pz, ox, oy, oz, dx, dy, dz);
      dx *= y;
      dy *= y;
      dz *= y;
      mn.x = m0.x + dx;
      mn.y = m0.y + dy;
      mn.z = m0.z + dz;
    } else if (mse > (R)0) {
      const R a = pb.z;  // alpha * alpha_scale
      const R s11 = fast_div(-gamma * dt, (R)1 + a * a);
      R tx, ty, tz, ux, uy, uz;
      cross3(mf.x, mf.y, mf.z, fx, fy, fz, tx, ty, tz);
      cross3(mf.x, mf.y, mf.z, tx, ty, tz, ux, uy, uz);
      dx = s11 * (tx + a * ux);
      dy = s11 * (ty + a * uy);
      dz = s11 * (tz + a * uz);
      tq2 = tx * tx + ty * ty + tz * tz;
      V4<R> m0;
      if (STAGE == kPred) {
        L.dm[n] = V4<R>{dx, dy, dz, (R)0};
        m0 = mf;
      } else {
        const V4<R> d1 = at4(DM, q);
        dx = (R)0.5 * (dx + d1.x);
        dy = (R)0.5 * (dy + d1.y);
        dz = (R)0.5 * (dz + d1.z);
        m0 = at4(M0, q);
      }
      mn.x = m0.x + dx;
      mn.y = m0.y + dy;
      mn.z = m0.z + dz;
      const R y = mn.x * mn.x + mn.y * mn.y + mn.z * mn.z;
      if (y > (R)0) {
        const R r = fast_rsqrt(y);
        mn.x *= r;
        mn.y *= r;
        mn.z *= r;
      }
    } else {
      // ms_scale <= 0: m along the (non-thermal) field (llg.f90:1140-1148)
      const R y = sqrt(hx * hx + hy * hy + hz * hz);
      if (y > (R)0) {
        mn.x = hx / y; mn.y = hy / y; mn.z = hz / y;
      } else {
        mn = (STAGE == kCorr) ? M0[q] : mf;
      }
    }
    if (!llb) mn.w = (R)0;
    if (STAGE == kPred) L.mp[n] = mn;
    else L.m[n] = mn;
    // the demag source of the next field evaluation (Ms ms_scale m): with
    // temperature scaling, the scale at that evaluation's time and state
    R msrc = mse;
    if constexpr (GEN == 2) {
      if (L.tsc) {
        const double t_src = (STAGE == kPred && mid) ? t_now + 0.5 * rd.dt : t_now + rd.dt;
        msrc = (R)((double)at4(PB, q).x * tsc_ms(*L.tsc, n, layer_temp(L, t_src, gi, gj), (double)mn.w));
      }
    }
    outr[(rr * 3 + 0) * rs + i] = msrc * mn.x;
    outr[(rr * 3 + 1) * rs + i] = msrc * mn.y;
    outr[(rr * 3 + 2) * rs + i] = msrc * mn.z;

    if constexpr (stats) {
      const V4<double> pv = L.pv[n];  // {vol, ms_scale, ms, 1}; (0, .., 0) on the extra cells of a grain
      const double msc = (GEN == 2 && L.tsc) ? sc_ms : pv.y;  // ms_scale of this evaluation
      const double v = pv.x, w = pv.z * msc * v;
      const double mx = mn.x, my = mn.y, mz = mn.z;
      rec[kSlotV] += v;
      rec[kSlotM + 0] += v * mx;
      rec[kSlotM + 1] += v * my;
      rec[kSlotM + 2] += v * mz;
      rec[kSlotM2 + 0] += v * mx * mx;
      rec[kSlotM2 + 1] += v * my * my;
      rec[kSlotM2 + 2] += v * mz * mz;
      rec[kSlotH + 0] += v * (double)hx;
      rec[kSlotH + 1] += v * (double)hy;
      rec[kSlotH + 2] += v * (double)hz;
      rec[kSlotWM + 0] += w * mx;
      rec[kSlotWM + 1] += w * my;
      rec[kSlotWM + 2] += w * mz;
      rec[kSlotW] += w;
      if (mx * L.hdir[0] + my * L.hdir[1] + mz * L.hdir[2] > 0.0) rec[kSlotNup] += pv.w;  // 1: counted grain record
      rec[kSlotMaxTq] = fmax(rec[kSlotMaxTq], (double)tq2 / (pv.z * pv.z));
      rec[kSlotMaxD2] = fmax(rec[kSlotMaxD2], d2x >= 0.0 ? d2x : (double)(dx * dx + dy * dy + dz * dz));
      // mmag1: |m| ms_scale vol (push_llg, llg.f90:1152), |m| vol (push_llb, :1062)
      rec[kSlotMmag] += llb ? (double)mn.w * v : sqrt(mx * mx + my * my + mz * mz) * msc * v;
      rec[kSlotVA] += v;  // volume of the grains pushed (do_grain)
      // energy at the evaluated state (field.f90:200, :360, :374, :339)
      const double e_d = -((double)mf.x * ((double)hdx + apx) + (double)mf.y * ((double)hdy + apy) +
                           (double)mf.z * ((double)hdz + apz)) * (double)mse;
      const double e_x = -((double)(ex + vx) * mf.x + (double)(ey + vy) * mf.y +
                           (double)(ez + vz) * mf.z) * (double)mse;
      rec[kSlotE] += (e_d + (double)e_k + e_x) * v;
    }
  }
  };
  if constexpr (GEN == 0 && !stats) {
    if (staged) grain_loop(IntC<1>{});
    else grain_loop(IntC<0>{});
  } else {
    grain_loop(IntC<2>{});
  }
  if constexpr (stats) {
    block_reduce_record(rec, sred, part + (size_t)blockIdx.x * kNPart);
  }
  if (STAGE == kEval || rd.demag == 0) return;  // (reloaded: one register less across the loop)

  // ---------------- forward row transform of Ms*m -> spectrum columns ----------------
  // (the register transforms of a row whose upper half is zero padding read
  // only its lower half)
  const int two_m = 2 * M;
  const bool half_in = regrow && nx <= M;
  const int zlim = half_in ? M : two_m;
  if (nx < zlim) {
    for (int s = 0; s < nseq; ++s)
      for (int i = nx + threadIdx.x; i < zlim; i += BLOCK) outr[s * rs + i] = (R)0;
  }
  __syncthreads();
  Cx<R>* scratch = (W == bufA) ? bufB : bufA;
  const int nys = rd.nys, lgct = rd.lgct, T = 1 << lgct, ntile = (ph + T - 1) >> lgct;
  if constexpr (kRegRowType) {
    if (regrow) {
      // X[k] = e - i w^k o (w = e^{-2 pi i / px}) for the group's sequence:
      // thread t takes k = t + j M/8 (and k = M), stored in column tiles of
      // T = 2^lgct columns, each tile row by row
      auto post = [&](int s, int t, int nt, const Cx<R>* Ys) {
        const int row = s / 3, comp = s - 3 * row;
        Cx<R>* dst = rd.specx + (size_t)(l * 3 + comp) * ntile * nys * T;
#pragma unroll 1
        for (int k = t; k <= M; k += nt) {
          const Cx<R> yk = Ys[k & (M - 1)];
          const Cx<R> ymk = cconj(Ys[(M - k) & (M - 1)]);
          const Cx<R> e = cscale(cadd(yk, ymk), (R)0.5);
          const Cx<R> o = cscale(csub(yk, ymk), (R)0.5);
          const Cx<R> wo = cmul(twpost[k], o);
          const long long at = (((long long)(k >> lgct) * nys + row0 + row) << lgct) + (k & (T - 1));
          if (!MRM_CHECK((long long)(l * 3 + comp) * ntile * nys * T + at < (long long)rd.nl * 3 * ntile * nys * T,
                         310, k))
            continue;
          dst[at] = csub(e, cmul_i(wo, (R)1));
        }
      };
      if (half_in) rrow_forward_any<BLOCK, LGMAX, true>(lgM, W, scratch, cs, nseq, twpass, post);
      else rrow_forward_any<BLOCK, LGMAX, false>(lgM, W, scratch, cs, nseq, twpass, post);
      return;
    }
  }
  Cx<R>* Y = block_fft_c<R, -1, NBMAX, BLOCK, LGMAX - 1>(W, scratch, lgM, nseq, twpass);
  // X[k] = e - i w^k o (w = e^{-2 pi i / px}), stored in column tiles of T =
  // 2^lgct columns (one column task), each tile row by row: consecutive threads
  // take the T columns of a row, then the task's next rows, then the next tile
  const int lgr = nrows > 1 ? 32 - __clz(nrows - 1) : 0;
  const int rmask = (1 << lgr) - 1;
#pragma unroll
  for (int comp = 0; comp < 3; ++comp) {
    Cx<R>* dst = rd.specx + (size_t)(l * 3 + comp) * ntile * nys * T;
    for (int t = threadIdx.x; t < (ntile << (lgct + lgr)); t += BLOCK) {
      const int c = t & (T - 1), row = (t >> lgct) & rmask, tile = t >> (lgct + lgr);
      const int k = (tile << lgct) + c;
      if (row >= nrows || k >= ph) continue;
      const Cx<R>* Ys = Y + (row * 3 + comp) * cs;
      const Cx<R> yk = Ys[k & (M - 1)];
      const Cx<R> ymk = cconj(Ys[(M - k) & (M - 1)]);
      const Cx<R> e = cscale(cadd(yk, ymk), (R)0.5);
      const Cx<R> o = cscale(csub(yk, ymk), (R)0.5);
      const Cx<R> wo = cmul(twpost[k], o);
      const long long at = (((long long)tile * nys + row0 + row) << lgct) + c;
      if (!MRM_CHECK((long long)(l * 3 + comp) * ntile * nys * T + at < (long long)rd.nl * 3 * ntile * nys * T, 300,
                     k))
        continue;
      dst[at] = csub(e, cmul_i(wo, (R)1));
    }
  }
}

// Column kernel: per spectral column k, forward FFT along y of the 3*nl
// half-spectra, H^_a = sum_b N^_ab M^_b, inverse FFT, written back row-major.
// PACKED: tensor stored as one real per (k, 0<=ky<=py/2) and component (the
// parity of each component restores the rest); otherwise the full complex
// tensor spectrum [k][pair][9][py] is used (FP64 runs).
//
// A task is one column tile (T = 2^lgct columns; a short last tile has fewer).
// Its 3*nl planes live in one shared buffer, transformed in place: the forward
// pass reads the M^ tile straight from global memory (rows >= ny are the zero
// padding, never loaded), the product runs in the transforms' digit-reversed
// order, and the last inverse pass writes rows < ny straight to H^.  Element j
// of column c in plane p sits at p*col_plane(py, lgct) + ((j + j/8) << lgct) + c:
// one pad row every 8 rows keeps the 8-element butterflies of the last forward
// (and first inverse) pass on distinct banks.
constexpr int kTensSliceBytes = 48 * 1024;
template <typename R>
MRM_HD bool tens_slice_fits(int reals) { return (size_t)reals * sizeof(R) <= (size_t)kTensSliceBytes; }

MRM_HD constexpr int col_plane(int py, int lgct) { return (py + (py >> 3)) << lgct; }
// complex values of one column buffer (even: what follows stays 16-byte aligned)
MRM_HD constexpr int col_buf_count(int py, int lgct, int nplane) { return even_up(nplane * col_plane(py, lgct)); }
// twiddles and buffers: one buffer up to two layers (6 planes), two beyond
template <typename R>
MRM_HD int col_fft_smem(int lgpy, int lgct, int nplane) {
  return (col_tw_count(lgpy) + (nplane > 6 ? 2 : 1) * col_buf_count(1 << lgpy, lgct, nplane)) * (int)sizeof(Cx<R>);
}

// H^ = N^ M^ at every position of the digit-reversed column buffer: in place
// for NLC = 1, 2 layers (a thread holds a position's 3*NLC inputs), otherwise
// (NLC = 0, nl layers) from A into the second buffer O.
template <typename R, bool PACKED, int NLC, int BLOCK>
MRM_D void col_product(const RunDev<R>& rd, Cx<R>* A, Cx<R>* O, const R* Ts, bool tsm, int k0, int nc, int* err) {
  const int nl = NLC > 0 ? NLC : rd.nl;
  const int py = rd.py, lgpy = rd.lgpy, pyhs = rd.pyhs, lgct = rd.lgct, T = 1 << lgct;
  const int plane = col_plane(py, lgct), npair = nl * nl;
  const int ph = (rd.px >> 1) + 1;
  const long long tens_len = PACKED ? (long long)ph * npair * 9 * pyhs * (long long)sizeof(R)
                                    : (long long)ph * npair * 9 * py * (long long)sizeof(Cx<R>);
  (void)tens_len;
  (void)err;
  // 3 outputs of layer ko at one position from the inputs of every layer
  auto mac = [&](int c, int ky, int ko, const Cx<R>* x, int xstride, Cx<R> h[3]) {
    h[0] = h[1] = h[2] = Cx<R>{(R)0, (R)0};
    for (int ks = 0; ks < nl; ++ks) {
      Cx<R> xm[3];
#pragma unroll
      for (int b = 0; b < 3; ++b) xm[b] = x[(size_t)(ks * 3 + b) * xstride];
      if constexpr (PACKED) {
        const bool upper = ky > (py >> 1);
        const int kyh = upper ? py - ky : ky;
        const size_t off = ((size_t)c * npair + ks * nl + ko) * 9 * pyhs;
        const R* Tp = tsm ? Ts + off : rd.tens + (size_t)k0 * npair * 9 * pyhs + off;
        const bool tok = MRM_CHECK(
            tsm || ((long long)k0 * npair * 9 * pyhs + (long long)off + 8 * pyhs + kyh) * (long long)sizeof(R) <
                       tens_len,
            430, kyh);
        R tv[9];
#pragma unroll
        for (int cc = 0; cc < 9; ++cc) tv[cc] = tok ? Tp[cc * pyhs + kyh] : (R)0;
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
          for (int b = 0; b < 3; ++b) {
            const int cc = 3 * a + b;
            R v = tv[cc];
            if (((kOddMask >> cc) & 1) && upper) v = -v;
            if ((kImagMask >> cc) & 1) h[a] = cadd(h[a], cmul_i(cscale(xm[b], v), (R)1));
            else h[a] = cadd(h[a], cscale(xm[b], v));
          }
      } else {
        const Cx<R>* Tc = reinterpret_cast<const Cx<R>*>(rd.tens) + ((size_t)(k0 + c) * npair + ks * nl + ko) * 9 * py;
        Cx<R> tv[9];
#pragma unroll
        for (int cc = 0; cc < 9; ++cc) tv[cc] = Tc[cc * py + ky];
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
          for (int b = 0; b < 3; ++b) h[a] = cadd(h[a], cmul(tv[3 * a + b], xm[b]));
      }
    }
  };
  if constexpr (NLC > 0) {
    for (int idx = threadIdx.x; idx < (py << lgct); idx += BLOCK) {
      const int c = idx & (T - 1), p = idx >> lgct;
      if (c >= nc) continue;
      const int ky = ip_freq(p, lgpy);
      const int at = ((p + (p >> 3)) << lgct) + c;
      Cx<R> xin[3 * NLC];
#pragma unroll
      for (int i = 0; i < 3 * NLC; ++i) xin[i] = A[(size_t)i * plane + at];
      Cx<R> h[NLC][3];
#pragma unroll
      for (int ko = 0; ko < NLC; ++ko) mac(c, ky, ko, xin, 1, h[ko]);
#pragma unroll
      for (int ko = 0; ko < NLC; ++ko)
#pragma unroll
        for (int a = 0; a < 3; ++a) A[(size_t)(ko * 3 + a) * plane + at] = h[ko][a];
    }
  } else {
    for (int idx = threadIdx.x; idx < (nl * py) << lgct; idx += BLOCK) {
      const int c = idx & (T - 1), p = (idx >> lgct) & (py - 1), ko = idx >> (lgct + lgpy);
      if (c >= nc) continue;
      const int ky = ip_freq(p, lgpy);
      const int at = ((p + (p >> 3)) << lgct) + c;
      Cx<R> h[3];
      mac(c, ky, ko, A + at, plane, h);
#pragma unroll
      for (int a = 0; a < 3; ++a) O[(size_t)(ko * 3 + a) * plane + at] = h[a];
    }
  }
}

// Accessors of the column transform (see ip_pass).  Shared buffer: element j
// of column c in plane h at h*plane + ((j + j/8) << lgT) + c; a butterfly's
// elements base + m*NS are affine in m there (NS = 1: base a multiple of 8;
// NS >= 8: a multiple of 8 apart).
template <typename R>
struct ColSmem {
  Cx<R>* A;
  int plane, lgT;
  MRM_D Cx<R>* ptr(int h, int c, int base) const { return A + h * plane + ((base + (base >> 3)) << lgT) + c; }
  MRM_D int stride(int ns) const { return (ns == 1 ? 1 : ns + (ns >> 3)) << lgT; }
  MRM_D bool valid(int) const { return true; }
};
// the task's tile of M^ in global memory: plane h at ((h*ntile + tile)*nys + j)*T + c;
// rows >= ny are the zero padding of the grid
template <typename R>
struct ColTileIn {
  const Cx<R>* src;  // the tile of plane 0
  size_t plane;
  int lgT, ny;
  MRM_D Cx<R>* ptr(int h, int c, int base) const {
    return const_cast<Cx<R>*>(src) + h * plane + ((size_t)base << lgT) + c;
  }
  MRM_D int stride(int ns) const { return ns << lgT; }
  MRM_D bool valid(int j) const { return j < ny; }
};
// H^ rows in global memory: plane h, row j at (h*ny + j)*phs + k0 + c; rows >= ny not stored
template <typename R>
struct ColRowsOut {
  Cx<R>* dst;  // column k0 of row 0, plane 0
  int ny, phs;
  MRM_D Cx<R>* ptr(int h, int c, int base) const { return dst + ((size_t)h * ny + base) * phs + c; }
  MRM_D int stride(int ns) const { return ns * phs; }
  MRM_D bool valid(int j) const { return j < ny; }
};

// The column transform of one task.  HALF when rows >= py/2 are the zero
// padding (open boundary: py >= 2 ny), so the first forward pass skips them and
// the last inverse pass does not produce them.
template <typename R, int LGN, bool PACKED, bool HALF, int BLOCK>
MRM_D void col_transform(const RunDev<R>& rd, Cx<R>* A, const Cx<R>* tws, const R* Ts, bool tsm, int k0, int nc,
                         int* err) {
  const int nl = rd.nl, ny = rd.ny, nys = rd.nys, lgct = rd.lgct;
  const int ph = (rd.px >> 1) + 1, ntile = (ph + (1 << lgct) - 1) >> lgct;
  const int plane = col_plane(1 << LGN, lgct), nplane = nl * 3;
  const ColTileIn<R> tile{rd.specx + ((size_t)(k0 >> lgct) * nys << lgct), (size_t)ntile * nys << lgct, lgct, ny};
  const ColSmem<R> sm{A, plane, lgct};
  const ColRowsOut<R> rows{rd.spech + k0, ny, rd.phs};
  MRM_CHECK((long long)(k0 + nc) <= ph && nys >= ny, 420, k0);
  ip_fft_fwd<R, LGN, HALF, BLOCK>(lgct, nc, nplane, tws, tile, sm);
  if (nl <= 2) {
    if (nl == 1) col_product<R, PACKED, 1, BLOCK>(rd, A, A, Ts, tsm, k0, nc, err);
    else col_product<R, PACKED, 2, BLOCK>(rd, A, A, Ts, tsm, k0, nc, err);
    __syncthreads();
    ip_fft_inv<R, LGN, HALF, BLOCK>(lgct, nc, nplane, tws, sm, rows);
  } else {
    // three or more layers: the product goes to the second buffer
    Cx<R>* O = A + col_buf_count(1 << LGN, lgct, nplane);
    col_product<R, PACKED, 0, BLOCK>(rd, A, O, Ts, tsm, k0, nc, err);
    __syncthreads();
    const ColSmem<R> so{O, plane, lgct};
    ip_fft_inv<R, LGN, HALF, BLOCK>(lgct, nc, nplane, tws, so, rows);
  }
}

template <typename R, int LGN, bool PACKED, int BLOCK>
MRM_D void col_transform_any(const RunDev<R>& rd, Cx<R>* A, const Cx<R>* tws, const R* Ts, bool tsm, int k0, int nc,
                             int* err) {
  if (rd.py >= 2 * rd.ny) col_transform<R, LGN, PACKED, true, BLOCK>(rd, A, tws, Ts, tsm, k0, nc, err);
  else col_transform<R, LGN, PACKED, false, BLOCK>(rd, A, tws, Ts, tsm, k0, nc, err);
}

template <typename R, bool PACKED, int BLOCK, int MINB>
__global__ void __launch_bounds__(BLOCK, MINB) col_kernel(const RunDev<R>* __restrict__ runs,
                                                          const Task* __restrict__ tasks,
                                                          const Cx<R>* __restrict__ twg, int istep,
                                                          int flags, int* __restrict__ err) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ uint64_t bars[1];
  pdl_launch_dependents();
  const Task tk = tasks[blockIdx.x];
  const RunDev<R>& rd = runs[tk.x];
  if (!rd.active || !rd.demag) return;
  const int k0 = tk.y, nc = tk.z;
  const int nl = rd.nl, py = rd.py, lgpy = rd.lgpy, lgct = rd.lgct;
  const int ph = (rd.px >> 1) + 1, pyhs = rd.pyhs;
  Cx<R>* tws = reinterpret_cast<Cx<R>*>(smem_raw);
  const int ntw = col_tw_count(lgpy);
  Cx<R>* A = tws + ntw;
  const int npair = nl * nl;
  const int tslice = nc * npair * 9 * pyhs;  // reals
  R* Ts = reinterpret_cast<R*>(A + (nl > 2 ? 2 : 1) * col_buf_count(py, lgct, nl * 3));
  // the slice is staged only where the launch's shared memory holds it (the
  // host leaves it out where it would cost resident blocks, and a smaller last
  // task may fit where the largest does not)
  const bool tsm = PACKED && tens_slice_fits<R>(tslice) &&
                   (long long)(reinterpret_cast<unsigned char*>(Ts) - smem_raw) + (long long)tslice * sizeof(R) <=
                       (long long)dynamic_smem_bytes();
  MRM_CHECK(k0 >= 0 && nc >= 1 && k0 + nc <= ph && (k0 & ((1 << lgct) - 1)) == 0 && nc <= (1 << lgct), 500, k0);
  MRM_CHECK((long long)col_fft_smem<R>(lgpy, lgct, nl * 3) <= (long long)dynamic_smem_bytes(), 501, lgpy);

  if (threadIdx.x == 0) {
    mbar_init(&bars[0], 1);
    mbar_fence_init();
  }
  __syncthreads();
  // static inputs: twiddles and this task's packed tensor slice (columns k0.. are contiguous)
  auto copy = [&](uint64_t* bar, void* dst, const void* src, long long src_off_bytes, long long src_len_bytes,
                  int bytes, int code) {
#ifdef MRM_CHECKS
    uint32_t dyn;
    asm volatile("mov.u32 %0, %%dynamic_smem_size;" : "=r"(dyn));
    const long long doff = (long long)smem_u32(dst) - (long long)smem_u32(smem_raw);
    if (!MRM_CHECK(src_off_bytes >= 0 && src_off_bytes + bytes <= src_len_bytes, code, src_off_bytes)) return;
    if (!MRM_CHECK(doff >= 0 && doff + bytes <= (long long)dyn, code + 1, doff)) return;
    if (!MRM_CHECK(((((uintptr_t)src) | (uintptr_t)doff | (uintptr_t)bytes) & 15) == 0, code + 2,
                   (long long)(uintptr_t)src))
      return;
#endif
    bulk_copy(bar, dst, src, (uint32_t)bytes);
  };
  const long long cb = (long long)sizeof(Cx<R>);
  if (threadIdx.x == 0) {
    copy(&bars[0], tws, twg + rd.tw_col, rd.tw_col * cb, (long long)tw_table_size() * cb, ntw * (int)cb, 400);
    if (tsm) {
      const long long off = (long long)k0 * npair * 9 * pyhs;
      copy(&bars[0], Ts, rd.tens + off, off * (long long)sizeof(R), (long long)ph * npair * 9 * pyhs * sizeof(R),
           tslice * (int)sizeof(R), 410);
    }
    mbar_arrive(&bars[0]);
  }
  pdl_wait();
  const bool run_it = (flags & kFlagForce) || step_due(rd, rd.step + istep);
  const bool ok = mbar_wait(&bars[0], 0);
  if (__syncthreads_or(!ok)) {
    if (threadIdx.x == 0) atomicOr(err, kErrBarrierTimeout);
    mbar_wait(&bars[0], 0);
    return;
  }
  if (!run_it) return;

  switch (lgpy) {
    case 1: col_transform_any<R, 1, PACKED, BLOCK>(rd, A, tws, Ts, tsm, k0, nc, err); break;
    case 2: col_transform_any<R, 2, PACKED, BLOCK>(rd, A, tws, Ts, tsm, k0, nc, err); break;
    case 3: col_transform_any<R, 3, PACKED, BLOCK>(rd, A, tws, Ts, tsm, k0, nc, err); break;
    case 4: col_transform_any<R, 4, PACKED, BLOCK>(rd, A, tws, Ts, tsm, k0, nc, err); break;
    case 5: col_transform_any<R, 5, PACKED, BLOCK>(rd, A, tws, Ts, tsm, k0, nc, err); break;
    case 6: col_transform_any<R, 6, PACKED, BLOCK>(rd, A, tws, Ts, tsm, k0, nc, err); break;
    case 7: col_transform_any<R, 7, PACKED, BLOCK>(rd, A, tws, Ts, tsm, k0, nc, err); break;
    case 8: col_transform_any<R, 8, PACKED, BLOCK>(rd, A, tws, Ts, tsm, k0, nc, err); break;
    case 9: col_transform_any<R, 9, PACKED, BLOCK>(rd, A, tws, Ts, tsm, k0, nc, err); break;
    case 10: col_transform_any<R, 10, PACKED, BLOCK>(rd, A, tws, Ts, tsm, k0, nc, err); break;
    case 11: col_transform_any<R, 11, PACKED, BLOCK>(rd, A, tws, Ts, tsm, k0, nc, err); break;
    default: col_transform_any<R, 12, PACKED, BLOCK>(rd, A, tws, Ts, tsm, k0, nc, err); break;
  }
}

// Grain average of the evaluation stage's demag over each grain's cells,
// written to every cell of the grain (get_magnetostatic, field.f90:449-470:
// FP64 sum over the cells, divided by their count).  Block row y: run y /
// kMaxLayers, layer y % kMaxLayers; layers with one grain per cell are skipped.
// A tabulated applied-field profile is averaged the same way into L.hapm
// (get_applied, field.f90:546-560), at the time of the stage that follows
// (istep, kFlagCorrTime, kFlagMid as the row kernel reads them).
template <typename R>
__global__ void gather_demag_kernel(const RunDev<R>* __restrict__ runs, int nruns, int istep, int flags) {
  const int r = blockIdx.y / kMaxLayers, l = blockIdx.y % kMaxLayers;
  if (r >= nruns) return;
  const RunDev<R>& rd = runs[r];
  if (!rd.active || l >= rd.nl) return;
  const LayerDev<R>& L = rd.L[l];
  if (!L.cgrain) return;
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= L.n) return;
  const int g = L.cgrain[c];
  if (g < 0) return;
  const int q0 = L.gci[g], q1 = L.gci[g + 1];
  double x = 0.0, y = 0.0, z = 0.0;
  for (int q = q0; q < q1; ++q) {
    const V4<R> h = L.hd[L.gcs[q]];
    x += (double)h.x;
    y += (double)h.y;
    z += (double)h.z;
  }
  const double k = (double)(q1 - q0);
  L.hdm[c] = V4<R>{(R)(x / k), (R)(y / k), (R)(z / k), (R)0};
  if (L.tab && L.hapm) {
    const TabDev& T = *L.tab;
    const long long step = rd.step + istep;
    const double t_now = rd.t_base + (double)(step - rd.step_base) * rd.dt;
    const double t = (flags & kFlagCorrTime) ? t_now + ((flags & kFlagMid) ? 0.5 * rd.dt : rd.dt) : t_now;
    const double s = ramp(L, t);
    const double ox = T.ox + T.vx * (t - T.t0) - T.rx;
    const double oy = T.oy + T.vy * (t - T.t0) - T.ry;
    double ax = 0.0, ay = 0.0, az = 0.0;
    for (int q = q0; q < q1; ++q) {
      const int cc = L.gcs[q], j = cc / rd.nx, i = cc - j * rd.nx;
      double vx, vy, vz;
      tab_value(T.v, T.nx, tab_weight(T.pos, T.nx, ((double)i + 0.5) * T.dx - ox),
                tab_weight(T.pos + T.nx, T.ny, ((double)j + 0.5) * T.dy - oy), s, vx, vy, vz);
      ax += vx;
      ay += vy;
      az += vz;
    }
    L.hapm[c] = V4<R>{(R)(ax / k), (R)(ay / k), (R)(az / k), (R)0};
  }
}

// Moving demag window (update_do_grain, data.f90:120-157): the copy of the
// current state into the other buffer (:139), m -> mp for every grain of
// run `slot`, so that grains outside the window read as their frozen state.
template <typename R>
__global__ void window_copy_kernel(const RunDev<R>* __restrict__ runs, int slot) {
  const RunDev<R>& rd = runs[slot];
  const int l = blockIdx.y;
  if (l >= rd.nl) return;
  const LayerDev<R>& L = rd.L[l];
  const long long n = (long long)rd.gnx * rd.gny;
  for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x)
    L.mp[c] = L.m[c];
}

// Stats records of the grains outside the window (frozen, do_grain false), one
// block per layer: volume, moments, the stale field of their last evaluation
// (llg.f90:215-233 reduces every grain), and |m| ms_scale vol of those whose
// index lies within the window's first and last grain (push_llg sums mmag1
// over min_n..max_n, llg.f90:1081,1152); into part[rd.frz + layer].
template <typename R>
__global__ void __launch_bounds__(256) frozen_stats_kernel(const RunDev<R>* __restrict__ runs, int slot,
                                                           double* __restrict__ part) {
  __shared__ double sred[32 * kNPart];
  const RunDev<R>& rd = runs[slot];
  const int l = blockIdx.x;
  if (l >= rd.nl || rd.frz < 0) return;
  const LayerDev<R>& L = rd.L[l];
  double rec[kNPart];
#pragma unroll
  for (int s = 0; s < kNPart; ++s) rec[s] = 0.0;
  const int gnx = rd.gnx, gny = rd.gny, i0 = rd.wi0, j0 = rd.wj0;
  const long long nmin = (long long)j0 * gnx + i0, nmax = (long long)(j0 + rd.ny - 1) * gnx + i0 + rd.nx - 1;
  for (long long c = threadIdx.x; c < (long long)gnx * gny; c += blockDim.x) {
    const int j = (int)(c / gnx), i = (int)(c - (long long)j * gnx);
    if (j >= j0 && j < j0 + rd.ny && i >= i0 && i < i0 + rd.nx) continue;
    const V4<double> pv = L.pv[c];
    const V4<R> mr = L.m[c], hr = L.hf[c];
    const double v = pv.x, w = pv.z * pv.y * v;
    const double mx = mr.x, my = mr.y, mz = mr.z;
    rec[kSlotV] += v;
    rec[kSlotM + 0] += v * mx;
    rec[kSlotM + 1] += v * my;
    rec[kSlotM + 2] += v * mz;
    rec[kSlotM2 + 0] += v * mx * mx;
    rec[kSlotM2 + 1] += v * my * my;
    rec[kSlotM2 + 2] += v * mz * mz;
    rec[kSlotH + 0] += v * (double)hr.x;
    rec[kSlotH + 1] += v * (double)hr.y;
    rec[kSlotH + 2] += v * (double)hr.z;
    rec[kSlotWM + 0] += w * mx;
    rec[kSlotWM + 1] += w * my;
    rec[kSlotWM + 2] += w * mz;
    rec[kSlotW] += w;
    if (mx * L.hdir[0] + my * L.hdir[1] + mz * L.hdir[2] > 0.0) rec[kSlotNup] += pv.w;
    if (c >= nmin && c <= nmax) rec[kSlotMmag] += L.llb ? (double)mr.w * v : sqrt(mx * mx + my * my + mz * mz) * pv.y * v;
  }
  block_reduce_record(rec, sred, part + (size_t)(rd.frz + l) * kNPart);
}

// llg_type 2: the predictor buffer holds m_{n+1} after the single push; copy
// it to the state (one row task per block).
template <typename R>
__global__ void __launch_bounds__(256) commit_kernel(const RunDev<R>* __restrict__ runs,
                                                     const Task* __restrict__ tasks, int istep, int flags) {
  pdl_launch_dependents();
  const Task tk = tasks[blockIdx.x];
  const RunDev<R>& rd = runs[tk.x];
  if (!rd.active) return;
  pdl_wait();
  const long long step = *reinterpret_cast<const volatile long long*>(&rd.step) + istep;
  if (!(flags & kFlagForce) && !step_due(rd, step)) return;
  const LayerDev<R>& L = rd.L[tk.y];
  // (a windowed run's task row is grid row wj0 + row from column wi0)
  const int n0 = rd.gnx ? (rd.wj0 + tk.z) * rd.gnx + rd.wi0 : tk.z * rd.nx, cnt = tk.w * rd.nx;
  for (int i = threadIdx.x; i < cnt; i += blockDim.x) L.m[n0 + i] = L.mp[n0 + i];
}

// Advances every active run's step counter after a captured chunk of k steps.
template <typename R>
__global__ void advance_kernel(RunDev<R>* runs, int nruns, int k) {
  pdl_launch_dependents();
  pdl_wait();
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nruns) return;
  RunDev<R>& rd = runs[r];
  if (!rd.active) return;
  long long left = rd.step_end - rd.step;
  if (left < 0) left = 0;
  rd.stats_ok = left >= k ? 1 : 0;
  rd.step += (left < k) ? left : k;
}

// mrm_gpu_stats layout
struct StatsDev {
  double t;
  long long step;
  double mave[3], mvar[3], have[3];
  double errmx, errmx1, mmag, energy;
  double mave_l[kMaxLayers][3], mvar_l[kMaxLayers][3], have_l[kMaxLayers][3], mms_l[kMaxLayers][3];
  double vol_l[kMaxLayers], msvol_l[kMaxLayers];
  long long nup_l[kMaxLayers];
  double errmx1_l[kMaxLayers];
};

// FP64 reduction of each run's per-task stats records into StatsDev; one
// 256-thread block per run, fixed reduction order (deterministic).
template <typename R>
__global__ void __launch_bounds__(256) finalize_stats_kernel(const RunDev<R>* __restrict__ runs,
                                                             const Task* __restrict__ tasks,
                                                             const double* __restrict__ part,
                                                             StatsDev* __restrict__ out, int nruns) {
  __shared__ double sred[32 * kNPart];
  __shared__ double acc[kMaxLayers][kNPart];
  pdl_launch_dependents();
  pdl_wait();
  const int r = blockIdx.x;
  if (r >= nruns) return;
  const RunDev<R>& rd = runs[r];
  if (!rd.active || !rd.stats_ok) return;  // keep the stats of the run's last stats step
  for (int l = 0; l < rd.nl; ++l) {
    double rec[kNPart];
#pragma unroll
    for (int s = 0; s < kNPart; ++s) rec[s] = 0.0;
    for (int q = rd.row_task0 + threadIdx.x; q < rd.row_task0 + rd.nrow_tasks; q += blockDim.x) {
      if (tasks[q].y != l) continue;
      const double* p = part + (size_t)q * kNPart;
#pragma unroll
      for (int s = 0; s < kNPart; ++s) rec[s] = slot_is_max(s) ? fmax(rec[s], p[s]) : rec[s] + p[s];
    }
    block_reduce_record(rec, sred, acc[l]);
    __syncthreads();
  }
  if (threadIdx.x != 0) return;
  if (rd.frz >= 0)  // the frozen grains outside a moving demag window
    for (int l = 0; l < rd.nl; ++l)
      for (int s = 0; s < kNPart; ++s) {
        const double f = part[(size_t)(rd.frz + l) * kNPart + s];
        acc[l][s] = slot_is_max(s) ? fmax(acc[l][s], f) : acc[l][s] + f;
      }
  StatsDev& st = out[r];
  st.step = rd.step;
  st.t = rd.t_base + (double)(rd.step - rd.step_base) * rd.dt;
  double vt = 0, mt = 0, m1 = 0, mmag = 0, en = 0;
  for (int a = 0; a < 3; ++a) { st.mave[a] = 0; st.mvar[a] = 0; st.have[a] = 0; }
  for (int l = 0; l < rd.nl; ++l) vt += acc[l][kSlotV];
  for (int l = 0; l < kMaxLayers; ++l) {
    const bool on = l < rd.nl;
    const double V = on ? acc[l][kSlotV] : 0.0;
    for (int a = 0; a < 3; ++a) {
      const double mean = (on && V > 0) ? acc[l][kSlotM + a] / V : 0.0;
      st.mave_l[l][a] = mean;
      st.mvar_l[l][a] = (on && V > 0) ? acc[l][kSlotM2 + a] / V - mean * mean : 0.0;
      st.have_l[l][a] = (on && V > 0) ? acc[l][kSlotH + a] / V : 0.0;
      const double W = on ? acc[l][kSlotW] : 0.0;
      st.mms_l[l][a] = on ? acc[l][kSlotWM + a] * W / (W * W + 1e-300) : 0.0;
    }
    st.vol_l[l] = V;
    st.msvol_l[l] = on ? acc[l][kSlotW] : 0.0;
    st.nup_l[l] = on ? (long long)acc[l][kSlotNup] : 0;
    st.errmx1_l[l] = on ? acc[l][kSlotMaxD2] : 0.0;
    if (on && V > 0) {
      for (int a = 0; a < 3; ++a) {
        st.mave[a] += V * st.mave_l[l][a] / vt;
        st.mvar[a] += V * st.mvar_l[l][a] / vt;
        st.have[a] += V * st.have_l[l][a] / vt;
      }
      mmag += acc[l][kSlotMmag] / acc[l][kSlotVA];  // over the pushed grains' volume (llg.f90:1239)
      mt = fmax(mt, acc[l][kSlotMaxTq]);
      m1 = fmax(m1, acc[l][kSlotMaxD2]);
      en += acc[l][kSlotE];
    }
  }
  st.errmx = sqrt(mt);
  st.errmx1 = m1;
  st.mmag = mmag;
  st.energy = en;
}

}  // namespace mrm
