// Host build of the double-double arithmetic of mrm_b200/csrc/dd.cuh (the
// device tensor's arithmetic) checked against quadruple precision
// (libquadmath): prints the largest relative errors of log, atan, sqrt and
// division over seeded random arguments spanning 26 decades.
#define MRM_HD inline
#include "../../mrm_b200/csrc/dd.cuh"

#include <quadmath.h>

#include <cstdio>
#include <random>

using mrm::dd;
static __float128 q(dd a) { return (__float128)a.hi + (__float128)a.lo; }
static dd from_q(__float128 x) {
  const double h = (double)x;
  return dd{h, (double)(x - (__float128)h)};
}

int main() {
  std::mt19937_64 g(7);
  std::uniform_real_distribution<double> u(-30.0, 30.0);
  double wl = 0, wa = 0, ws = 0, wd = 0;
  for (int i = 0; i < 100000; ++i) {
    const dd a = from_q(expq((__float128)u(g)) * (1 + (__float128)u(g) * (__float128)1e-20));
    const __float128 x = q(a);
    const double el = (double)(fabsq(q(mrm::dd_log(a)) - logq(x)) / fmaxq((__float128)1, fabsq(logq(x))));
    const dd s = (i & 1) ? mrm::dd_neg(a) : a;
    const double ea = (double)(fabsq(q(mrm::dd_atan(s)) - atanq(q(s))) / fabsq(atanq(q(s))));
    const double es = (double)(fabsq(q(mrm::dd_sqrt(a)) - sqrtq(x)) / sqrtq(x));
    const dd b = from_q(expq((__float128)u(g)));
    const double ed = (double)(fabsq(q(mrm::dd_div(a, b)) - x / q(b)) / (x / q(b)));
    wl = el > wl ? el : wl;
    wa = ea > wa ? ea : wa;
    ws = es > ws ? es : ws;
    wd = ed > wd ? ed : wd;
  }
  std::printf("%.6e %.6e %.6e %.6e\n", wl, wa, ws, wd);
  return 0;
}
