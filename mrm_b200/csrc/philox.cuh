// philox.cuh -- counter-based thermal-noise stream.
//
// Philox (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy as 1,
// 2, 3", SC'11) with the Box-Muller transform, one draw of three normals per
// grain, step and layer (the predictor stores them for the corrector, as the
// reference reuses hthm, src/llg.f90:1262-1266).
//  * FP64 runs: Philox4x64-10, counter (grain, step, layer, 0), key
//    (seed, 0x6d726d), 53-bit uniforms;
//  * FP32 runs: Philox4x32-10, counter (grain, step low, step high, layer),
//    key (seed low, seed high ^ 0x6d726d), 24-bit uniforms and the hardware
//    approximations of log, sqrt and sin/cos (the 64-bit multiplies of the
//    4x64 form were a sixth of the predictor's time).
#pragma once
#include "common.cuh"

namespace mrm {

MRM_D void philox4x64_10(unsigned long long c[4], unsigned long long k0, unsigned long long k1) {
  const unsigned long long M0 = 0xD2E7470EE14C6C93ull, M1 = 0xCA5A826395121157ull;
  const unsigned long long W0 = 0x9E3779B97F4A7C15ull, W1 = 0xBB67AE8584CAA73Bull;
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    unsigned long long hi0 = __umul64hi(M0, c[0]), lo0 = M0 * c[0];
    unsigned long long hi1 = __umul64hi(M1, c[2]), lo1 = M1 * c[2];
    unsigned long long n0 = hi1 ^ c[1] ^ k0;
    unsigned long long n2 = hi0 ^ c[3] ^ k1;
    c[0] = n0;
    c[1] = lo1;
    c[2] = n2;
    c[3] = lo0;
    k0 += W0;
    k1 += W1;
  }
}

MRM_D void philox4x32_10(unsigned int c[4], unsigned int k0, unsigned int k1) {
  const unsigned int M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
  const unsigned int W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    const unsigned int hi0 = __umulhi(M0, c[0]), lo0 = M0 * c[0];
    const unsigned int hi1 = __umulhi(M1, c[2]), lo1 = M1 * c[2];
    const unsigned int n0 = hi1 ^ c[1] ^ k0;
    const unsigned int n2 = hi0 ^ c[3] ^ k1;
    c[0] = n0;
    c[1] = lo1;
    c[2] = n2;
    c[3] = lo0;
    k0 += W0;
    k1 += W1;
  }
}

// Three standard normals of grain `grain` at step `step` in stream `layer`.
MRM_D void thermal_normals(unsigned long long seed, unsigned long long layer,
                           unsigned long long step, unsigned long long grain, double n[3]) {
  unsigned long long c[4] = {grain, step, layer, 0ull};
  philox4x64_10(c, seed, 0x6d726dull);
  const double s53 = 1.0 / 9007199254740992.0;
  double u0 = ((double)(c[0] >> 11) + 0.5) * s53;
  double u1 = ((double)(c[1] >> 11) + 0.5) * s53;
  double u2 = ((double)(c[2] >> 11) + 0.5) * s53;
  double u3 = ((double)(c[3] >> 11) + 0.5) * s53;
  double ra = sqrt(-2.0 * log(u0));
  double rb = sqrt(-2.0 * log(u2));
  double s, co;
  sincospi(2.0 * u1, &s, &co);
  n[0] = ra * co;
  n[1] = ra * s;
  n[2] = rb * cospi(2.0 * u3);
}

MRM_D void thermal_normals(unsigned long long seed, unsigned long long layer,
                           unsigned long long step, unsigned long long grain, float n[3]) {
  unsigned int c[4] = {(unsigned int)grain, (unsigned int)step, (unsigned int)(step >> 32), (unsigned int)layer};
  philox4x32_10(c, (unsigned int)seed, (unsigned int)(seed >> 32) ^ 0x6d726du);
  const float s24 = 1.0f / 16777216.0f;
  float u0 = ((float)(c[0] >> 8) + 0.5f) * s24;
  float u1 = ((float)(c[1] >> 8) + 0.5f) * s24;
  float u2 = ((float)(c[2] >> 8) + 0.5f) * s24;
  float u3 = ((float)(c[3] >> 8) + 0.5f) * s24;
  // Box-Muller on the hardware approximations (__logf, rsqrtf, __sincosf with
  // the angle in (-pi, pi), where they are accurate to about 1e-6 absolute).
  // The floor keeps the radius finite when __logf of a u just below 1 rounds
  // to a non-negative value (the radius there is below 1e-3 either way).
  const float la = fmaxf(-2.0f * __logf(u0), 1e-30f), lb = fmaxf(-2.0f * __logf(u2), 1e-30f);
  const float ra = la * rsqrtf(la), rb = lb * rsqrtf(lb);
  const float kPi = 3.14159265358979f;
  float s, co;
  __sincosf(kPi * (2.0f * u1 - 1.0f), &s, &co);
  n[0] = ra * co;
  n[1] = ra * s;
  n[2] = rb * __cosf(kPi * (2.0f * u3 - 1.0f));
}

}  // namespace mrm
