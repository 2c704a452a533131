// tma.cuh -- 1-D bulk copies (cp.async.bulk, the TMA engine) from global into
// shared memory, completed on an mbarrier, with bounded waits (sm_90+).
//
// One elected thread arms a barrier with the byte count it is about to
// request and issues the copies; every thread then waits on the barrier's
// phase 0.  Each barrier is used once per kernel.  Source and destination
// must be 16-byte aligned and sizes multiples of 16 bytes.  A wait gives up
// after about a second (kWaitCycles) or kSpinLimit polls: the copies then
// count as failed, and the kernel raises an error flag, waits once more
// (bounded) for its copies to land and returns.
#pragma once
#include <cstdint>

#include "common.cuh"

namespace mrm {

constexpr int kSpinLimit = 1 << 22;
constexpr long long kWaitCycles = 2000000000LL;  // ~1 s at the B200's 1.9-2 GHz SM clock
enum DeviceError { kErrBarrierTimeout = 1, kErrShape = 2, kErrCheck = 4 };

// Self-checks of the MRM_CHECKS build: a failed check records its code (first
// failure wins, err[1]; the offending value in err[2..3]) and the access is
// skipped.  Off in normal builds.
#ifdef MRM_CHECKS
MRM_D bool mrm_check(bool ok, int* err, int code, long long v) {
  if (!ok) {
    atomicOr(err, kErrCheck);
    if (atomicCAS(err + 1, 0, code) == 0) {
      err[2] = (int)(v & 0xffffffff);
      err[3] = (int)(v >> 32);
    }
  }
  return ok;
}
#define MRM_CHECK(cond, code, v) mrm_check((cond), err, (code), (long long)(v))
#else
#define MRM_CHECK(cond, code, v) true
#endif

MRM_D uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// dynamic shared memory of the running launch (bytes)
MRM_D uint32_t dynamic_smem_bytes() {
  uint32_t v;
  asm volatile("mov.u32 %0, %%dynamic_smem_size;" : "=r"(v));
  return v;
}

MRM_D void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
// makes barrier initialisation visible to the async (TMA) proxy
MRM_D void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

MRM_D void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

MRM_D bool mbar_try_wait(uint64_t* bar, uint32_t phase) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(phase)
      : "memory");
  return ok != 0;
}

// bounded wait on phase `phase` (about one second of SM clock); false if the
// limit ran out
MRM_D bool mbar_wait(uint64_t* bar, uint32_t phase) {
  if (mbar_try_wait(bar, phase)) return true;
  const long long t0 = clock64();
  for (int i = 0; i < kSpinLimit; ++i) {
    if (mbar_try_wait(bar, phase)) return true;
    if (clock64() - t0 > kWaitCycles) break;
  }
  return false;
}

// bulk prefetch of `bytes` (a multiple of 16, 16-byte aligned source) from
// global memory into L2; nothing waits for it
MRM_D void bulk_prefetch_l2(const void* src, uint32_t bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src), "r"(bytes) : "memory");
}

// global -> shared bulk copy of `bytes` (multiple of 16) completing on `bar`
MRM_D void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// Issuer-side pattern: copy(bar, ...) for each piece (raises the barrier's
// expected byte count, then issues the copy), then one mbar_arrive(bar).  The
// transaction count may dip below zero while copies land before the arrive;
// the phase completes only after the arrive, once every byte has landed.
MRM_D void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.expect_tx.relaxed.cta.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
MRM_D void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
MRM_D void bulk_copy(uint64_t* bar, void* dst, const void* src, uint32_t bytes) {
  mbar_expect_tx(bar, bytes);
  bulk_g2s(dst, src, bytes, bar);
}

}  // namespace mrm
