// device_common.cuh -- device helpers shared by the radiation kernels (sm_100a).
//
//  * 1-D TMA bulk copies global -> shared (cp.async.bulk ... mbarrier::complete_tx::bytes), with
//    mbarrier waits that give up after a bounded number of polls and raise an error flag instead
//    of hanging the GPU.
//  * Argument reduction of the retarded phase to [-pi, pi] (Cody & Waite two-constant reduction;
//    the first step is exact with FMA for |phase| < 2^52 ulp(2pi), see reduce_2pi below).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace osc {
namespace dev {

// Error flags written by kernels (bit mask, OR-ed into a device word read back by the host).
// kErrPlan: a kernel was launched with a tile size other than the one it was compiled for (the
// host sized its partial sums for that tile); the kernel returns before touching memory.
enum : unsigned { kErrTmaTimeout = 1u, kErrBadArgs = 2u, kErrSuperluminal = 4u, kErrPlan = 8u };

// Polls of an mbarrier before a wait is declared stuck (each poll is a try_wait that itself may
// suspend the thread for a hardware-defined interval), i.e. far beyond any legitimate latency.
constexpr uint32_t kMaxPolls = 1u << 22;

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_barrier_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}

// Returns true once the barrier phase with parity `parity` has completed; false if it did not
// complete within kMaxPolls polls.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  const uint32_t a = smem_addr(bar);
  for (uint32_t i = 0; i < kMaxPolls; ++i) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// Bulk copy `bytes` (multiple of 16, both addresses 16-byte aligned) from global to shared memory,
// completing on `bar`.
__device__ __forceinline__ void tma_load_1d(void* smem_dst, const void* gmem_src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_addr(smem_dst)),
      "l"(gmem_src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}

// ---------------------------------------------------------------------------------------------
// Phase reduction.  For a double `phi` with |phi| < 2^40, k = rint(phi / 2pi) and
//   r1 = fma(-k, P1, phi)    is exact: phi and k*P1 are both multiples of 2^-50 once |phi| >= 4
//                            and |r1| < 4, so r1 fits in 53 bits;
//   r  = fma(-k, P2, r1)     adds the second term of 2pi = P1 + P2 (+ O(2^-107)).
// The reduced argument carries an absolute error below 1e-15 for |phi| < 2^40 (4 x 10^11 rad at
// 3 keV and 30 m is 2^38.7), so sin/cos of it agree with the correctly rounded sin/cos of phi to a
// few 1e-16.  (Cody & Waite, "Software Manual for the Elementary Functions", 1980.)
// ---------------------------------------------------------------------------------------------
constexpr double kTwoPiHi = 6.283185307179586232;      // RN(2 pi)
constexpr double kTwoPiLo = 2.4492935982947064e-16;    // RN(2 pi - kTwoPiHi)
constexpr double kInvTwoPi = 0.15915494309189535;      // RN(1 / (2 pi))

__device__ __forceinline__ double reduce_2pi(double phi) {
  const double k = rint(phi * kInvTwoPi);
  const double r1 = __fma_rn(-k, kTwoPiHi, phi);
  return __fma_rn(-k, kTwoPiLo, r1);
}

}  // namespace dev
}  // namespace osc
