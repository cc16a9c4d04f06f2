// tma.cuh -- bulk asynchronous copies (cp.async.bulk, the TMA engine) into
// shared memory, completed on mbarriers, with bounded waits.
//
// A producer thread arms a stage's "full" barrier with the bytes it will
// copy (mbarrier.arrive.expect_tx), then issues one cp.async.bulk per
// contiguous array; the barrier's phase completes when every byte has
// landed.  Consumers wait on the phase, read the stage, and arrive on the
// stage's "empty" barrier; the producer waits on that before it refills the
// stage.  Every wait is bounded: after kWaitLimitNs of global time it gives
// up, counts a timeout in g_wait_timeouts (read by op2b_wait_timeouts) and
// reports failure, so a lost completion can never hang the GPU.
//
// Copies here are plain CTA-local loads from this GPU's memory: no cluster
// multicast.  Source and destination addresses and sizes are multiples of
// 16 bytes (the hardware's rule for the untiled bulk copy); callers round
// sizes down and read the remainder with ordinary loads.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace op2b {

constexpr unsigned long long kWaitLimitNs = 1000000000ull;  // one second

// waits that ran out, summed over every kernel of the including file since
// the last reset (one counter per translation unit: no relocatable device
// code); the file exposes it on the host
static __device__ unsigned g_wait_timeouts;

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void mbar_init(uint32_t bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

// make the initialised barriers visible to the async (copy) proxy
__device__ __forceinline__ void mbar_init_fence() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint32_t bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.release.cta.shared::cta.b64 _, [%0], %1;" ::"r"(bar),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.release.cta.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.acquire.cta.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

// wait for the phase of parity `parity` to complete; false (and one
// timeout counted) if it has not after kWaitLimitNs
__device__ __forceinline__ bool mbar_wait(uint32_t bar, unsigned parity) {
  if (mbar_try_wait(bar, parity)) return true;
  const unsigned long long t0 = global_ns();
  for (;;) {
    for (int i = 0; i < 64; i++)
      if (mbar_try_wait(bar, parity)) return true;
    if (global_ns() - t0 > kWaitLimitNs) {
      atomicAdd(&g_wait_timeouts, 1u);
      return false;
    }
  }
}

// bytes [src, src + bytes) of global memory to shared memory at dst,
// completing on barrier bar; all three multiples of 16
__device__ __forceinline__ void bulk_load(uint32_t dst, const void *src, unsigned bytes,
                                          uint32_t bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          dst),
      "l"(src), "r"(bytes), "r"(bar)
      : "memory");
}

}  // namespace op2b
