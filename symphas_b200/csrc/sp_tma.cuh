/*
 * sp_tma.cuh -- thin inline-PTX wrappers for the Blackwell (sm_100a) bulk
 * tensor copy engine (TMA) and shared-memory mbarriers.
 *
 * Only non-multicast loads are used (`cp.async.bulk.tensor.{2,3}d.shared::cluster
 * .global.tile.mbarrier::complete_tx::bytes`); every wait is bounded and
 * reports failure instead of spinning forever.
 */
#pragma once

#include <cuda.h>
#include <stdint.h>

namespace sp {
namespace tma {

__device__ __forceinline__ uint32_t saddr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(saddr(bar)), "r"(count) : "memory");
}

// make the initialised barriers visible to the async (TMA) proxy
__device__ __forceinline__ void fence_barrier_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(saddr(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(saddr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// try_wait with a suspend-time hint (ns): the thread sleeps in hardware until
// the phase completes or the hint expires, instead of re-issuing the poll
__device__ __forceinline__ bool mbar_try_wait_for(uint64_t* bar, uint32_t parity, uint32_t ns) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(saddr(bar)), "r"(parity), "r"(ns)
      : "memory");
  return ok != 0;
}

// Bounded wait for phase `parity` of `bar`: each try sleeps up to `sleep_ns`
// in hardware (woken when the phase completes); give up once more than
// `limit` SM cycles have passed.
__device__ __forceinline__ bool mbar_wait_limit(uint64_t* bar, uint32_t parity, long long limit,
                                                uint32_t sleep_ns) {
  if (mbar_try_wait(bar, parity)) return true;
  const long long t0 = clock64();
  while (!mbar_try_wait_for(bar, parity, sleep_ns))
    if (clock64() - t0 > limit) return false;
  return true;
}

// The waits of the step kernels: 1 ms tries, give up after about 2^31 SM
// cycles (~1 s).
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  return mbar_wait_limit(bar, parity, 1LL << 31, 1000000u);
}

// Error path of a CTA that gave up on a wait: before it leaves, wait (again
// bounded) for the loads it still has in flight, so that no copy lands in
// shared memory after the CTA has exited.  Load number q went to ring slot
// q % nslot with barrier phase (q / nslot) & 1.
__device__ __forceinline__ void drain(uint64_t* bars, int nslot, int first, int last) {
  for (int q = first; q <= last; ++q) mbar_wait(&bars[q % nslot], uint32_t((q / nslot) & 1));
}

__device__ __forceinline__ void load_2d(void* dst, const CUtensorMap* map, uint64_t* bar, int x,
                                        int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4}], [%2];" ::"r"(saddr(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(saddr(bar)), "r"(x), "r"(y)
      : "memory");
}

__device__ __forceinline__ void load_3d(void* dst, const CUtensorMap* map, uint64_t* bar, int x,
                                        int y, int z) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4, %5}], [%2];" ::"r"(saddr(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(saddr(bar)), "r"(x), "r"(y), "r"(z)
      : "memory");
}

__device__ __forceinline__ void prefetch_map(const CUtensorMap* map) {
  asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(map)) : "memory");
}

}  // namespace tma
}  // namespace sp
