// fr_tma.cuh -- one-dimensional bulk copies (the TMA unit's cp.async.bulk,
// sm_90 and later; used here on sm_100a) between global and shared memory,
// completed through a shared-memory mbarrier, and bulk stores back to global
// memory.  Single-GPU copies of this GPU's own memory, no multicast.
//
// Rules the callers keep: every source, destination and size is a multiple of
// 16 bytes; the mbarrier is armed with the byte count of the copies it tracks
// before they are issued; waits are bounded (about one second of
// %globaltimer) and report a timeout through a device flag instead of
// spinning for ever.
#pragma once

#include <cuda_runtime.h>

namespace frb {

__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count)
{
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// makes initialised mbarriers visible to the asynchronous (TMA) proxy
__device__ __forceinline__ void mbar_fence_init()
{
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}

// one arrival that also announces `bytes` of copies still to complete
__device__ __forceinline__ void mbar_arrive_tx(unsigned long long* bar, unsigned bytes)
{
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity)
{
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ unsigned long long global_ns()
{
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;\n" : "=l"(t));
  return t;
}

// Bounded wait for phase `parity` of the barrier.  Returns false (and sets
// *err to 1) when about one second passes without completion; a set *err
// makes later waits give up at once, so a failed launch ends quickly.
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity, int* err)
{
  if (mbar_try_wait(bar, parity)) return true;
  const unsigned long long t0 = global_ns();
  for (;;) {
    if (mbar_try_wait(bar, parity)) return true;
    if (err && *(volatile int*)err) return false;
    if (global_ns() - t0 > 1000000000ull) {
      if (err) atomicExch(err, 1);
      return false;
    }
  }
}

// global -> shared, completion counted on `bar` (bytes and addresses multiples of 16)
__device__ __forceinline__ void bulk_load(void* dst, const void* src, unsigned bytes, unsigned long long* bar)
{
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// generic-proxy shared-memory writes become visible to the bulk (async) proxy
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }

// shared -> global (bytes and addresses multiples of 16), tracked by bulk groups
__device__ __forceinline__ void bulk_store(void* dst, const void* src, unsigned bytes)
{
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;\n" ::"l"(dst), "r"(smem_u32(src)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;\n" ::: "memory"); }
// the shared-memory sources of every committed bulk store have been read
__device__ __forceinline__ void bulk_wait_read() { asm volatile("cp.async.bulk.wait_group.read 0;\n" ::: "memory"); }
// every committed bulk store has completed
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;\n" ::: "memory"); }

}  // namespace frb
