// Asynchronous global -> shared copies (cp.async, sm_80+ form, kept on sm_100a for per-thread
// prefetch rings where every thread stages its own data and no block barrier is wanted).
#pragma once
#include <cstdint>

namespace zkb {

// 16-byte asynchronous copy global -> shared (both addresses 16-byte aligned), L2 only
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const uint32_t sa = (uint32_t)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
// wait until at most N of this thread's commit groups are still in flight
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

}  // namespace zkb
