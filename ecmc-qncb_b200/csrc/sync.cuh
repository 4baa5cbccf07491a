// sync.cuh — device-side flag waits shared by the persistent kernels.
//
// A block that depends on work of other blocks of the same launch polls counters or flags
// with acquire loads.  Every wait is bounded by wall-clock time (%globaltimer) and by a poll
// count; a block that gives up counts a timeout in status[1] and raises the abort flag
// status[2], which makes every other waiting block give up too, so the launch always ends.
#pragma once
#include <stdint.h>

namespace qcb {

constexpr uint64_t WAIT_NS = 2000000000ull;  // 2 s per wait
// Iteration bound of one wait, besides its time bound (a wait whose clock reads stall still
// ends): far above the iterations of a 2 s wait of L2 round trips.
constexpr uint64_t WAIT_MAX_ITERS = 1ull << 28;

// Programmatic dependent launch (sm_90+): a kernel launched with programmatic stream
// serialization may be scheduled while the previous kernel of the stream is finishing; it must
// call pdl_wait() before touching memory the previous kernel writes (the wait ends when that
// kernel has completed and its writes are visible).  pdl_launch_dependents() lets the next
// kernel be scheduled once every block of this one has issued it.
__device__ __forceinline__ void pdl_launch_dependents() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

__device__ __forceinline__ uint32_t ld_acquire_u32(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_u32(uint32_t* p, uint32_t v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// One thread waits until *p >= target.  Returns false on abort or timeout.
__device__ __forceinline__ bool wait_geq(const uint32_t* p, uint32_t target, uint32_t* status,
                                         uint64_t limit_ns = WAIT_NS) {
  if (ld_acquire_u32(p) >= target) return true;
  const uint64_t t0 = global_ns();
  for (uint64_t it = 0;; ++it) {
    if (ld_acquire_u32(p) >= target) return true;
    if (ld_acquire_u32(&status[2])) return false;
    if (global_ns() - t0 > limit_ns || it > WAIT_MAX_ITERS) {
      atomicAdd(&status[1], 1u);
      atomicExch(&status[2], 1u);
      return false;
    }
    __nanosleep(64);
  }
}

}  // namespace qcb
