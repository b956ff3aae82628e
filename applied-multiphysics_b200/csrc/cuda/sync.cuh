// Inter-CTA ordering of the persistent solve sweeps: epoch-stamped ready flags and completion counters in global
// memory, written with release and read with acquire semantics at GPU scope, and bounded waits on them. A wait that
// runs out records a device time-out in the status word (read by the host after the sweep) and returns false, so the
// CTA leaves instead of hanging.
#pragma once
#include <cuda_runtime.h>

#include "devplan.cuh"

namespace amp {

constexpr long long kSpinLimit = 1ll << 24;  // ~ seconds with the back-off below

__device__ __forceinline__ int ld_acquire(const int *p) {
  int v;
  asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release(int *p, int v) {
  asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void red_release_add(int *p, int v) {
  asm volatile("red.release.gpu.global.add.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Wait until *flag == epoch; false on time-out (status set for supernode s).
__device__ __forceinline__ bool wait_flag(const int *flag, int epoch, unsigned long long *status, int s) {
  long long spins = 0;
  while (ld_acquire(flag) != epoch) {
    if (++spins > kSpinLimit) {
      atomicMin(status, status_word(0x7fffffff, 3, s));
      return false;
    }
    __nanosleep(32);
  }
  return true;
}

// Wait until *cnt >= need; false on time-out (status set for supernode s).
__device__ __forceinline__ bool wait_count(const int *cnt, int need, unsigned long long *status, int s) {
  long long spins = 0;
  while (ld_acquire(cnt) < need) {
    if (++spins > kSpinLimit) {
      atomicMin(status, status_word(0x7fffffff, 3, s));
      return false;
    }
    __nanosleep(32);
  }
  return true;
}

}  // namespace amp
