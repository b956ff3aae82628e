// Inter-CTA ordering of the persistent solve sweeps: epoch-stamped ready flags and completion counters in global
// memory, written with release and read with acquire semantics at GPU scope, and bounded waits on them. A wait that
// runs out records a device time-out in the status word (read by the host after the sweep) and returns false, so the
// CTA leaves instead of hanging.
#pragma once
#include <cuda_runtime.h>

#include "devplan.cuh"

namespace amp {


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

// Tagged words: the high 32 bits carry the sweep's epoch, the low 32 bits half of a double. A strong 8-byte store is
// seen whole, so a reader that finds its epoch in the tag holds the value without a separate flag round trip.
__device__ __forceinline__ unsigned long long ld_relaxed_u64(const unsigned long long *p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_relaxed_u64(unsigned long long *p, unsigned long long v) {
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
// the two tagged words of x: the low half, then the high half
__device__ __forceinline__ void st_tagged(unsigned long long *p, int epoch, double x) {
  const unsigned long long u = (unsigned long long)__double_as_longlong(x), tag = (unsigned long long)(unsigned)epoch
                                                                                    << 32;
  st_relaxed_u64(p, tag | (u & 0xffffffffull));
  st_relaxed_u64(p + 1, tag | (u >> 32));
}
__device__ __forceinline__ double untag(unsigned lo, unsigned hi) {
  return __longlong_as_double((long long)(((unsigned long long)hi << 32) | lo));
}

// The waits below poll at most `limit` times (DevPlan::spin: kSpinLimit unless the caller set a bound).

// Wait until the tag of *w is epoch and return its low 32 bits in lo; false on time-out (status set for s).
__device__ __forceinline__ bool wait_tagged(const unsigned long long *w, int epoch, unsigned long long *status, int s,
                                            unsigned &lo, long long limit) {
  long long spins = 0;
  unsigned long long v;
  while (((v = ld_relaxed_u64(w)) >> 32) != (unsigned long long)(unsigned)epoch) {
    if (++spins > limit) {
      atomicMin(status, status_word(0x7fffffff, 3, s));
      return false;
    }
    __nanosleep(32);
  }
  lo = (unsigned)v;
  return true;
}

// Wait until *flag == epoch; false on time-out (status set for supernode s).
__device__ __forceinline__ bool wait_flag(const int *flag, int epoch, unsigned long long *status, int s,
                                          long long limit) {
  long long spins = 0;
  while (ld_acquire(flag) != epoch) {
    if (++spins > limit) {
      atomicMin(status, status_word(0x7fffffff, 3, s));
      return false;
    }
    __nanosleep(32);
  }
  return true;
}

// Wait until *cnt >= need; false on time-out (status set for supernode s).
__device__ __forceinline__ bool wait_count(const int *cnt, int need, unsigned long long *status, int s,
                                           long long limit) {
  long long spins = 0;
  while (ld_acquire(cnt) < need) {
    if (++spins > limit) {
      atomicMin(status, status_word(0x7fffffff, 3, s));
      return false;
    }
    __nanosleep(32);
  }
  return true;
}

}  // namespace amp
