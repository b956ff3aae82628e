// Device-side view of a plan (plain pointers into device memory; passed by value to every kernel).
#pragma once
#include <cstdint>

namespace amp {

struct DevPlan {
  int n, nsuper, maxFront;
  const int *snF, *snNc, *snM, *snParent;
  const int64_t *snLxp, *snUoff, *snTOff, *snSp;
  const int *chPtr, *chList;
  const int *asmColPtr, *asmDst, *asmSrc;
  const int64_t *eaPtr;
  const int *eaMap;
  const int *lvlSn;
  const int *perm, *Sp, *Si;
  const int *blkOff;       // first 64-column diagonal block of supernode s (nsuper + 1)
  const int64_t *invOff;   // offset of the inverse of each diagonal block (w x w, column-major)
};

// Failure record: the lowest failing global column wins (atomicMin), code in the low bits.
// kStatusOk means no failure. code 1: Cholesky pivot not > 0; code 2: non-finite LDL^T pivot; code 3: device timeout.
constexpr unsigned long long kStatusOk = ~0ull;
__host__ __device__ inline unsigned long long status_word(int col, int code, int sn) {
  return ((unsigned long long)(unsigned)col << 32) | ((unsigned long long)(unsigned)(code & 0xff) << 24) |
         (unsigned long long)((unsigned)sn & 0xffffffu);
}

}  // namespace amp
