// Device-side view of a plan (plain pointers into device memory; passed by value to every kernel).
#pragma once
#include <cuda_bf16.h>

#include <cstdint>

#include "cplx.cuh"

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
  const int *rowBlk;       // 64-column diagonal block holding column i (n; the flag a backward reader of row i waits for)
  const int64_t *invOff;   // offset of the inverse of each diagonal block (w x w, column-major)
  const int *diagSlot;     // CSR slot of A(i, i), original row i (the LDL^T pivot scale)
  const int *solveSmall;   // supernodes solved whole by one warp (solve tasks of kind 2 index this list)
  long long spin;          // bound of every inter-CTA wait of the solve sweeps, in polls (kSpinLimit by default)
  // Bunch-Kaufman LDL^T factor (null otherwise): the pivot order inside every 64-column pivot block of every
  // supernode, lpiv[f + c0 + i] = the block column (0..63) that became pivot i. Set per factor for its solves.
  const int *lpiv;
};

// LDL^T variant of the panel and update kernels (ldlt.mjs:450-562); all null for Cholesky.
template <class T>
struct LdltArgs {
  using DT = value_of<T>;  // type of the stored pivots: FP64 (real factors, FP32 ones too) or complex
  const double *scal;  // [0] pivotTol (copied per factorization), [1] tau = pivotTol * max |A(i, i)| (device)
  int *counts;         // [0] nNeg, [1] nPerturbed
  T *W;                // L21 D (rows of the solved panel times the pivots): the A operand of the FP64 update
  DT *D;               // the pivots, permuted order
  __nv_bfloat16 *Whi, *Wlo;  // mixed precision: BF16 split of L21 D (the A operand of the tensor-core update)
  // Bunch-Kaufman pivoting inside each 64-column pivot block (null: static perturbation as the reference):
  // piv[f + c0 + i] = the block column (0..63) that became pivot i; Doff[j] = D(j + 1, j) when (j, j + 1) is a 2 x 2
  // pivot, else 0 (D[j] holds the diagonal of both 1 x 1 and 2 x 2 pivots)
  int *piv;
  DT *Doff;
};

// Default bound of an inter-CTA wait of the solve sweeps, in polls (about a second with their back-off).
constexpr long long kSpinLimit = 1ll << 24;

// Failure record: the lowest failing global column wins (atomicMin), code in the low bits.
// kStatusOk means no failure. code 1: Cholesky pivot not > 0; code 2: non-finite LDL^T pivot; code 3: device timeout.
constexpr unsigned long long kStatusOk = ~0ull;
__host__ __device__ inline unsigned long long status_word(int col, int code, int sn) {
  return ((unsigned long long)(unsigned)col << 32) | ((unsigned long long)(unsigned)(code & 0xff) << 24) |
         (unsigned long long)((unsigned)sn & 0xffffffu);
}

}  // namespace amp
