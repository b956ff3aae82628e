// Solves of supernodes with m <= 32 by one warp each (solve tasks of kind 2), one right-hand side (lane = front row)
// or several interleaved ones (lane = vector, the front vectors in shared memory). Forward: gather the front vector
// (y rows of the pivot columns, the children's pass-up vectors in the reference's child order), eliminate column by
// column (y_k = v_k / L(k, k), v_i -= L(i, k) y_k), write y and the pass-up vector and count the supernode done.
// Backward: gather the rows below from the ancestors' final values, then x_k = (r_k - sum_{i > k} L(i, k) x_i) /
// L(k, k) from the last column down (r = y, divided by D for LDL^T, whose stored L(k, k) is 1), and release the
// supernode's block flag. Waits are bounded (status set on time-out). A Bunch-Kaufman factor (P.lpiv set) takes the
// pivot rows in its pivot order after the gather and writes x back to their original rows (its D solve runs between
// the sweeps).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "../host/plan.hpp"
#include "devplan.cuh"
#include "sync.cuh"

namespace amp {

// lane 0 waits (bounded) until *p == v (eq) or *p >= v; the result is broadcast to the warp, and the warp barrier
// orders the other lanes' later loads after lane 0's acquire
__device__ __forceinline__ bool warp_wait(const int *p, int v, bool eq, unsigned long long *status, int s,
                                          long long limit) {
  int ok = 1;
  if ((threadIdx.x & 31) == 0) ok = eq ? wait_flag(p, v, status, s, limit) : wait_count(p, v, status, s, limit);
  ok = __shfl_sync(0xffffffffu, ok, 0);
  __syncwarp();
  return ok != 0;
}

// children of s complete in the forward sweep (their pass-up vectors written)
__device__ __forceinline__ bool warp_wait_children(const DevPlan &P, int s, const int *done,
                                                   unsigned long long *status) {
  for (int qq = P.chPtr[s]; qq < P.chPtr[s + 1]; qq++) {
    const int c = P.chList[qq];
    const int need = (P.snM[c] - P.snNc[c] + 63) / 64;
    if (!warp_wait(done + c, need, false, status, s, P.spin)) return false;
  }
  return true;
}

// ---- one right-hand side --------------------------------------------------------------------------------------------
// vs: the warp's 32 doubles of shared memory
template <class TL>
__device__ bool small_fwd_warp(int s, const DevPlan &P, const TL *__restrict__ Lx, double *__restrict__ y,
                               double *__restrict__ T, int *done, unsigned long long *status, double *vs) {
  const int lane = threadIdx.x & 31;
  const int f = P.snF[s], nc = P.snNc[s], m = P.snM[s];
  if (!warp_wait_children(P, s, done, status)) return false;
  vs[lane] = lane < nc ? y[f + lane] : 0.0;
  __syncwarp();
  for (int qq = P.chPtr[s]; qq < P.chPtr[s + 1]; qq++) {
    const int c = P.chList[qq];
    const int muc = P.snM[c] - P.snNc[c];
    const int *map = P.eaMap + P.eaPtr[c];
    const double *tc = T + P.snTOff[c];
    for (int a = lane; a < muc; a += 32) vs[map[a]] += __ldcg(tc + a);
    __syncwarp();
  }
  double v = vs[lane];
  if (P.lpiv) v = __shfl_sync(0xffffffffu, v, lane < nc ? P.lpiv[f + lane] : lane);  // Bunch-Kaufman pivot order
  const TL *Lp = Lx + P.snLxp[s];
  double lk = lane < m ? (double)Lp[lane] : 0.0;  // column 0
  for (int k = 0; k < nc; k++) {
    const double ln = (k + 1 < nc && lane < m) ? (double)Lp[(int64_t)(k + 1) * m + lane] : 0.0;
    const double yk = __shfl_sync(0xffffffffu, lane == k ? v / lk : 0.0, k);
    if (lane == k)
      v = yk;
    else if (lane > k)
      v -= lk * yk;
    lk = ln;
  }
  if (lane < nc)
    y[f + lane] = v;
  else if (lane < m)
    T[P.snTOff[s] + lane - nc] = v;
  __syncwarp();  // orders the warp's stores before the counted arrival
  if (lane == 0) red_release_add(done + s, 1);
  return true;
}

template <class TL>
__device__ bool small_bwd_warp(int s, const DevPlan &P, const TL *__restrict__ Lx, const double *__restrict__ Dpiv,
                               double *__restrict__ y, int *flags, int epoch, unsigned long long *status) {
  const int lane = threadIdx.x & 31;
  const int f = P.snF[s], nc = P.snNc[s], m = P.snM[s];
  const int par = P.snParent[s];
  if (par >= 0 && m > nc && !warp_wait(flags + P.blkOff[par], epoch, true, status, s, P.spin)) return false;
  double x = 0.0;
  if (lane >= nc && lane < m) {
    x = __ldcg(y + P.Si[P.Sp[s] + lane]);
  } else if (lane < nc) {
    x = y[f + lane];
    if (Dpiv) x = x / Dpiv[f + lane];  // LDL^T: y /= D before the backward sweep (ldlt.mjs:629)
  }
  const TL *Lp = Lx + P.snLxp[s];
  for (int k = nc - 1; k >= 0; k--) {
    const double lk = (lane >= k && lane < m) ? (double)Lp[(int64_t)k * m + lane] : 0.0;
    double p = lane > k ? lk * x : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) p += __shfl_xor_sync(0xffffffffu, p, o);
    if (lane == k) x = (x - p) / lk;
  }
  if (lane < nc) y[f + (P.lpiv ? P.lpiv[f + lane] : lane)] = x;  // back to the original order (Bunch-Kaufman)
  __syncwarp();  // orders the warp's stores before the release
  if (lane == 0) st_release(flags + P.blkOff[s], epoch);
  return true;
}

// ---- q interleaved right-hand sides (q <= 64; lane l holds vectors l and l + 32) -------------------------------------
// Vs: the warp's 32 x 64 doubles of shared memory, row r of the front vectors at Vs[64 r + k]
template <class TL>
__device__ bool small_fwd_warp_multi(int s, const DevPlan &P, const TL *__restrict__ Lx, double *__restrict__ y,
                                     double *__restrict__ T, int *done, int q, int ns, unsigned long long *status,
                                     double *Vs) {
  const int lane = threadIdx.x & 31;
  const int f = P.snF[s], nc = P.snNc[s], m = P.snM[s];
  const int k0 = lane, k1 = lane + 32;
  const bool v0 = k0 < q, v1 = k1 < q;
  for (int sl = 0; sl < ns; sl++)  // every vector slice of the children done
    if (!warp_wait_children(P, s, done + (int64_t)sl * P.nsuper, status)) return false;
  for (int r = 0; r < m; r++) {
    if (v0) Vs[64 * r + k0] = r < nc ? y[(int64_t)(f + r) * q + k0] : 0.0;
    if (v1) Vs[64 * r + k1] = r < nc ? y[(int64_t)(f + r) * q + k1] : 0.0;
  }
  for (int qq = P.chPtr[s]; qq < P.chPtr[s + 1]; qq++) {  // each lane touches only its own vectors: no barrier
    const int c = P.chList[qq];
    const int muc = P.snM[c] - P.snNc[c];
    const int *map = P.eaMap + P.eaPtr[c];
    const double *tc = T + P.snTOff[c] * q;
    for (int a = 0; a < muc; a++) {
      const int r = map[a];
      if (v0) Vs[64 * r + k0] += __ldcg(tc + (int64_t)a * q + k0);
      if (v1) Vs[64 * r + k1] += __ldcg(tc + (int64_t)a * q + k1);
    }
  }
  if (P.lpiv) {  // Bunch-Kaufman pivot order of the pivot rows (each lane permutes its own vectors)
    double t0[kTinyFront], t1[kTinyFront];
    for (int r = 0; r < nc; r++) {
      const int src = P.lpiv[f + r];
      t0[r] = v0 ? Vs[64 * src + k0] : 0.0;
      t1[r] = v1 ? Vs[64 * src + k1] : 0.0;
    }
    for (int r = 0; r < nc; r++) {
      if (v0) Vs[64 * r + k0] = t0[r];
      if (v1) Vs[64 * r + k1] = t1[r];
    }
  }
  // column k of L is held one row per lane (loaded one column ahead) and broadcast by shuffles
  const TL *Lp = Lx + P.snLxp[s];
  double lcol = lane < m ? (double)Lp[lane] : 0.0;
  for (int k = 0; k < nc; k++) {
    const double lnext = (k + 1 < nc && lane < m) ? (double)Lp[(int64_t)(k + 1) * m + lane] : 0.0;
    const double lkk = __shfl_sync(0xffffffffu, lcol, k);
    const double y0 = v0 ? Vs[64 * k + k0] / lkk : 0.0, y1 = v1 ? Vs[64 * k + k1] / lkk : 0.0;
    if (v0) Vs[64 * k + k0] = y0;
    if (v1) Vs[64 * k + k1] = y1;
    for (int r = k + 1; r < m; r++) {
      const double l = __shfl_sync(0xffffffffu, lcol, r);
      if (v0) Vs[64 * r + k0] -= l * y0;
      if (v1) Vs[64 * r + k1] -= l * y1;
    }
    lcol = lnext;
  }
  for (int r = 0; r < m; r++) {
    double *dst = r < nc ? y + (int64_t)(f + r) * q : T + (P.snTOff[s] + r - nc) * q;
    if (v0) dst[k0] = Vs[64 * r + k0];
    if (v1) dst[k1] = Vs[64 * r + k1];
  }
  __syncwarp();
  if (lane < ns) red_release_add(done + (int64_t)lane * P.nsuper + s, 1);  // one count per vector slice
  return true;
}

template <class TL>
__device__ bool small_bwd_warp_multi(int s, const DevPlan &P, const TL *__restrict__ Lx,
                                     const double *__restrict__ Dpiv, double *__restrict__ y, int *flags, int nflags,
                                     int epoch, int q, int ns, unsigned long long *status, double *Vs) {
  const int lane = threadIdx.x & 31;
  const int f = P.snF[s], nc = P.snNc[s], m = P.snM[s];
  const int k0 = lane, k1 = lane + 32;
  const bool v0 = k0 < q, v1 = k1 < q;
  const int par = P.snParent[s];
  if (par >= 0 && m > nc)
    for (int sl = 0; sl < ns; sl++)  // the parent's every vector slice final
      if (!warp_wait(flags + (int64_t)sl * nflags + P.blkOff[par], epoch, true, status, s, P.spin)) return false;
  const int *rowsOf = P.Si + P.Sp[s];
  for (int r = 0; r < m; r++) {
    const int64_t gi = r < nc ? f + r : rowsOf[r];
    const double d = (r < nc && Dpiv) ? Dpiv[f + r] : 1.0;
    if (v0) {
      const double xv = r < nc ? y[gi * q + k0] : __ldcg(y + gi * q + k0);
      Vs[64 * r + k0] = (r < nc && Dpiv) ? xv / d : xv;
    }
    if (v1) {
      const double xv = r < nc ? y[gi * q + k1] : __ldcg(y + gi * q + k1);
      Vs[64 * r + k1] = (r < nc && Dpiv) ? xv / d : xv;
    }
  }
  // column k of L one row per lane (loaded one column ahead), broadcast by shuffles
  const TL *Lp = Lx + P.snLxp[s];
  double lcol = (nc > 0 && lane < m) ? (double)Lp[(int64_t)(nc - 1) * m + lane] : 0.0;
  for (int k = nc - 1; k >= 0; k--) {
    const double lnext = (k > 0 && lane < m) ? (double)Lp[(int64_t)(k - 1) * m + lane] : 0.0;
    double s0 = 0.0, s1 = 0.0;
    for (int r = k + 1; r < m; r++) {
      const double l = __shfl_sync(0xffffffffu, lcol, r);
      if (v0) s0 += l * Vs[64 * r + k0];
      if (v1) s1 += l * Vs[64 * r + k1];
    }
    const double lkk = __shfl_sync(0xffffffffu, lcol, k);
    lcol = lnext;
    if (v0) Vs[64 * k + k0] = (Vs[64 * k + k0] - s0) / lkk;
    if (v1) Vs[64 * k + k1] = (Vs[64 * k + k1] - s1) / lkk;
  }
  for (int r = 0; r < nc; r++) {
    const int64_t gr = f + (P.lpiv ? P.lpiv[f + r] : r);  // back to the original order (Bunch-Kaufman)
    if (v0) y[gr * q + k0] = Vs[64 * r + k0];
    if (v1) y[gr * q + k1] = Vs[64 * r + k1];
  }
  __syncwarp();
  if (lane < ns) st_release(flags + (int64_t)lane * nflags + P.blkOff[s], epoch);  // one flag per vector slice
  return true;
}

}  // namespace amp
