// Small fronts: one warp (m <= 32, four fronts per CTA) or one CTA (32 < m <= 128) per front does all of the front's
// work for its level in shared memory, in one launch per level and size class:
//   zero the front, add A's entries of the pivot columns (sparse.mjs:965-973), extend-add the children's update
//   matrices in the reference's child order (sparse.mjs:974-985), factor the nc pivot columns right-looking over the
//   whole trailing triangle (Cholesky sparse.mjs:995-1098; LDL^T with static pivot perturbation ldlt.mjs:450-562), and
//   write the first nc columns to L (the reference layout) and the rest to the update matrix U (the arena).
// Such fronts dominate 2D problems (the batched heat set: median m = 5, 97% with m <= 32), where the general path's
// 64 x 64 pivot-block kernels and 128-row tiles would spend almost all of their work on padding, one launch per step.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "../host/plan.hpp"
#include "devplan.cuh"

namespace amp {

constexpr int kTinyWarps = 4;  // tiny fronts per CTA

template <int G>
__device__ __forceinline__ void group_sync() {
  if constexpr (G == 32)
    __syncwarp();
  else
    __syncthreads();
}

__device__ __forceinline__ bool status_failed(const unsigned long long *st) {
  return *(volatile const unsigned long long *)st != kStatusOk;
}

// |d| < tau (or NaN) becomes -tau / +tau by the sign of d; a non-finite small pivot fails (ldlt.mjs:513-522)
template <class T>
__device__ __forceinline__ bool small_ldlt_pivot(T &d, T tau, int &neg, int &pert) {
  if (!(fabs(d) >= tau)) {
    if (!isfinite(d)) return false;
    d = d < T(0) ? -tau : tau;
    pert++;
  }
  if (d < T(0)) neg++;
  return true;
}

// The whole front of supernode s by a group of G threads (thread t) over the shared m x m column-major tile F, in the
// compute type TC (the storage type T of L and U, or FP64: an FP32 LDL^T factor's small fronts are computed in FP64
// and rounded once when stored, since the indefinite factor's pivots cancel). pv / flag: the group's shared scalars.
template <class T, class TC, int G>
__device__ void factor_front(int s, const DevPlan &P, const double *__restrict__ values, T *__restrict__ Lx,
                             T *__restrict__ U, TC *F, unsigned long long *status, const LdltArgs<T> &la, int t,
                             TC *pv, int *flag) {
  const int f = P.snF[s], nc = P.snNc[s], m = P.snM[s], mu = m - nc;
  const bool ldlt = la.scal != nullptr;
  const TC tau = ldlt ? (TC)(T)la.scal[1] : TC(0);
  for (int e = t; e < m * m; e += G) F[e] = TC(0);
  if (t == 0) *flag = 0;
  group_sync<G>();
  // A's entries of the pivot columns: slot dst = j m + i of the L panel, each (i, j) once
  for (int j = 0; j < nc; j++) {
    const int p0 = P.asmColPtr[f + j], p1 = P.asmColPtr[f + j + 1];
    for (int p = p0 + t; p < p1; p += G) F[P.asmDst[p]] += (TC)(T)__ldg(values + P.asmSrc[p]);
  }
  group_sync<G>();
  // children's update matrices, one after another (the map is injective within a child)
  for (int q = P.chPtr[s]; q < P.chPtr[s + 1]; q++) {
    const int c = P.chList[q];
    const int muc = P.snM[c] - P.snNc[c];
    if (muc <= 0) continue;
    const int *map = P.eaMap + P.eaPtr[c];
    const T *Uc = U + P.snUoff[c];
    for (int e = t; e < muc * muc; e += G) {
      const int b = e / muc, a = e - b * muc;
      if (a >= b) F[map[b] * m + map[a]] += (TC)Uc[e];
    }
    group_sync<G>();
  }
  // partial factorization of the nc pivot columns; the trailing triangle (pivot columns and U) updated per column
  int neg = 0, pert = 0;  // thread 0
  for (int k = 0; k < nc; k++) {
    if (t == 0) {
      TC d = F[k * m + k];
      int bad = 0;
      if (ldlt) {
        if (!small_ldlt_pivot(d, tau, neg, pert)) bad = 2;
        la.D[f + k] = (double)(T)d;
        pv[0] = d;
        pv[1] = TC(1) / d;
        F[k * m + k] = TC(1);
      } else {
        if (!(d > TC(0))) bad = 1;
        const TC r = sqrt(d);
        pv[0] = TC(1);
        pv[1] = TC(1) / r;
        F[k * m + k] = r;
      }
      if (bad) {
        atomicMin(status, status_word(f + k, bad, s));
        *flag = 1;
      }
    }
    group_sync<G>();
    if (*flag) return;  // group-uniform
    const TC inv = pv[1], dk = pv[0];
    TC *Fk = F + k * m;
    for (int i = k + 1 + t; i < m; i += G) Fk[i] *= inv;
    group_sync<G>();
    const int w = m - k - 1;
    for (int e = t; e < w * w; e += G) {
      const int jj = e / w, ii = e - jj * w;
      if (ii >= jj) {
        const int i = k + 1 + ii, j = k + 1 + jj;
        F[j * m + i] -= Fk[i] * (Fk[j] * dk);
      }
    }
    group_sync<G>();
  }
  if (ldlt && t == 0 && (neg | pert)) {
    atomicAdd(la.counts, neg);
    atomicAdd(la.counts + 1, pert);
  }
  T *Lp = Lx + P.snLxp[s];
  for (int e = t; e < nc * m; e += G) {
    const int j = e / m, i = e - j * m;
    if (i >= j) Lp[e] = (T)F[e];
  }
  if (mu > 0) {
    T *Up = U + P.snUoff[s];
    for (int e = t; e < mu * mu; e += G) {
      const int jj = e / mu, ii = e - jj * mu;
      if (ii >= jj) Up[e] = (T)F[(nc + jj) * m + nc + ii];
    }
  }
}

// m <= 32: one warp per front, kTinyWarps fronts per CTA
template <class T, class TC>
__global__ void __launch_bounds__(32 * kTinyWarps) k_front_tiny(const int *__restrict__ fronts, int count, DevPlan P,
                                                                const double *__restrict__ values, T *__restrict__ Lx,
                                                                T *__restrict__ U, unsigned long long *status,
                                                                LdltArgs<T> la) {
  __shared__ TC F[kTinyWarps][kTinyFront * kTinyFront];
  __shared__ TC pv[kTinyWarps][2];
  __shared__ int flag[kTinyWarps];
  if (status_failed(status)) return;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int idx = blockIdx.x * kTinyWarps + warp;
  if (idx >= count) return;  // warp-uniform; no CTA-wide barrier follows
  factor_front<T, TC, 32>(fronts[idx], P, values, Lx, U, F[warp], status, la, lane, pv[warp], &flag[warp]);
}

// 32 < m <= 128: one CTA per front; dynamic shared memory = the launch's largest m squared
template <class T, class TC>
__global__ void __launch_bounds__(256) k_front_small(const int *__restrict__ fronts, int count, DevPlan P,
                                                     const double *__restrict__ values, T *__restrict__ Lx,
                                                     T *__restrict__ U, unsigned long long *status, LdltArgs<T> la) {
  extern __shared__ __align__(16) unsigned char fs_dyn[];
  __shared__ TC pv[2];
  __shared__ int flag;
  if (status_failed(status)) return;
  factor_front<T, TC, 256>(fronts[blockIdx.x], P, values, Lx, U, reinterpret_cast<TC *>(fs_dyn), status, la,
                           threadIdx.x, pv, &flag);
}

void init_front_small_attributes() {
  cudaFuncSetAttribute(k_front_small<double, double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       kSmallFront * kSmallFront * (int)sizeof(double));
  cudaFuncSetAttribute(k_front_small<float, float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       kSmallFront * kSmallFront * (int)sizeof(float));
  cudaFuncSetAttribute(k_front_small<float, double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       kSmallFront * kSmallFront * (int)sizeof(double));
}

template <class T, class TC>
static void launch_fronts_tc(const int *tiny, int ntiny, const int *small, int nsmall, int maxM, const DevPlan &P,
                             const double *values, T *Lx, T *U, unsigned long long *status, const LdltArgs<T> &la,
                             cudaStream_t st) {
  if (ntiny > 0)
    k_front_tiny<T, TC><<<(ntiny + kTinyWarps - 1) / kTinyWarps, 32 * kTinyWarps, 0, st>>>(tiny, ntiny, P, values, Lx,
                                                                                           U, status, la);
  if (nsmall > 0)
    k_front_small<T, TC><<<nsmall, 256, (size_t)maxM * maxM * sizeof(TC), st>>>(small, nsmall, P, values, Lx, U,
                                                                                status, la);
}
template <class T>
void launch_fronts_small(const int *tiny, int ntiny, const int *small, int nsmall, int maxM, const DevPlan &P,
                         const double *values, T *Lx, T *U, unsigned long long *status, const LdltArgs<T> &la,
                         cudaStream_t st) {
  if (la.scal != nullptr)  // LDL^T: FP64 arithmetic whatever the storage
    launch_fronts_tc<T, double>(tiny, ntiny, small, nsmall, maxM, P, values, Lx, U, status, la, st);
  else
    launch_fronts_tc<T, T>(tiny, ntiny, small, nsmall, maxM, P, values, Lx, U, status, la, st);
}
template void launch_fronts_small<double>(const int *, int, const int *, int, int, const DevPlan &, const double *,
                                          double *, double *, unsigned long long *, const LdltArgs<double> &,
                                          cudaStream_t);
template void launch_fronts_small<float>(const int *, int, const int *, int, int, const DevPlan &, const double *,
                                         float *, float *, unsigned long long *, const LdltArgs<float> &, cudaStream_t);

}  // namespace amp
