// Small fronts: one warp (m <= 32, four or eight fronts per CTA) or one CTA (32 < m <= 128) per front does all of the
// front's work for its level in shared memory, in one launch per level and size class:
//   zero the front, add A's entries of the pivot columns (sparse.mjs:965-973), extend-add the children's update
//   matrices in the reference's child order (sparse.mjs:974-985), factor the nc pivot columns right-looking over the
//   whole trailing triangle (Cholesky sparse.mjs:995-1098; LDL^T with static pivot perturbation ldlt.mjs:450-562, or
//   with Bunch-Kaufman pivots inside each 64-column block of the pivot columns), and
//   write the first nc columns to L (the reference layout) and the rest to the update matrix U (the arena).
// Such fronts dominate 2D problems (the batched heat set: median m = 5, 97% with m <= 32), where the general path's
// 64 x 64 pivot-block kernels and 128-row tiles would spend almost all of their work on padding, one launch per step.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <type_traits>

#include "../host/plan.hpp"
#include "devplan.cuh"

namespace amp {

// Tiny fronts come in two size classes (sorted by m within each level by the plan): m <= kTinyMid with 8 warps per
// CTA and 16 x 16 tiles, and kTinyMid < m <= 32 with 4 warps per CTA and 32 x 32 tiles, so that the many smallest fronts
// are not held to the shared memory of the largest.
template <int MAXM>
constexpr int tiny_warps() {
  return MAXM <= kTinyMid ? 8 : 4;
}

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

// Children of one front whose metadata a group holds at a time (fetched in parallel, applied in the reference's order)
constexpr int kChildChunk = 32;
struct ChildMeta {
  int muc[kChildChunk];
  int64_t ea[kChildChunk], uo[kChildChunk];
};

// Zero F (m x m), add A's entries of the pivot columns and the children's update matrices in the reference's order.
template <class T, class TC, int G>
__device__ void assemble_front(int s, const DevPlan &P, const double *__restrict__ values, const T *__restrict__ U,
                               TC *F, int t, ChildMeta *cm) {
  const int warp = t >> 5, lane = t & 31;
  const int f = P.snF[s], nc = P.snNc[s], m = P.snM[s];
  for (int e = t; e < m * m; e += G) F[e] = TC(0);
  group_sync<G>();
  // A's entries of all nc pivot columns (one contiguous CSR range): slot dst = j m + i of the L panel, each (i, j) once
  {
    const int p0 = P.asmColPtr[f], p1 = P.asmColPtr[f + nc];
    for (int p = p0 + t; p < p1; p += G) F[P.asmDst[p]] += (TC)(T)__ldg(values + P.asmSrc[p]);
  }
  group_sync<G>();
  // children's update matrices, one after another (the map is injective within a child); the metadata of up to
  // kChildChunk children is fetched at once, one child per thread
  const int q0 = P.chPtr[s], q1 = P.chPtr[s + 1];
  for (int qb = q0; qb < q1; qb += kChildChunk) {
    const int nq = min(kChildChunk, q1 - qb);
    int muc = 0;
    int64_t ea = 0, uo = 0;
    if (warp == 0 && lane < nq) {
      const int c = P.chList[qb + lane];
      muc = P.snM[c] - P.snNc[c];
      ea = P.eaPtr[c];
      uo = P.snUoff[c];
    }
    if constexpr (G > 32) {
      if (qb > q0) __syncthreads();  // the previous chunk's metadata is read by all warps before it is replaced
      if (warp == 0 && lane < nq) {
        cm->muc[lane] = muc;
        cm->ea[lane] = ea;
        cm->uo[lane] = uo;
      }
      __syncthreads();
    }
    for (int q = 0; q < nq; q++) {
      int mq;
      int64_t eq, uq;
      if constexpr (G == 32) {
        mq = __shfl_sync(0xffffffffu, muc, q);
        eq = __shfl_sync(0xffffffffu, ea, q);
        uq = __shfl_sync(0xffffffffu, uo, q);
      } else {
        mq = cm->muc[q];
        eq = cm->ea[q];
        uq = cm->uo[q];
      }
      if (mq <= 0) continue;  // group-uniform
      const int *map = P.eaMap + eq;
      const T *Uc = U + uq;
      for (int e = t; e < mq * mq; e += G) {
        const int b = e / mq, a = e - b * mq;
        if (a >= b) F[map[b] * m + map[a]] += (TC)Uc[e];
      }
      group_sync<G>();
    }
  }
}

// The whole front of supernode s by a group of G threads (thread t) over the shared m x m column-major tile F, in the
// compute type TC (the storage type T of L and U, or FP64: an FP32 LDL^T factor's small fronts are computed in FP64
// and rounded once when stored, since the indefinite factor's pivots cancel). cm: the group's child metadata (G > 32;
// a warp passes its child metadata by shuffles).
//
// Column k of the elimination is one phase with one barrier: every thread reads the pivot F(k, k) (final since the
// previous barrier), computes the same pivot decision and scale, writes its share of L's column k straight to Lx and
// updates its share of the trailing triangle from the unscaled column k, which nobody writes in the phase. The
// arithmetic is the column-scaled form's: l_i = F(i, k) / r (Cholesky, r = sqrt F(k, k)) or F(i, k) / d (LDL^T), and
// F(i, j) -= l_i (l_j d) with d = 1 for Cholesky.
template <class T, class TC, int G>
__device__ void factor_front(int s, const DevPlan &P, const double *__restrict__ values, T *__restrict__ Lx,
                             T *__restrict__ U, TC *F, unsigned long long *status, const LdltArgs<T> &la, int t,
                             ChildMeta *cm) {
  constexpr int NW = G / 32;
  const int warp = t >> 5, lane = t & 31;
  const int f = P.snF[s], nc = P.snNc[s], m = P.snM[s], mu = m - nc;
  const bool ldlt = la.scal != nullptr;
  const TC tau = ldlt ? (TC)(T)la.scal[1] : TC(0);
  assemble_front<T, TC, G>(s, P, values, U, F, t, cm);
  // partial factorization of the nc pivot columns, one barrier per column; warps over the trailing columns j, lanes
  // over the rows i >= j
  int neg = 0, pert = 0;  // thread 0
  T *Lp = Lx + P.snLxp[s];
  for (int k = 0; k < nc; k++) {
    TC d = F[k * m + k], inv, dk, diag;
    if (ldlt) {
      int n1 = 0, p1 = 0;
      const bool ok = small_ldlt_pivot(d, tau, n1, p1);
      if (!ok) {
        if (t == 0) atomicMin(status, status_word(f + k, 2, s));
        return;  // group-uniform: every thread saw the same pivot
      }
      if (t == 0) {
        neg += n1;
        pert += p1;
        la.D[f + k] = (double)(T)d;
      }
      dk = d;
      inv = TC(1) / d;
      diag = TC(1);
    } else {
      if (!(d > TC(0))) {
        if (t == 0) atomicMin(status, status_word(f + k, 1, s));
        return;  // group-uniform
      }
      const TC r = sqrt(d);
      dk = TC(1);
      inv = TC(1) / r;
      diag = r;
    }
    const TC *Fk = F + k * m;
    T *Lk = Lp + (int64_t)k * m;
    for (int i = k + t; i < m; i += G) Lk[i] = (T)(i == k ? diag : Fk[i] * inv);
    const int w = m - k - 1;
    for (int jj = warp; jj < w; jj += NW) {
      const int j = k + 1 + jj;
      const TC lj = (Fk[j] * inv) * dk;
      TC *Fj = F + j * m;
      for (int i = j + lane; i < m; i += 32) Fj[i] -= (Fk[i] * inv) * lj;
    }
    group_sync<G>();
  }
  if (ldlt && t == 0 && (neg | pert)) {
    atomicAdd(la.counts, neg);
    atomicAdd(la.counts + 1, pert);
  }
  if (mu > 0) {
    T *Up = U + P.snUoff[s];
    for (int e = t; e < mu * mu; e += G) {
      const int jj = e / mu, ii = e - jj * mu;
      if (ii >= jj) Up[e] = (T)F[(nc + jj) * m + nc + ii];
    }
  }
}

// (value, index) of the largest value over the warp, the smallest index on ties (every lane gets the result)
__device__ __forceinline__ void front_warp_argmax(double &v, int &i) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const double ov = __shfl_xor_sync(0xffffffffu, v, o);
    const int oi = __shfl_xor_sync(0xffffffffu, i, o);
    if (ov > v || (ov == v && oi < i)) {
      v = ov;
      i = oi;
    }
  }
}

// The whole front with Bunch-Kaufman pivots inside each 64-column block of its pivot columns (AMP_LDLT_BK; the rule,
// the 2 x 2 inverse and the outputs of bk_block in factor_f64.cu), FP64 arithmetic. At column k of block [c0, c1):
// colmax and rowmax over the block's rows only, computed by every warp with shuffles (the same values in the same
// order, so every thread takes the same decision without sharing it); the interchange applied in lower storage to
// the block's earlier columns (their rows) and to the whole trailing triangle (rows below the pivot columns
// included); the rank-1 or rank-2 update of the trailing triangle from the unscaled column(s); then the column(s)
// scaled in place to L. Three barriers per step. A block's L columns go to Lx once the block is done (its later
// steps may still interchange their rows), with its pivot order; D and D(k + 1, k) as they are decided. A column
// with no usable entry in its block keeps the static perturbation to +-tau (counted); a non-finite pivot fails.
template <class T, int G>
__device__ void factor_front_bk(int s, const DevPlan &P, const double *__restrict__ values, T *__restrict__ Lx,
                                T *__restrict__ U, double *F, unsigned long long *status, const LdltArgs<T> &la,
                                int t, ChildMeta *cm) {
  constexpr int NW = G / 32;
  const int warp = t >> 5, lane = t & 31;
  const int f = P.snF[s], nc = P.snNc[s], m = P.snM[s], mu = m - nc;
  const double tau = la.scal[1];
  const double alpha = 0.64038820320220756;  // (1 + sqrt(17)) / 8
  assemble_front<T, double, G>(s, P, values, U, F, t, cm);
  auto at = [&](int i, int j) -> double & { return F[j * m + i]; };  // entry (i, j), i >= j
  int neg = 0, pert = 0;  // thread 0
  int perm[64];           // thread 0: the current block's pivot order
  T *Lp = Lx + P.snLxp[s];
  for (int c0 = 0; c0 < nc; c0 += 64) {
    const int c1 = min(nc, c0 + 64);
    if (t == 0)
      for (int i = 0; i < c1 - c0; i++) perm[i] = i;
    for (int k = c0; k < c1;) {
      double cmx = -1.0;
      int im = -1;
      for (int i = k + 1 + lane; i < c1; i += 32) {
        const double a = fabs(at(i, k));
        if (a > cmx) {
          cmx = a;
          im = i;
        }
      }
      front_warp_argmax(cmx, im);
      const double colmax = cmx > 0.0 ? cmx : 0.0, absakk = fabs(at(k, k));
      int step = 1, kp = k;
      if (colmax > 0.0 && !(absakk >= alpha * colmax)) {
        double rm = 0.0;
        for (int j = k + lane; j < c1; j += 32)
          if (j != im) rm = fmax(rm, fabs(j > im ? at(j, im) : at(im, j)));
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) rm = fmax(rm, __shfl_xor_sync(0xffffffffu, rm, o));
        if (absakk * rm >= alpha * colmax * colmax) {
          kp = k;
        } else if (fabs(at(im, im)) >= alpha * rm) {
          kp = im;
        } else {
          step = 2;
          kp = im;
        }
      }
      const int kk = k + step - 1;
      if (kp != kk) {  // interchange p = kk and r = kp (p < r), lower storage
        const int p = kk, r = kp, nBelow = m - r - 1, nMid = r - p - 1, nLeft = p - c0;
        for (int e = t; e < 1 + nBelow + nMid + nLeft; e += G) {
          double *x, *y;
          if (e == 0) {
            x = &at(p, p);
            y = &at(r, r);
          } else if (e <= nBelow) {
            x = &at(r + e, p);
            y = &at(r + e, r);
          } else if (e <= nBelow + nMid) {
            const int i = p + (e - nBelow);
            x = &at(i, p);
            y = &at(r, i);
          } else {
            const int j = c0 + (e - nBelow - nMid - 1);
            x = &at(p, j);
            y = &at(r, j);
          }
          const double tmp = *x;
          *x = *y;
          *y = tmp;
        }
        if (t == 0) {
          const int tmp = perm[p - c0];
          perm[p - c0] = perm[r - c0];
          perm[r - c0] = tmp;
        }
        group_sync<G>();
      }
      if (step == 1) {
        double d = at(k, k);
        const bool small = !(fabs(d) >= tau);
        if (small && isfinite(d)) d = d < 0.0 ? -tau : tau;
        if (!isfinite(d)) {
          if (t == 0) atomicMin(status, status_word(f + k, 2, s));
          return;  // group-uniform
        }
        if (t == 0) {
          neg += d < 0.0 ? 1 : 0;
          pert += small ? 1 : 0;
          la.D[f + k] = d;
          la.Doff[f + k] = 0.0;
        }
        const double inv = 1.0 / d;
        for (int jj = warp; jj < m - k - 1; jj += NW) {
          const int j = k + 1 + jj;
          const double lj = at(j, k);
          for (int i = j + lane; i < m; i += 32) at(i, j) -= (at(i, k) * inv) * lj;
        }
        group_sync<G>();
        for (int i = k + 1 + t; i < m; i += G) at(i, k) *= inv;  // L(i, k)
        group_sync<G>();
      } else {
        // D_k = e [[a, 1], [1, c]], D_k^-1 = (t / e) [[c, -1], [-1, a]] with a = d11 / e, c = d22 / e, t = 1 / (a c - 1)
        const double d11 = at(k, k), e21 = at(k + 1, k), d22 = at(k + 1, k + 1);
        const double a = d11 / e21, c = d22 / e21, te = (1.0 / (a * c - 1.0)) / e21;
        if (!(isfinite(te) && isfinite(a) && isfinite(c))) {
          if (t == 0) atomicMin(status, status_word(f + k, 2, s));
          return;  // group-uniform
        }
        if (t == 0) {
          neg += a * c - 1.0 < 0.0 ? 1 : (d11 < 0.0 ? 2 : 0);
          la.D[f + k] = d11;
          la.D[f + k + 1] = d22;
          la.Doff[f + k] = e21;
          la.Doff[f + k + 1] = 0.0;
        }
        for (int jj = warp; jj < m - k - 2; jj += NW) {
          const int j = k + 2 + jj;
          const double pj = at(j, k), qj = at(j, k + 1);
          for (int i = j + lane; i < m; i += 32) {
            const double pi = at(i, k), qi = at(i, k + 1);
            at(i, j) -= te * (c * pi - qi) * pj + te * (a * qi - pi) * qj;
          }
        }
        group_sync<G>();
        for (int i = k + 2 + t; i < m; i += G) {
          const double pi = at(i, k), qi = at(i, k + 1);
          at(i, k) = te * (c * pi - qi);      // L(i, k)
          at(i, k + 1) = te * (a * qi - pi);  // L(i, k + 1)
        }
        if (t == 0) at(k + 1, k) = 0.0;  // L(k + 1, k)
        group_sync<G>();
      }
      k += step;
    }
    for (int j = c0; j < c1; j++)  // the block's L columns, unit diagonal, rows in the block's pivot order
      for (int i = j + t; i < m; i += G) Lp[(int64_t)j * m + i] = (T)(i == j ? 1.0 : at(i, j));
    if (t == 0)
      for (int i = 0; i < c1 - c0; i++) la.piv[f + c0 + i] = perm[i];
  }
  if (t == 0 && (neg | pert)) {
    atomicAdd(la.counts, neg);
    atomicAdd(la.counts + 1, pert);
  }
  if (mu > 0) {
    T *Up = U + P.snUoff[s];
    for (int e = t; e < mu * mu; e += G) {
      const int jj = e / mu, ii = e - jj * mu;
      if (ii >= jj) Up[e] = (T)F[(nc + jj) * m + nc + ii];
    }
  }
}

// m <= MAXM (16 or 32): one warp per front, tiny_warps<MAXM>() fronts per CTA
// BK: Bunch-Kaufman pivots (FP64 factors with la.piv set)
template <class T, class TC, int MAXM, bool BK>
__global__ void __launch_bounds__(32 * tiny_warps<MAXM>()) k_front_tiny(const int *__restrict__ fronts, int count,
                                                                         DevPlan P, const double *__restrict__ values,
                                                                         T *__restrict__ Lx, T *__restrict__ U,
                                                                         unsigned long long *status, LdltArgs<T> la) {
  constexpr int W = tiny_warps<MAXM>();
  __shared__ TC F[W][MAXM * MAXM];
  if (status_failed(status)) return;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int idx = blockIdx.x * W + warp;
  if (idx >= count) return;  // warp-uniform; no CTA-wide barrier follows
  if constexpr (BK)
    factor_front_bk<T, 32>(fronts[idx], P, values, Lx, U, F[warp], status, la, lane, nullptr);
  else
    factor_front<T, TC, 32>(fronts[idx], P, values, Lx, U, F[warp], status, la, lane, nullptr);
}

// 32 < m <= 128: one CTA per front; dynamic shared memory = the launch's largest m squared
template <class T, class TC, bool BK>
__global__ void __launch_bounds__(256) k_front_small(const int *__restrict__ fronts, int count, DevPlan P,
                                                     const double *__restrict__ values, T *__restrict__ Lx,
                                                     T *__restrict__ U, unsigned long long *status, LdltArgs<T> la) {
  extern __shared__ __align__(16) unsigned char fs_dyn[];
  __shared__ ChildMeta cm;
  if (status_failed(status)) return;
  if constexpr (BK)
    factor_front_bk<T, 256>(fronts[blockIdx.x], P, values, Lx, U, reinterpret_cast<double *>(fs_dyn), status, la,
                            threadIdx.x, &cm);
  else
    factor_front<T, TC, 256>(fronts[blockIdx.x], P, values, Lx, U, reinterpret_cast<TC *>(fs_dyn), status, la,
                             threadIdx.x, &cm);
}

cudaError_t init_front_small_attributes() {
  cudaError_t e = cudaFuncSetAttribute(k_front_small<double, double, false>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       kSmallFront * kSmallFront * (int)sizeof(double));
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_front_small<float, float, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             kSmallFront * kSmallFront * (int)sizeof(float));
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_front_small<float, double, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             kSmallFront * kSmallFront * (int)sizeof(double));
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_front_small<double, double, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             kSmallFront * kSmallFront * (int)sizeof(double));
  return e;
}

template <class T, class TC, int MAXM, bool BK>
static int launch_tiny(const int *fronts, int count, const DevPlan &P, const double *values, T *Lx, T *U,
                       unsigned long long *status, const LdltArgs<T> &la, cudaStream_t st) {
  constexpr int W = tiny_warps<MAXM>();
  if (count <= 0) return 0;
  k_front_tiny<T, TC, MAXM, BK><<<(count + W - 1) / W, 32 * W, 0, st>>>(fronts, count, P, values, Lx, U, status,
                                                                        la);
  return 1;
}

template <class T, class TC, bool BK>
static int launch_fronts_tc(const int *tiny, int ntiny, int ntinyMid, const int *small, int nsmall, int maxM,
                            const DevPlan &P, const double *values, T *Lx, T *U, unsigned long long *status,
                            const LdltArgs<T> &la, cudaStream_t st) {
  int k = launch_tiny<T, TC, kTinyMid, BK>(tiny, ntinyMid, P, values, Lx, U, status, la, st);
  k += launch_tiny<T, TC, kTinyFront, BK>(tiny + ntinyMid, ntiny - ntinyMid, P, values, Lx, U, status, la, st);
  if (nsmall > 0)
    k_front_small<T, TC, BK><<<nsmall, 256, (size_t)maxM * maxM * sizeof(TC), st>>>(small, nsmall, P, values, Lx, U,
                                                                                    status, la);
  return k + (nsmall > 0 ? 1 : 0);
}
template <class T>
int launch_fronts_small(const int *tiny, int ntiny, int ntinyMid, const int *small, int nsmall, int maxM,
                        const DevPlan &P, const double *values, T *Lx, T *U, unsigned long long *status,
                        const LdltArgs<T> &la, cudaStream_t st) {
  if constexpr (std::is_same<T, double>::value)
    if (la.piv != nullptr)  // Bunch-Kaufman pivots (FP64)
      return launch_fronts_tc<T, double, true>(tiny, ntiny, ntinyMid, small, nsmall, maxM, P, values, Lx, U, status,
                                               la, st);
  if (la.scal != nullptr)  // LDL^T: FP64 arithmetic whatever the storage
    return launch_fronts_tc<T, double, false>(tiny, ntiny, ntinyMid, small, nsmall, maxM, P, values, Lx, U, status,
                                              la, st);
  return launch_fronts_tc<T, T, false>(tiny, ntiny, ntinyMid, small, nsmall, maxM, P, values, Lx, U, status, la, st);
}
template int launch_fronts_small<double>(const int *, int, int, const int *, int, int, const DevPlan &,
                                         const double *, double *, double *, unsigned long long *,
                                         const LdltArgs<double> &, cudaStream_t);
template int launch_fronts_small<float>(const int *, int, int, const int *, int, int, const DevPlan &,
                                        const double *, float *, float *, unsigned long long *,
                                        const LdltArgs<float> &, cudaStream_t);

}  // namespace amp
