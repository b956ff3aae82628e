// Multifrontal numeric factorization on sm_100a: Cholesky (FP64, or FP32 fronts for the mixed-precision path) and
// LDL^T with static pivot perturbation (FP64).
//
// Per level of the supernodal tree (leaves first):
//   k_assemble  zero the front, scatter A's entries (sparse.mjs:965-973) and extend-add the children's update
//               matrices in the reference's child order (sparse.mjs:974-985). One CTA owns a block of 32 front
//               columns, so every entry has a single writer and the summation order is the reference's.
//   per group of up to kGroup pivot blocks of 64 columns:
//     k_group_panel  one dataflow launch: POTRF (or LDL^T) of each 64 x 64 pivot block in registers, the rows below
//                    it against it (TRSM, 64-row strips, one CTA each) and the update of the group's remaining
//                    columns, ordered by flags between the strips of the launch.
//     k_update       FP64 update F -= A B^T of the columns right of the group (A = L21, or L21 D for LDL^T; B = L21;
//                    K = the group) on 128 x 64 tiles with the FP64 tensor-core MMA (mma.sync m16n8k16), covering
//                    the remaining pivot columns (in Lx) and the update block (in the U arena). The mixed-precision
//                    update is k_update_mx (update_bf16x3.cu).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <type_traits>
#include <cstdint>

#include "devplan.cuh"
#include "sync.cuh"
#include "../host/plan.hpp"

namespace amp {

template <class T>
__device__ __forceinline__ T *front_addr(T *Lp, T *Up, int m, int nc, int i, int j) {
  // front entry (i, j), i >= j: first nc columns in the L panel (ld m), the rest in the U block (ld mu)
  return j < nc ? Lp + (int64_t)j * m + i : Up + (int64_t)(j - nc) * (m - nc) + (i - nc);
}

// 1/d by Newton-Raphson refinement of the FP32 reciprocal (x <- x + x (1 - d x), quadratic convergence: 2^-23 ->
// 2^-46 -> full double precision). Not correctly rounded (within a few ulp of 1/d); used only for the trailing
// update scale of the pivot block, where the factor's own rounding dominates. Finite nonzero d of either sign; other
// values take the division.
__device__ __forceinline__ double recip_nr(double d) {
  const double a = fabs(d);
  if (!(a > 1e-30 && a < 1e30)) return 1.0 / d;  // outside the float range of the first approximation
  double x = (double)__frcp_rn((float)d);
  double e = fma(-d, x, 1.0);
  x = fma(x, e, x);
  e = fma(-d, x, 1.0);
  x = fma(x, e, x);
  e = fma(-d, x, 1.0);
  return fma(x, e, x);
}

// Static pivot perturbation of LDL^T (ldlt.mjs:513-522): |d| < tau (or NaN) becomes -tau / +tau by the sign of d,
// a non-finite small pivot fails the factorization. flags: bit 0 negative pivot, bit 1 perturbed. false = failure.
template <class T>
__device__ __forceinline__ bool ldlt_pivot(T &d, T tau, unsigned char &flags) {
  flags = 0;
  if (!(fabs(d) >= tau)) {
    if (!isfinite(d)) return false;
    d = d < T(0) ? -tau : tau;
    flags = 2;
  }
  if (d < T(0)) flags |= 1;
  return true;
}

// Complex pivot of the complex-symmetric LDL^T (ldlt.mjs:715-730): a magnitude below tau (or not a number) becomes
// tau, keeping the pivot's phase (tau itself when d = 0); a non-finite small magnitude fails the factorization.
// flags: bit 1 perturbed (a complex factor has no inertia).
__device__ __forceinline__ bool ldlt_pivot(cplx &d, double tau, unsigned char &flags) {
  flags = 0;
  const double mag = hypot(d.re, d.im);
  if (!(mag >= tau)) {
    if (!isfinite(mag)) return false;
    if (mag == 0)
      d.re = tau;
    else
      d = cplx(d.re * (tau / mag), d.im * (tau / mag));
    flags = 2;
  }
  return true;
}
// magnitude of a pivot
__device__ __forceinline__ double pivot_mag(double d) { return fabs(d); }
__device__ __forceinline__ double pivot_mag(float d) { return fabs((double)d); }
__device__ __forceinline__ double pivot_mag(cplx d) { return hypot(d.re, d.im); }
// Cholesky's pivot test and diagonal (real factors only; a complex factor is always LDL^T)
template <class T>
__device__ __forceinline__ bool chol_pivot_ok(T d) { return d > T(0); }
__device__ __forceinline__ bool chol_pivot_ok(cplx) { return false; }
template <class T>
__device__ __forceinline__ T chol_sqrt(T d) { return sqrt(d); }
__device__ __forceinline__ cplx chol_sqrt(cplx d) { return d; }
// loads through L2 (data another CTA of the running launch wrote) and read-only loads, for every scalar type
__device__ __forceinline__ double ldcg_v(const double *p) { return __ldcg(p); }
__device__ __forceinline__ float ldcg_v(const float *p) { return __ldcg(p); }
__device__ __forceinline__ cplx ldcg_v(const cplx *p) {
  const double2 v = __ldcg(reinterpret_cast<const double2 *>(p));
  return cplx(v.x, v.y);
}
__device__ __forceinline__ double ldg_v(const double *p) { return __ldg(p); }
__device__ __forceinline__ cplx ldg_v(const cplx *p) {
  const double2 v = __ldg(reinterpret_cast<const double2 *>(p));
  return cplx(v.x, v.y);
}

// tau = pivotTol * max |A(i, i)| (1 when that maximum is 0 or not a number, ldlt.mjs:419-424). One CTA.
__global__ void __launch_bounds__(1024) k_ldlt_tau(const double *__restrict__ values, const int *__restrict__ diagSlot,
                                                    int n, double *scal) {
  __shared__ double red[32];
  double mx = 0.0;
  bool nan = false;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const double a = fabs(values[diagSlot[i]]);
    if (a != a) nan = true;
    mx = fmax(mx, a);
  }
  nan = __syncthreads_or(nan);
  for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = mx;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); w++) mx = fmax(mx, red[w]);
    scal[1] = scal[0] * ((mx > 0.0 && !nan) ? mx : 1.0);
  }
}

__device__ __forceinline__ bool failed(const unsigned long long *st) {
  return *(volatile const unsigned long long *)st != kStatusOk;
}

// ---------------------------------------------------------------------------------------------------------------
// Assembly + extend-add
// ---------------------------------------------------------------------------------------------------------------
constexpr int kAsmChildren = 64;  // children whose column ranges an assembly CTA stages in shared memory up front
constexpr int kAsmInFlight = 4;   // extend-add entries per lane in flight

// ranges[t.ch0 + q]: the columns of child q's update matrix that map into the task's front columns (computed with
// the schedule, so a CTA starts without searching the children's maps)
template <class T>
__global__ void __launch_bounds__(256) k_assemble(const AsmTask *__restrict__ tasks, const ChildRange *__restrict__ ranges,
                                                  DevPlan P, const value_of<T> *__restrict__ values, T *__restrict__ Lx,
                                                  T *__restrict__ U, const unsigned long long *status) {
  if (failed(status)) return;
  const AsmTask t = tasks[blockIdx.x];
  const int s = t.s, j0 = t.j0;
  const int f = P.snF[s], nc = P.snNc[s], m = P.snM[s];
  const int jend = min(j0 + kAsmCols, m);
  T *Lp = Lx + P.snLxp[s];
  T *Up = (m > nc) ? U + P.snUoff[s] : nullptr;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
  // 0. the child columns mapping into [j0, jend) (one range per child, the first kAsmChildren children staged in
  // shared memory while the columns are zeroed)
  __shared__ ChildRange chRange[kAsmChildren];
  const int q0 = P.chPtr[s], nch = P.chPtr[s + 1] - q0;
  const ChildRange *rg = ranges + t.ch0;
  if ((int)threadIdx.x < min(nch, kAsmChildren)) chRange[threadIdx.x] = rg[threadIdx.x];
  // 1. zero the lower part of the owned columns
  for (int j = j0 + warp; j < jend; j += nwarps)
    for (int i = j + lane; i < m; i += 32) *front_addr(Lp, Up, m, nc, i, j) = T(0);
  __syncthreads();
  // 2. A's entries of the owned pivot columns (each (row, col) once); 4 entries per lane in flight
  for (int j = j0 + warp; j < min(jend, nc); j += nwarps) {
    const int p0 = P.asmColPtr[f + j], p1 = P.asmColPtr[f + j + 1];
    for (int p = p0 + lane; p < p1; p += 128) {
      int dst[4];
      T v[4];
#pragma unroll
      for (int u = 0; u < 4; u++) {
        const int pp = p + 32 * u;
        dst[u] = pp < p1 ? P.asmDst[pp] : -1;
        v[u] = pp < p1 ? (T)ldg_v(values + P.asmSrc[pp]) : T(0);
      }
      T cur[4];
#pragma unroll
      for (int u = 0; u < 4; u++) cur[u] = dst[u] >= 0 ? Lp[dst[u]] : T(0);
#pragma unroll
      for (int u = 0; u < 4; u++)
        if (dst[u] >= 0) Lp[dst[u]] = cur[u] + v[u];
    }
  }
  __syncthreads();
  // 3. children, one after another (stack order of the reference)
  for (int q = 0; q < nch; q++) {
    const int c = P.chList[q0 + q];
    const int muc = P.snM[c] - P.snNc[c];
    if (muc <= 0) continue;  // block-uniform
    const int *map = P.eaMap + P.eaPtr[c];
    const T *Uc = U + P.snUoff[c];
    const ChildRange br = q < kAsmChildren ? chRange[q] : rg[q];
    for (int b = br.b0 + warp; b < br.b1; b += nwarps) {
      const int jj = map[b];
      const T *col = Uc + (int64_t)b * muc;
      // kAsmInFlight entries per lane in flight: gather the child's values and target rows, then read-modify-write
      for (int a = b + lane; a < muc; a += 32 * kAsmInFlight) {
        T v[kAsmInFlight], cur[kAsmInFlight];
        T *dst[kAsmInFlight];
#pragma unroll
        for (int u = 0; u < kAsmInFlight; u++) {
          const int aa = a + 32 * u;
          dst[u] = aa < muc ? front_addr(Lp, Up, m, nc, __ldg(map + aa), jj) : nullptr;
          v[u] = aa < muc ? col[aa] : T(0);
        }
#pragma unroll
        for (int u = 0; u < kAsmInFlight; u++) cur[u] = dst[u] ? *dst[u] : T(0);
#pragma unroll
        for (int u = 0; u < kAsmInFlight; u++)
          if (dst[u]) *dst[u] = cur[u] + v[u];
      }
    }
    __syncthreads();
  }
}

// Scale factors of the pivot block's right-looking update (not stored): FP64 as recip_nr, FP32 the hardware estimate.
__device__ __forceinline__ double fast_recip(double d) { return recip_nr(d); }
__device__ __forceinline__ float fast_recip(float d) { return __fdividef(1.0f, d); }
__device__ __forceinline__ cplx fast_recip(cplx d) { return cplx(1.0) / d; }

// ---------------------------------------------------------------------------------------------------------------
// Group panel: the pivot blocks of a group of up to kGroup 64-column blocks of a front, factored in one dataflow
// launch (POTRF of each pivot block, TRSM of the rows below it, and the update of the group's remaining columns).
// ---------------------------------------------------------------------------------------------------------------

// Pivot block: POTRF (or LDL^T) of the 64 x 64 diagonal block of a front, called by all 256 threads of a CTA, the
// block in registers. T = double: the FP64 factor; T = float: the mixed-precision factor. src: the updated block in
// shared memory, entry (i, j) at src[j lds + i]; Lp: the block's (0, 0) entry in the front (ld m), where the factor is
// written; w <= 64 its columns. Thread t < 136 owns the 4 x 4 tile (ti, tj), ti >= tj, of the lower triangle.
// Right-looking on the unscaled columns, four columns per step kb with two barriers: (1) the diagonal tile eliminates
// its four columns (settling the pivots) and publishes them; (2) the tiles below it in column block kb eliminate the
// same four columns against it and publish theirs; then every tile right of the block applies the rank-4 update
// S(i, j) -= sum S(i, k) S(j, k) / d_k. Cholesky tests d > 0 (sparse.mjs:1151-1156); LDL^T (ld.scal != null,
// ldlt.mjs:450-562) perturbs |d| < tau to +-tau and counts negative and perturbed pivots. At the end the columns are
// scaled: Cholesky L = a / sqrt(d) with sqrt(d) on the diagonal, LDL^T L = a / d with a unit diagonal (D to ld.D).
// Returns false (status set for the first failing column f + c0 + k) when a pivot failed; the block is then not
// written back.
// LB (the Bunch-Kaufman fast path): also returns 2, writing nothing, when a multiplier |L(i, k)| of the block exceeds
// lbound or a pivot was perturbed.
template <class T, class TC, bool LB = false>
__device__ int potrf_core(const T *src, int lds, T *Lp, int m, int w, int f, int c0, int s,
                          unsigned long long *status, const LdltArgs<T> &ld, double promoteBelow,
                          double lbound = -1.0) {
  __shared__ TC col[2][4][kPanel];  // per 4-column block (double-buffered): the block's unscaled columns, by row
  __shared__ TC pd[kPanel], piv[2][4];
  __shared__ unsigned char pflag[kPanel];
  __shared__ int fail, promote;
  const int tid = threadIdx.x;
  const bool ldlt = ld.scal != nullptr;
  using RT = typename real_of<TC>::type;
  const RT tau = ldlt ? (RT)ld.scal[1] : RT(0);
  // tile of this thread: row block ti, column block tj (ti >= tj), from tid by the triangular numbering
  int ti = 0;
  while ((ti + 1) * (ti + 2) / 2 <= tid) ti++;
  const int tj = tid - ti * (ti + 1) / 2;
  const bool owner = tid < 136;
  int myFail = -1;  // diagonal tiles only
  TC a[4][4];
#pragma unroll
  for (int r = 0; r < 4; r++)
#pragma unroll
    for (int c = 0; c < 4; c++) {
      const int i = 4 * ti + r, j = 4 * tj + c;
      a[r][c] = !owner || i < j ? TC(0) : (i < w ? (TC)src[j * lds + i] : (i == j ? TC(1) : TC(0)));
    }
  if (tid == 0) {
    fail = kPanel;  // none
    promote = 0;
  }
  for (int kb = 0; kb < kPanel / 4; kb++) {
    const int buf = kb & 1;
    if (owner && ti == kb && tj == kb) {
#pragma unroll
      for (int kk = 0; kk < 4; kk++) {
        const int k = 4 * kb + kk;
        TC d = a[kk][kk];
        unsigned char fl = 0;
        const bool bad = k < w && (ldlt ? !ldlt_pivot(d, tau, fl) : !chol_pivot_ok(d));
        if (bad && myFail < 0) myFail = k;  // first failing pivot of this diagonal tile
        const TC iv = fast_recip(d);          // the update scale only; L is scaled with the exact 1 / d at the end
        pd[k] = d;
        pflag[k] = fl;
        piv[buf][kk] = iv;
#pragma unroll
        for (int r = kk + 1; r < 4; r++)
#pragma unroll
          for (int c = kk + 1; c <= r; c++) a[r][c] -= a[r][kk] * (a[c][kk] * iv);
      }
#pragma unroll
      for (int kk = 0; kk < 4; kk++)
#pragma unroll
        for (int r = 0; r < 4; r++) col[buf][kk][4 * kb + r] = a[r][kk];
    }
    __syncthreads();
    if (owner && tj == kb && ti > kb) {
#pragma unroll
      for (int kk = 0; kk < 4; kk++) {
        const TC iv = piv[buf][kk];
#pragma unroll
        for (int c = kk + 1; c < 4; c++) {
          const TC cj = col[buf][kk][4 * kb + c] * iv;
#pragma unroll
          for (int r = 0; r < 4; r++) a[r][c] -= a[r][kk] * cj;
        }
      }
#pragma unroll
      for (int kk = 0; kk < 4; kk++)
#pragma unroll
        for (int r = 0; r < 4; r++) col[buf][kk][4 * ti + r] = a[r][kk];
    }
    __syncthreads();
    if (owner && tj > kb) {
#pragma unroll
      for (int kk = 0; kk < 4; kk++) {
        const TC iv = piv[buf][kk];
        TC ci[4], cj[4];
#pragma unroll
        for (int r = 0; r < 4; r++) ci[r] = col[buf][kk][4 * ti + r];
#pragma unroll
        for (int c = 0; c < 4; c++) cj[c] = col[buf][kk][4 * tj + c] * iv;
#pragma unroll
        for (int r = 0; r < 4; r++)
#pragma unroll
          for (int c = 0; c < 4; c++)
            if (ti > tj || c <= r) a[r][c] -= ci[r] * cj[c];
      }
    }
  }
  if (myFail >= 0) atomicMin(&fail, myFail);
  if (promoteBelow > 0.0 && tid < w && !(pivot_mag(pd[tid]) >= promoteBelow)) promote = 1;
  if constexpr (LB && !is_cplx<TC>::value) {
    {  // every multiplier within the bound and no pivot perturbed, else redo with pivoting
      if (tid < w && (pflag[tid] & 2)) promote = 1;
      if (owner) {
#pragma unroll
        for (int r = 0; r < 4; r++)
#pragma unroll
          for (int c = 0; c < 4; c++) {
            const int i = 4 * ti + r, j = 4 * tj + c;
            if (i > j && i < w && !(fabs((double)a[r][c]) <= lbound * fabs((double)pd[j]))) promote = 1;
          }
      }
    }
  }
  __syncthreads();
  if (promote) return 2;  // the caller redoes the block in higher precision (nothing written)
  if (fail < kPanel) {
    if (tid == 0) atomicMin(status, status_word(f + c0 + fail, ldlt ? 2 : 1, s));
    return 1;
  }
  if (owner) {
#pragma unroll
    for (int c = 0; c < 4; c++) {
      const int j = 4 * tj + c;
      const TC d = pd[j];
      const TC lj = ldlt ? d : chol_sqrt(d);
      const TC inv = TC(1) / lj;
#pragma unroll
      for (int r = 0; r < 4; r++) {
        const int i = 4 * ti + r;
        if (i >= j && i < w && j < w) Lp[(int64_t)j * m + i] = (T)(i == j ? (ldlt ? TC(1) : lj) : a[r][c] * inv);
      }
    }
  }
  if (ldlt) {
    if (tid < w) ld.D[f + c0 + tid] = (typename LdltArgs<T>::DT)pd[tid];
    if (tid == 0) {
      int neg = 0, pert = 0;
      for (int k = 0; k < w; k++) neg += pflag[k] & 1, pert += pflag[k] >> 1;
      atomicAdd(ld.counts, neg);
      atomicAdd(ld.counts + 1, pert);
    }
  }
  return 0;
}

// POTRF / LDL^T of a pivot block (potrf_core in the factor's precision). An FP32 LDL^T block with a pivot of
// magnitude below FLT_EPSILON x max_i |A(i, i)| (a pivot with no correct FP32 digit left) is factored again from the
// same entries (src is left unchanged) in FP64 arithmetic (stored FP32): the small-pivot blocks of the mixed-precision
// indefinite factor get FP64 pivots. Returns false when a pivot failed (status set).
template <class T>
__device__ bool potrf_block(const T *src, int lds, T *Lp, int m, int w, int f, int c0, int s,
                            unsigned long long *status, const LdltArgs<T> &ld) {
  if constexpr (std::is_same<T, float>::value) {
    if (ld.scal != nullptr) {
      const double amax = ld.scal[0] > 0.0 ? ld.scal[1] / ld.scal[0] : 0.0;
      const int r = potrf_core<float, float>(src, lds, Lp, m, w, f, c0, s, status, ld, amax * (double)FLT_EPSILON);
      if (r != 2) return r == 0;
      return potrf_core<float, double>(src, lds, Lp, m, w, f, c0, s, status, ld, -1.0) == 0;
    }
  }
  return potrf_core<T, T>(src, lds, Lp, m, w, f, c0, s, status, ld, -1.0) == 0;
}

// (value, index) of the largest value over the warp, the smallest index on ties (every lane gets the result)
__device__ __forceinline__ void warp_argmax(double &v, int &i) {
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

// Bunch-Kaufman LDL^T of a pivot block, the pivot search restricted to the block's w columns (so the supernode
// partition and every row structure stay the reference's): at column k, with colmax = max_{i>k} |B(i, k)| (row r),
// a 1 x 1 pivot k when |B(k, k)| >= alpha colmax or |B(k, k)| rowmax >= alpha colmax^2 (rowmax = max_{j != r}
// |B(r, j)|), a 1 x 1 pivot r when |B(r, r)| >= alpha rowmax, else the 2 x 2 pivot (k, r); alpha = (1 + sqrt 17) / 8
// (Bunch and Kaufman, Math. Comp. 31, 1977). Each interchange is applied to the block's whole rows, the L columns
// already computed included, so that P B P^T = L D L^T with L unit lower triangular (L(k + 1, k) = 0 inside a 2 x 2
// pivot, whose off-diagonal is D(k + 1, k)). A column with no entry at or above tau keeps the reference's static
// perturbation (|d| < tau -> -+tau, a non-finite one fails; ldlt.mjs:513-522). FP64 arithmetic for every T.
// S: 64 x 65 doubles of shared workspace (a full symmetric copy, S[j][i] = B(i, j)); src: the updated block (entry
// (i, j), i >= j, at src[j lds + i]). Writes L to Lp (ld m), D, Doff and piv, adds the inertia (a 2 x 2 pivot with a
// negative determinant has one negative eigenvalue, with a positive one two when its diagonal is negative) and the
// perturbed count. Returns false (status set) on a non-finite pivot; nothing is written then. Called by every thread.
template <class T>
__device__ bool bk_block(const T *src, int lds, double (*S)[kPanel + 1], T *Lp, int m, int w, int f, int c0, int s,
                         unsigned long long *status, const LdltArgs<T> &ld) {
  __shared__ int sPerm[kPanel];
  __shared__ double sD[kPanel], sE[kPanel], sC0[kPanel], sC1[kPanel];
  __shared__ int sStep, sKp, sFail, sNeg, sPert;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nthr = blockDim.x;
  const double tau = ld.scal[1];
  const double alpha = 0.64038820320220756;  // (1 + sqrt(17)) / 8
  for (int e = tid; e < kPanel * kPanel; e += nthr) {
    const int i = e & (kPanel - 1), j = e >> 6;
    double v = i == j ? 1.0 : 0.0;
    if (i < w && j < w) v = (double)(i >= j ? src[j * lds + i] : src[i * lds + j]);
    S[j][i] = v;
  }
  if (tid < kPanel) {
    sPerm[tid] = tid;
    sD[tid] = 1.0;
    sE[tid] = 0.0;
  }
  if (tid == 0) {
    sFail = -1;
    sNeg = 0;
    sPert = 0;
  }
  __syncthreads();
  for (int k = 0; k < w;) {
    if (warp == 0) {  // the pivot choice
      double cm = -1.0;
      int im = -1;
      for (int i = k + 1 + lane; i < w; i += 32) {
        const double a = fabs(S[k][i]);
        if (a > cm) {
          cm = a;
          im = i;
        }
      }
      warp_argmax(cm, im);
      const double colmax = cm > 0.0 ? cm : 0.0, absakk = fabs(S[k][k]);
      int step = 1, kp = k;
      if (colmax > 0.0 && !(absakk >= alpha * colmax)) {  // (a NaN diagonal takes the 1 x 1 path and fails below)
        double rm = 0.0;
        for (int j = k + lane; j < w; j += 32)
          if (j != im) rm = fmax(rm, fabs(S[j][im]));
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) rm = fmax(rm, __shfl_xor_sync(0xffffffffu, rm, o));
        if (absakk * rm >= alpha * colmax * colmax) {
          kp = k;
        } else if (fabs(S[im][im]) >= alpha * rm) {
          kp = im;
        } else {
          step = 2;
          kp = im;
        }
      }
      if (lane == 0) {
        sStep = step;
        sKp = kp;
      }
    }
    __syncthreads();
    const int step = sStep, kp = sKp, kk = k + step - 1, k1 = k + step;
    if (kp != kk) {  // interchange kk and kp: whole rows (L columns included), then the trailing columns
      if (tid < w) {
        const double t = S[tid][kk];
        S[tid][kk] = S[tid][kp];
        S[tid][kp] = t;
      }
      __syncthreads();
      if (tid >= k && tid < w) {
        const double t = S[kk][tid];
        S[kk][tid] = S[kp][tid];
        S[kp][tid] = t;
      }
      if (tid == 0) {
        const int t = sPerm[kk];
        sPerm[kk] = sPerm[kp];
        sPerm[kp] = t;
      }
      __syncthreads();
    }
    const int nt = w - k1;
    if (step == 1) {
      double d = S[k][k];
      const bool small = !(fabs(d) >= tau);
      if (small && isfinite(d)) d = d < 0.0 ? -tau : tau;
      if (tid < w) sC0[tid] = S[k][tid];  // column k, unscaled
      if (tid == 0) {
        sD[k] = d;
        if (!isfinite(d) && sFail < 0) sFail = k;
        sNeg += d < 0.0 ? 1 : 0;
        sPert += small ? 1 : 0;
      }
      __syncthreads();
      if (sFail >= 0) break;  // block-uniform
      const double inv = 1.0 / d;
      for (int e = tid; e < nt * nt; e += nthr) {
        const int i = k1 + e % nt, j = k1 + e / nt;
        S[j][i] -= sC0[i] * (sC0[j] * inv);
      }
      if (tid >= k1 && tid < w) S[k][tid] = sC0[tid] * inv;  // L(i, k)
    } else {
      // D_k = e [[a, 1], [1, c]], D_k^-1 = (t / e) [[c, -1], [-1, a]] with a = d11 / e, c = d22 / e, t = 1 / (a c - 1)
      const double d11 = S[k][k], e21 = S[k][k + 1], d22 = S[k + 1][k + 1];
      const double a = d11 / e21, c = d22 / e21, te = (1.0 / (a * c - 1.0)) / e21;
      if (tid < w) {
        sC0[tid] = S[k][tid];
        sC1[tid] = S[k + 1][tid];
      }
      if (tid == 0) {
        sD[k] = d11;
        sD[k + 1] = d22;
        sE[k] = e21;
        if (!(isfinite(te) && isfinite(a) && isfinite(c)) && sFail < 0) sFail = k;
        sNeg += a * c - 1.0 < 0.0 ? 1 : (d11 < 0.0 ? 2 : 0);
      }
      __syncthreads();
      if (sFail >= 0) break;  // block-uniform
      for (int e = tid; e < nt * nt; e += nthr) {
        const int i = k1 + e % nt, j = k1 + e / nt;
        const double l1 = te * (c * sC0[i] - sC1[i]), l2 = te * (a * sC1[i] - sC0[i]);
        S[j][i] -= l1 * sC0[j] + l2 * sC1[j];
      }
      if (tid >= k1 && tid < w) {
        S[k][tid] = te * (c * sC0[tid] - sC1[tid]);  // L(i, k)
        S[k + 1][tid] = te * (a * sC1[tid] - sC0[tid]);  // L(i, k + 1)
      }
      if (tid == 0) S[k][k + 1] = 0.0;  // L(k + 1, k)
    }
    __syncthreads();
    k += step;
  }
  __syncthreads();
  if (sFail >= 0) {
    if (tid == 0) atomicMin(status, status_word(f + c0 + sFail, 2, s));
    return false;
  }
  for (int e = tid; e < w * w; e += nthr) {
    const int i = e % w, j = e / w;
    if (i >= j) Lp[(int64_t)j * m + i] = (T)(i == j ? 1.0 : S[j][i]);
  }
  if (tid < w) {
    ld.D[f + c0 + tid] = sD[tid];
    ld.Doff[f + c0 + tid] = sE[tid];
    ld.piv[f + c0 + tid] = sPerm[tid];
  }
  if (tid == 0) {
    atomicAdd(ld.counts, sNeg);
    atomicAdd(ld.counts + 1, sPert);
  }
  return true;
}

// TRSM of up to 64 rows [r0, r1) of a front (L: its column-major block, ld m) against its factored pivot block
// [c0, c0 + w): x_k = (a_k - sum_{c<k} x_c M(k, c)) / M(k, k). Four threads per row, thread (row, q) holds columns
// 16 q .. 16 q + 15 in registers. Phase p: the threads of quarter p solve their 16 columns (the earlier quarters'
// contributions already applied) and publish them; after a barrier the threads of the later quarters subtract
// quarter p's contribution (16 x 16 products) from theirs. Cholesky: M = L11, x = L21. LDL^T: M(k, c) = L11(k, c) d_c,
// M(k, k) = d_k, x = L21, and w = x D = L21 D (the update's A operand, written to ld.W for the FP64 factor). The rows
// are also written as BF16 hi / lo pairs (hi = bf16(x), lo = bf16(x - hi)) into the split columns of the tensor-core
// update (mixed precision). The pivot block and D come from another CTA of the launch: read through L2 (__ldcg).
// x: this thread's 16 entries of its row (row r0 + tid % 64, columns c0 + 16 (tid / 64) + u), loaded by the caller
// before it waited for the pivot block (the strip's own rows are final by then).
// On return Ws[c][r] holds this strip's update operand (x, or x D for LDL^T) and M[c][r] the solved rows x
// (c < w, r < r1 - r0; zero elsewhere): a diagonal strip's X_c for its own column block.
template <class T, bool BK>
__device__ void trsm_strip(T *L, int m, int f, int c0, int w, int r0, int r1, int64_t lxp, int64_t sp,
                           __nv_bfloat16 *Shi, __nv_bfloat16 *Slo, const LdltArgs<T> &ld, T (*M)[kPanel + 1],
                           T (*Ws)[kPanel + 1], T *invd, T *dv, T (&x)[16]) {
  const bool ldlt = ld.scal != nullptr;
  // Bunch-Kaufman pivots (real factors): the strip's columns are taken in the block's pivot order, solved against the
  // unit L11 (W = x L11^-T, the update's operand), then L21 = W D^-1 with the block's 1 x 1 and 2 x 2 pivots:
  // column c of L21 is dA[c] W_c + dB[c] W_dP[c] (dP[c] = the other column of its 2 x 2 pivot, dB = 0 for a 1 x 1)
  constexpr bool bk = BK && !is_cplx<T>::value;
  __shared__ double dA[kPanel], dB[kPanel];
  __shared__ int dP[kPanel], sPiv[kPanel];
  const int tid = threadIdx.x, r = tid & (kPanel - 1), q = tid >> 6;
  {  // the pivot block: thread (r, q) loads row r of columns 16 q .. 16 q + 15 (times their pivots for LDL^T), and
     // thread r < 64 the pivot of column r, in one round trip
    T v[16];
#pragma unroll
    for (int u = 0; u < 16; u++) {
      const int c = 16 * q + u;
      v[u] = (r < w && c < r) ? ldcg_v(L + (int64_t)(c0 + c) * m + c0 + r) : T(0);
    }
    if (ldlt && !bk) {
#pragma unroll
      for (int u = 0; u < 16; u++) {
        const int c = 16 * q + u;
        v[u] = v[u] * (c < w ? (T)ldcg_v(ld.D + f + c0 + c) : T(1));
      }
    }
    if (tid < kPanel) {
      if constexpr (bk) {
        {
          const int c = tid;
          double a = 1.0, b = 0.0;
          int pc = c;
          if (c < w) {
            const double d = ldcg_v(ld.D + f + c0 + c);
            const double en = ldcg_v(ld.Doff + f + c0 + c), ep = c > 0 ? ldcg_v(ld.Doff + f + c0 + c - 1) : 0.0;
            if (en != 0.0 || ep != 0.0) {  // 2 x 2 pivot (c, c + 1) or (c - 1, c): the inverse as in bk_block
              const bool first = en != 0.0;
              const double e = first ? en : ep;
              const double d11 = first ? d : ldcg_v(ld.D + f + c0 + c - 1);
              const double d22 = first ? ldcg_v(ld.D + f + c0 + c + 1) : d;
              const double aa = d11 / e, cc = d22 / e, te = (1.0 / (aa * cc - 1.0)) / e;
              a = te * (first ? cc : aa);
              b = -te;
              pc = first ? c + 1 : c - 1;
            } else {
              a = 1.0 / d;
            }
          }
          dA[c] = a;
          dB[c] = b;
          dP[c] = pc;
          sPiv[c] = c < w ? __ldcg(ld.piv + f + c0 + c) : c;
        }
      }
      const T d = bk ? T(1)
                     : tid < w ? (ldlt ? (T)ldcg_v(ld.D + f + c0 + tid) : ldcg_v(L + (int64_t)(c0 + tid) * m + c0 + tid))
                               : T(1);
      dv[tid] = d;
      invd[tid] = T(1) / d;
    }
#pragma unroll
    for (int u = 0; u < 16; u++) M[r][16 * q + u] = v[u];
  }
  const int row = r0 + r;
  const bool active = row < r1;
  __syncthreads();
  if constexpr (bk) {  // the strip's columns in the block's pivot order: x_new(c) = x(piv(c))
#pragma unroll
    for (int u = 0; u < 16; u++) Ws[16 * q + u][r] = x[u];
    __syncthreads();
#pragma unroll
    for (int u = 0; u < 16; u++) x[u] = Ws[sPiv[16 * q + u]][r];
    __syncthreads();
  }
  for (int p = 0; p < 4; p++) {
    if (q == p) {  // solve this quarter
#pragma unroll
      for (int u = 0; u < 16; u++) {
        const int c = 16 * p + u;
        x[u] *= invd[c];
#pragma unroll
        for (int u2 = u + 1; u2 < 16; u2++) x[u2] -= x[u] * M[16 * p + u2][c];
      }
#pragma unroll
      for (int u = 0; u < 16; u++) Ws[16 * p + u][r] = x[u];
    }
    __syncthreads();
    if (q > p) {  // subtract quarter p's contribution
#pragma unroll 4
      for (int kk = 0; kk < 16; kk++) {
        const int k = 16 * p + kk;
        const T xk = Ws[k][r];
#pragma unroll
        for (int u = 0; u < 16; u++) x[u] -= xk * M[16 * q + u][k];
      }
    }
  }
  __syncthreads();  // every quarter read Ws: overwrite it with the update operand
  const int ld8 = (m + 7) & ~7;
#pragma unroll
  for (int u = 0; u < 16; u++) {
    const int cc = 16 * q + u;
    T xv = x[u];
    T wv = ldlt ? xv * dv[cc] : xv;
    if constexpr (bk) {
      {  // x[u] is W (already in Ws, zero outside the strip and the block); L21 = W D^-1
        wv = x[u];
        xv = (T)(dA[cc] * (double)x[u] + dB[cc] * (double)Ws[dP[cc]][r]);
      }
    }
    if (!bk) Ws[cc][r] = active && cc < w ? wv : T(0);
    M[cc][r] = active && cc < w ? xv : T(0);  // the pivot block in M is no longer read
    if (!active || cc >= w) continue;
    L[(int64_t)(c0 + cc) * m + row] = xv;
    if (ldlt && ld.W) ld.W[lxp + (int64_t)(c0 + cc) * m + row] = wv;
    if constexpr (!is_cplx<T>::value)
    if (Shi) {
      const int64_t g = sp + (int64_t)(c0 + cc) * ld8 + row;
      const __nv_bfloat16 hi = __float2bfloat16_rn((float)xv);
      Shi[g] = hi;
      Slo[g] = __float2bfloat16_rn((float)xv - __bfloat162float(hi));
      if (ldlt) {
        const __nv_bfloat16 whi = __float2bfloat16_rn((float)wv);
        ld.Whi[g] = whi;
        ld.Wlo[g] = __float2bfloat16_rn((float)wv - __bfloat162float(whi));
      }
    }
  }
  __syncthreads();
}

// Wait (thread 0, bounded) until *p >= need; false when the factorization has failed (a pivot, or a wait that ran
// out: status set). Thread 0 decides and the CTA follows it after the barrier, so every thread returns the same.
__device__ __forceinline__ bool panel_wait(const int *p, int need, unsigned long long *status, long long limit) {
  __shared__ int ok;
  if (threadIdx.x == 0) {
    long long spins = 0;
    int v = 1;
    while (ld_acquire(p) < need) {
      if (failed(status)) {
        v = 0;
        break;
      }
      if (++spins > limit) {
        atomicMin(status, status_word(0x7fffffff, 3, 0));
        v = 0;
        break;
      }
      __nanosleep(64);
    }
    if (failed(status)) v = 0;  // a failed pivot also releases its flag
    ok = v;
  }
  __syncthreads();
  return ok != 0;
}

// Publish *p = v after this CTA's global writes: all threads pass the barrier first, and thread 0's release store
// orders every write made before the barrier (by any thread of the CTA) before the flag, for a reader that acquires it.
__device__ __forceinline__ void panel_release(int *p, int v) {
  __syncthreads();
  if (threadIdx.x == 0) st_release(p, v);
}

// One group of pivot blocks [g0, g1) of a front, a strip of up to 64 rows per CTA, CTAs ordered by an atomic ticket
// (the diagonal strips of every item first, then the strips below the group). Per pivot block b of the group:
//   the diagonal strip of block b (rows [c0, c0 + w)) factors it once its own updates are done and publishes P[b];
//   every strip with rows below block b waits for P[b], solves its rows against the block (TRSM) and, when it is a
//   diagonal strip, publishes D[j] = b + 1; then it updates its rows of the group's remaining columns [c0 + w, g1)
//   with block b (C -= W_r X_c^T, K = w; X_c: the rows of those columns, from the diagonal strips' TRSM, waited for
//   by D[j] >= b + 1; a diagonal strip updates only the lower part, columns up to its own rows).
// Every wait is on a strip with a smaller ticket, which runs to completion without waiting on a larger one, so the
// launch cannot deadlock whatever the number of resident CTAs. The columns right of the group receive the group's
// update afterwards (k_update / k_update_mx, K = the group). Failure (a pivot, a bounded wait) sets the status and
// releases P[b], so every waiter leaves.
constexpr int kGroupSmem = 3 * kPanel * (kPanel + 1) * (int)sizeof(double);
// two CTAs per SM for the real factors (registers capped at 128); the complex one is held to one by its shared memory
template <class T>
constexpr int group_min_blocks() { return is_cplx<T>::value ? 1 : 2; }
template <class T, bool BK>
__global__ void __launch_bounds__(256, group_min_blocks<T>()) k_group_panel(const GroupItem *__restrict__ items,
                                                     const StripTask *__restrict__ strips, int nstrips, int *ticket,
                                                     int *flags, DevPlan P, T *__restrict__ Lx,
                                                     unsigned long long *status, __nv_bfloat16 *__restrict__ Shi,
                                                     __nv_bfloat16 *__restrict__ Slo, LdltArgs<T> ld) {
  extern __shared__ __align__(16) unsigned char gp_raw[];
  T(*M)[kPanel + 1] = reinterpret_cast<T(*)[kPanel + 1]>(gp_raw);  // pivot block (TRSM), then the X_c chunk
  T(*Ws)[kPanel + 1] = reinterpret_cast<T(*)[kPanel + 1]>(gp_raw + kPanel * (kPanel + 1) * sizeof(T));
  T(*Ds)[kPanel + 1] = reinterpret_cast<T(*)[kPanel + 1]>(gp_raw + 2 * kPanel * (kPanel + 1) * sizeof(T));
  __shared__ T invd[kPanel], dv[kPanel];
  __shared__ int sTicket;
  if (threadIdx.x == 0) sTicket = failed(status) ? nstrips : atomicAdd(ticket, 1);
  __syncthreads();
  const int t = sTicket;
  if (t >= nstrips) return;
  const StripTask st = strips[t];
  const GroupItem it = items[st.item];
  const int s = it.s, g0 = it.g0, g1 = it.g1;
  const int f = P.snF[s], m = P.snM[s];
  const int nb = (g1 - g0 + kPanel - 1) / kPanel;
  const int r0 = st.r0, r1 = st.r1, jd = st.diag;
  const int bmax = jd >= 0 ? jd : nb;  // pivot blocks whose rows below include this strip
  T *L = Lx + P.snLxp[s];
  int *Pf = flags + it.flag0, *Df = Pf + nb;
  const int tid = threadIdx.x, tr = tid & 15, tc = tid >> 4;
  // A diagonal strip keeps its own pivot block (columns [r0, r1), lower part) in shared memory while it updates it
  // (Ds[j][i] = block (i, j)), and its POTRF reads it from there: no round trip through the front.
  if (jd >= 0) {
    for (int e = tid; e < kPanel * kPanel; e += blockDim.x) {
      const int i = e & 63, j = e >> 6;
      Ds[j][i] = (r0 + i < r1 && j <= i) ? L[(int64_t)(r0 + j) * m + r0 + i] : T(0);
    }
  }
  for (int b = 0; b < bmax; b++) {
    const int c0 = g0 + b * kPanel, w = min(kPanel, g1 - c0), c1 = c0 + w;
    T x[16];  // this thread's part of the strip's rows of block b, loaded while the pivot block is not yet ready
    {
      const int xr = r0 + (tid & (kPanel - 1)), xq = tid >> 6;
#pragma unroll
      for (int u = 0; u < 16; u++) {
        const int c = 16 * xq + u;
        x[u] = xr < r1 && c < w ? L[(int64_t)(c0 + c) * m + xr] : T(0);
      }
    }
    if (!panel_wait(Pf + b, 1, status, P.spin)) return;
    trsm_strip<T, BK>(L, m, f, c0, w, r0, r1, P.snLxp[s], P.snSp[s], Shi, Slo, ld, M, Ws, invd, dv, x);
    if (jd >= 0) panel_release(Df + jd, b + 1);
    // Update with block b (C -= W_r X_c^T, K = w): a diagonal strip first its own pivot block (X_c = its solved rows,
    // left in M by the TRSM; into Ds), then the blocks between block b and its own; a strip below every remaining
    // column block of the group.
    const int hi = jd >= 0 ? r0 : g1, nown = jd >= 0 ? 1 : 0;
    const int nchunk = nown + (hi > c1 ? (hi - c1 + kPanel - 1) / kPanel : 0);
    for (int ch = 0; ch < nchunk; ch++) {
      const bool own = ch < nown;
      const int cb = own ? r0 : c1 + (ch - nown) * kPanel, ncol = own ? r1 - r0 : min(kPanel, hi - cb);
      if (!own) {
        if (!panel_wait(Df + (cb - g0) / kPanel, b + 1, status, P.spin)) return;
        for (int e = tid; e < kPanel * kPanel; e += blockDim.x) {  // X_c[k][jj] = L(cb + jj, c0 + k)
          const int k = e >> 6, jj = e & 63;
          M[k][jj] = (k < w && jj < ncol) ? ldcg_v(L + (int64_t)(c0 + k) * m + cb + jj) : T(0);
        }
        __syncthreads();
      }
      T acc[4][4];
#pragma unroll
      for (int a = 0; a < 4; a++)
#pragma unroll
        for (int bb = 0; bb < 4; bb++) acc[a][bb] = T(0);
      for (int k = 0; k < w; k++) {
        T wv[4], xv[4];
#pragma unroll
        for (int a = 0; a < 4; a++) wv[a] = Ws[k][tr + 16 * a];
#pragma unroll
        for (int bb = 0; bb < 4; bb++) xv[bb] = M[k][tc + 16 * bb];
#pragma unroll
        for (int a = 0; a < 4; a++)
#pragma unroll
          for (int bb = 0; bb < 4; bb++) acc[a][bb] += wv[a] * xv[bb];
      }
#pragma unroll
      for (int a = 0; a < 4; a++)
#pragma unroll
        for (int bb = 0; bb < 4; bb++) {
          const int i = tr + 16 * a, jj = tc + 16 * bb;
          if (own) {
            if (jj <= i) Ds[jj][i] -= acc[a][bb];
          } else if (r0 + i < r1 && jj < ncol) {
            T *cptr = L + (int64_t)(cb + jj) * m + r0 + i;
            *cptr = *cptr - acc[a][bb];
          }
        }
      __syncthreads();  // M is reloaded by the next chunk, or by the next TRSM
    }
  }
  if (jd >= 0) {  // this strip's own pivot block, fully updated: factor it and publish it (also after a failure)
    const int c0 = g0 + jd * kPanel, w = min(kPanel, g1 - c0);
    __syncthreads();  // Ds complete (also when the strip had no earlier pivot block)
    if constexpr (BK && !is_cplx<T>::value) {
      // Bunch-Kaufman keeps every pivot of the block in place exactly when each multiplier is at most 1 / alpha in
      // magnitude and no pivot needs the perturbation: try the unpivoted LDL^T first (it writes nothing unless it
      // passes that test), else redo the block with pivots from the untouched entries
      const int r = potrf_core<T, T, true>(&Ds[0][0], kPanel + 1, L + (int64_t)c0 * m + c0, m, w, f, c0, s, status, ld,
                                           -1.0, 1.0 / 0.64038820320220756);
      if (r == 2) {  // FP64 workspace in M (and Ws for FP32 fronts), both free here
        bk_block<T>(&Ds[0][0], kPanel + 1, reinterpret_cast<double(*)[kPanel + 1]>(gp_raw),
                    L + (int64_t)c0 * m + c0, m, w, f, c0, s, status, ld);
      } else if (r == 0 && threadIdx.x < w) {  // the identity pivot order, 1 x 1 pivots
        ld.piv[f + c0 + threadIdx.x] = threadIdx.x;
        ld.Doff[f + c0 + threadIdx.x] = 0.0;
      }
    } else
      potrf_block<T>(&Ds[0][0], kPanel + 1, L + (int64_t)c0 * m + c0, m, w, f, c0, s, status, ld);
    panel_release(Pf + jd, 1);
  }
}

// ---------------------------------------------------------------------------------------------------------------
// Trailing update: F[i0:i0+128, j0:j0+64] -= A B^T with A = panel rows i, B = panel rows j, K = pivot block width.
// Persistent CTAs (two per SM, so one loads while the other computes) walk the step's tiles. The panel rows arrive in
// shared memory by cp.async; the product runs on the FP64 tensor cores with mma.sync m16n8k16 (fragment layouts of
// the SM90 FP64 MMA atoms: A (m = g + 8 (v & 1), k = t + 4 (v >> 1)), B (n = g, k = t + 4 v), C (m = g + 8 (v >> 1),
// n = 2 t + (v & 1)), g = lane / 4, t = lane % 4). 8 warps as 4 (rows) x 2 (cols), 32 x 32 per warp.
// ---------------------------------------------------------------------------------------------------------------
__device__ __forceinline__ void dmma_16x8x16(double (&c)[4], const double (&a)[8], const double (&b)[4]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7,%8,%9,%10,%11}, "
      "{%12,%13,%14,%15}, {%0,%1,%2,%3};\n"
      : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
      : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(a[4]), "d"(a[5]), "d"(a[6]), "d"(a[7]), "d"(b[0]), "d"(b[1]),
        "d"(b[2]), "d"(b[3]));
}

__device__ __forceinline__ void cp_async8(void *smem, const void *gmem, bool valid) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  const int bytes = valid ? 8 : 0;  // zero-fill when out of range
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(sa), "l"(gmem), "r"(bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

constexpr int kLdA = kTileM + 4;  // 132 doubles (== 4 mod 16): conflict-free fragment loads
constexpr int kLdB = kTile + 4;   // 68 doubles
constexpr int kStage = kPanel * kLdA + kPanel * kLdB;  // doubles per pipeline stage
constexpr int kUpdateSmem = 2 * kStage * (int)sizeof(double);

// Panel rows of one tile and one 64-column chunk of its K range into a pipeline stage. Thread t owns one row of A
// (t % 128) and of B (t % 64) and walks the pivot columns with a pointer step of 2 m (A) or 4 m (B).
__device__ __forceinline__ void tile_loads(const TileTask &t, int chunk, const double *Ax, const double *Lx,
                                           double *stage) {
  const int kc = t.c0 + chunk * kPanel, kw = min(kPanel, t.w - chunk * kPanel), wk = (kw + 15) & ~15;
  const double *Ap = Ax + t.lp, *Lp = Lx + t.lp;
  const int tid = threadIdx.x;
  {
    const int i = tid & (kTileM - 1), k0 = tid >> 7, r = t.i0 + i;
    const bool rowok = r < t.m;
    const double *src = Ap + (int64_t)(kc + k0) * t.m + (rowok ? r : 0);
    double *dst = stage + k0 * kLdA + i;
    const int64_t step = 2 * (int64_t)t.m;
#pragma unroll 4
    for (int k = k0; k < wk; k += 2, src += step, dst += 2 * kLdA)
      cp_async8(dst, rowok && k < kw ? src : Ap, rowok && k < kw);
  }
  {
    const int i = tid & (kTile - 1), k0 = tid >> 6, r = t.j0 + i;
    const bool rowok = r < t.m;
    const double *src = Lp + (int64_t)(kc + k0) * t.m + (rowok ? r : 0);
    double *dst = stage + kPanel * kLdA + k0 * kLdB + i;
    const int64_t step = 4 * (int64_t)t.m;
#pragma unroll 4
    for (int k = k0; k < wk; k += 4, src += step, dst += 4 * kLdB)
      cp_async8(dst, rowok && k < kw ? src : Lp, rowok && k < kw);
  }
}

// Update tiles F[i0:i0+128, j0:j0+64] -= A B^T, K = w pivot columns in 64-column chunks. Persistent CTAs walk
// (tile, chunk) items; the next item's panel rows stream into the other stage while the current one runs on the
// FP64 tensor cores; the C tile is read once (prefetched into registers during its first chunk) and written once.
__global__ void __launch_bounds__(256, 1) k_update(const TileTask *__restrict__ tasks, int ntasks,
                                                   double *__restrict__ Lx, double *__restrict__ U,
                                                   const double *__restrict__ W, const unsigned long long *status) {
  if (failed(status)) return;
  const double *Ax = W ? W : Lx;  // LDL^T: A = L21 D
  extern __shared__ double smem_upd[];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int wr = (warp >> 1) * 32, wc = (warp & 1) * 32;
  const int g = lane >> 2, t4 = lane & 3;
  int t = blockIdx.x;
  if (t >= ntasks) return;
  TileTask cur = tasks[t];
  TileTask nxtTask = cur;
  if (t + (int)gridDim.x < ntasks) nxtTask = tasks[t + gridDim.x];
  int chunk = 0, nch = (cur.w + kPanel - 1) / kPanel;
  int stage = 0;
  tile_loads(cur, 0, Ax, Lx, smem_upd);
  cp_async_commit();
  double *cp[4][2];
  int jj[4][2], ii[2][2];
  double cpre[2][4][4], acc[2][4][4];
  bool newTile = true;
  while (true) {
    // the next (tile, chunk) item
    const bool sameTile = chunk + 1 < nch;
    const bool hasNext = sameTile || t + (int)gridDim.x < ntasks;
    if (hasNext)
      tile_loads(sameTile ? cur : nxtTask, sameTile ? chunk + 1 : 0, Ax, Lx, smem_upd + (stage ^ 1) * kStage);
    cp_async_commit();
    const int m = cur.m, nc = cur.nc, mu = m - nc;
    if (newTile) {
      // this thread's 8 columns (base pointers indexed by the front row) and 4 rows of the C tile; C prefetch
      double *Lp = Lx + cur.lp;
      double *Up = cur.up >= 0 ? U + cur.up : Lp;
#pragma unroll
      for (int b = 0; b < 4; b++)
#pragma unroll
        for (int u = 0; u < 2; u++) {
          const int j = cur.j0 + wc + 8 * b + 2 * t4 + u;
          jj[b][u] = j < cur.jend ? j : 0x3fffffff;  // columns beyond jend are masked
          cp[b][u] = j < nc ? Lp + (int64_t)j * m : Up + (int64_t)(j - nc) * mu - nc;
        }
#pragma unroll
      for (int a = 0; a < 2; a++)
#pragma unroll
        for (int h = 0; h < 2; h++) ii[a][h] = cur.i0 + wr + 16 * a + g + 8 * h;
#pragma unroll
      for (int a = 0; a < 2; a++)
#pragma unroll
        for (int b = 0; b < 4; b++)
#pragma unroll
          for (int v = 0; v < 4; v++) {
            const int i = ii[a][v >> 1], j = jj[b][v & 1];
            cpre[a][b][v] = (i < m && i >= j) ? cp[b][v & 1][i] : 0.0;
            acc[a][b][v] = 0.0;
          }
      newTile = false;
    }
    if (hasNext) cp_async_wait<1>(); else cp_async_wait<0>();
    __syncthreads();
    const double *As = smem_upd + stage * kStage + wr + g, *Bs = smem_upd + stage * kStage + kPanel * kLdA + wc + g;
    const int kw = min(kPanel, cur.w - chunk * kPanel), wk = (kw + 15) & ~15;
    for (int kk = 0; kk < wk; kk += 16) {
      const double *Ak = As + (kk + t4) * kLdA, *Bk = Bs + (kk + t4) * kLdB;
      double bf[4][4];
#pragma unroll
      for (int b = 0; b < 4; b++)
#pragma unroll
        for (int v = 0; v < 4; v++) bf[b][v] = Bk[4 * v * kLdB + 8 * b];
#pragma unroll
      for (int a = 0; a < 2; a++) {
        double af[8];
#pragma unroll
        for (int v = 0; v < 8; v++) af[v] = Ak[4 * (v >> 1) * kLdA + 16 * a + 8 * (v & 1)];
#pragma unroll
        for (int b = 0; b < 4; b++) dmma_16x8x16(acc[a][b], af, bf[b]);
      }
    }
    __syncthreads();  // this stage is free for the item after next
    stage ^= 1;
    if (sameTile) {
      chunk++;
      continue;
    }
    // last chunk of the tile: write C once
#pragma unroll
    for (int a = 0; a < 2; a++)
#pragma unroll
      for (int b = 0; b < 4; b++)
#pragma unroll
        for (int v = 0; v < 4; v++) {
          const int i = ii[a][v >> 1], j = jj[b][v & 1];
          if (i < m && i >= j) cp[b][v & 1][i] = cpre[a][b][v] - acc[a][b][v];
        }
    if (!hasNext) break;
    t += gridDim.x;
    cur = nxtTask;
    if (t + (int)gridDim.x < ntasks) nxtTask = tasks[t + gridDim.x];
    chunk = 0;
    nch = (cur.w + kPanel - 1) / kPanel;
    newTile = true;
  }
}


// Complex-symmetric update tiles (no conjugation): F[i0:i0+128, j0:j0+64] -= W B^T with W = L21 D (the A operand of
// the LDL^T update) and B = L21, K = the task's pivot columns, on the CUDA cores (four FP64 products per complex
// product). One CTA per tile: 256 threads as 32 (rows) x 8 (columns), 4 x 8 outputs each; K in chunks of 8 staged
// in shared memory. Same tiles and masks as k_update.
__global__ void __launch_bounds__(256) k_update_c(const TileTask *__restrict__ tasks, cplx *__restrict__ Lx,
                                                  cplx *__restrict__ U, const cplx *__restrict__ W,
                                                  const unsigned long long *status) {
  __shared__ int sOk;
  if (threadIdx.x == 0) sOk = !failed(status);
  __syncthreads();
  if (!sOk) return;
  const TileTask t = tasks[blockIdx.x];
  constexpr int KC = 8;
  __shared__ cplx As[KC][kTileM], Bs[KC][kTile];
  const int tid = threadIdx.x, tr = tid & 31, tc = tid >> 5;
  const int m = t.m, nc = t.nc, mu = m - nc;
  const cplx *Ap = W + t.lp, *Bp = Lx + t.lp;
  cplx acc[4][8];
#pragma unroll
  for (int a = 0; a < 4; a++)
#pragma unroll
    for (int b = 0; b < 8; b++) acc[a][b] = cplx(0.0);
  for (int k0 = 0; k0 < t.w; k0 += KC) {
    for (int e = tid; e < KC * kTileM; e += 256) {
      const int k = e / kTileM, i = e % kTileM, r = t.i0 + i;
      As[k][i] = (k0 + k < t.w && r < m) ? Ap[(int64_t)(t.c0 + k0 + k) * m + r] : cplx(0.0);
    }
    for (int e = tid; e < KC * kTile; e += 256) {
      const int k = e / kTile, j = e % kTile, r = t.j0 + j;
      Bs[k][j] = (k0 + k < t.w && r < m) ? Bp[(int64_t)(t.c0 + k0 + k) * m + r] : cplx(0.0);
    }
    __syncthreads();
#pragma unroll 4
    for (int k = 0; k < KC; k++) {
      cplx av[4], bv[8];
#pragma unroll
      for (int a = 0; a < 4; a++) av[a] = As[k][tr + 32 * a];
#pragma unroll
      for (int b = 0; b < 8; b++) bv[b] = Bs[k][tc + 8 * b];
#pragma unroll
      for (int a = 0; a < 4; a++)
#pragma unroll
        for (int b = 0; b < 8; b++) acc[a][b] += av[a] * bv[b];
    }
    __syncthreads();
  }
  cplx *Lp = Lx + t.lp;
  cplx *Up = t.up >= 0 ? U + t.up : Lp;
#pragma unroll
  for (int a = 0; a < 4; a++)
#pragma unroll
    for (int b = 0; b < 8; b++) {
      const int i = t.i0 + tr + 32 * a, j = t.j0 + tc + 8 * b;
      if (i < m && j < t.jend && i >= j) {
        cplx *c = j < nc ? Lp + (int64_t)j * m + i : Up + (int64_t)(j - nc) * mu + (i - nc);
        *c = *c - acc[a][b];
      }
    }
}

// ---------------------------------------------------------------------------------------------------------------
// Solves. Vectors: q right-hand sides stored one after another (y[k n + i]) in the permuted order.
// ---------------------------------------------------------------------------------------------------------------
__global__ void k_permute_in(const double *__restrict__ b, double *__restrict__ y, const int *__restrict__ perm, int n,
                             int q) {
  int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (int64_t)n * q) return;
  int k = (int)(idx / n), i = (int)(idx % n);
  y[idx] = b[(int64_t)k * n + perm[i]];
}

__global__ void k_permute_out(const double *__restrict__ y, double *__restrict__ x, const int *__restrict__ perm, int n,
                              int q) {
  int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (int64_t)n * q) return;
  int k = (int)(idx / n), i = (int)(idx % n);
  x[(int64_t)k * n + perm[i]] = y[idx];
}

// ---------------------------------------------------------------------------------------------------------------
// Launchers (host side)
// ---------------------------------------------------------------------------------------------------------------
static int g_num_sms = 148;

cudaError_t init_mixed_attributes();
cudaError_t init_solve_attributes();
cudaError_t init_solve_multi_attributes();
cudaError_t init_front_small_attributes();
cudaError_t init_kernel_attributes() {
  // function attributes belong to the current device's context: the caller runs this once per device
  cudaError_t e =
      cudaFuncSetAttribute(k_group_panel<double, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, kGroupSmem);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_group_panel<double, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kGroupSmem);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_group_panel<float, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, kGroupSmem / 2);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_group_panel<cplx, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, kGroupSmem * 2);
  if (e == cudaSuccess) e = init_mixed_attributes();
  if (e == cudaSuccess) e = init_solve_attributes();
  if (e == cudaSuccess) e = init_solve_multi_attributes();
  if (e == cudaSuccess) e = init_front_small_attributes();
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_update, cudaFuncAttributeMaxDynamicSharedMemorySize, kUpdateSmem);
  int dev = 0;
  if (e == cudaSuccess) e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&g_num_sms, cudaDevAttrMultiProcessorCount, dev);
  return e;
}

template <class T>
void launch_assemble(const AsmTask *tasks, const ChildRange *ranges, int64_t ntasks, const DevPlan &P,
                     const value_of<T> *values, T *Lx, T *U, const unsigned long long *status, cudaStream_t st) {
  if (ntasks > 0) k_assemble<T><<<(unsigned)ntasks, 256, 0, st>>>(tasks, ranges, P, values, Lx, U, status);
}
template void launch_assemble<double>(const AsmTask *, const ChildRange *, int64_t, const DevPlan &, const double *,
                                      double *, double *, const unsigned long long *, cudaStream_t);
template void launch_assemble<float>(const AsmTask *, const ChildRange *, int64_t, const DevPlan &, const double *,
                                     float *, float *, const unsigned long long *, cudaStream_t);
template void launch_assemble<cplx>(const AsmTask *, const ChildRange *, int64_t, const DevPlan &, const cplx *,
                                    cplx *, cplx *, const unsigned long long *, cudaStream_t);
template <class T>
void launch_group_panel(const GroupItem *items, const StripTask *strips, int nstrips, int *ticket, int *flags,
                        const DevPlan &P, T *Lx, unsigned long long *status, __nv_bfloat16 *Shi, __nv_bfloat16 *Slo,
                        const LdltArgs<T> &ld, cudaStream_t st) {
  if (nstrips <= 0) return;
  const size_t smem = 3 * kPanel * (kPanel + 1) * sizeof(T);
  if constexpr (std::is_same<T, double>::value)  // Bunch-Kaufman pivot blocks (FP64 LDL^T with ld.piv set)
    if (ld.piv) {
      k_group_panel<T, true><<<(unsigned)nstrips, 256, smem, st>>>(items, strips, nstrips, ticket, flags, P, Lx, status,
                                                                  Shi, Slo, ld);
      return;
    }
  k_group_panel<T, false><<<(unsigned)nstrips, 256, smem, st>>>(items, strips, nstrips, ticket, flags, P, Lx, status, Shi,
                                                               Slo, ld);
}
template void launch_group_panel<double>(const GroupItem *, const StripTask *, int, int *, int *, const DevPlan &,
                                         double *, unsigned long long *, __nv_bfloat16 *, __nv_bfloat16 *,
                                         const LdltArgs<double> &, cudaStream_t);
template void launch_group_panel<float>(const GroupItem *, const StripTask *, int, int *, int *, const DevPlan &,
                                        float *, unsigned long long *, __nv_bfloat16 *, __nv_bfloat16 *,
                                        const LdltArgs<float> &, cudaStream_t);
template void launch_group_panel<cplx>(const GroupItem *, const StripTask *, int, int *, int *, const DevPlan &,
                                       cplx *, unsigned long long *, __nv_bfloat16 *, __nv_bfloat16 *,
                                       const LdltArgs<cplx> &, cudaStream_t);

void launch_update_c(const TileTask *tasks, int64_t ntasks, cplx *Lx, cplx *U, const cplx *W,
                     const unsigned long long *status, cudaStream_t st) {
  if (ntasks > 0) k_update_c<<<(unsigned)ntasks, 256, 0, st>>>(tasks, Lx, U, W, status);
}
void launch_ldlt_tau(const double *values, const DevPlan &P, double *scal, cudaStream_t st) {
  k_ldlt_tau<<<1, 1024, 0, st>>>(values, P.diagSlot, P.n, scal);
}
int num_sms() { return g_num_sms; }
void launch_update(const TileTask *tasks, int64_t ntasks, const DevPlan &P, double *Lx, double *U, const double *W,
                   const unsigned long long *status, cudaStream_t st) {
  (void)P;
  const int grid = (int)std::min<int64_t>(ntasks, g_num_sms);
  if (ntasks > 0) k_update<<<grid, 256, kUpdateSmem, st>>>(tasks, (int)ntasks, Lx, U, W, status);
}
void launch_permute_in(const double *b, double *y, const int *perm, int n, int q, cudaStream_t st) {
  int64_t tot = (int64_t)n * q;
  if (tot > 0) k_permute_in<<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(b, y, perm, n, q);
}
void launch_permute_out(const double *y, double *x, const int *perm, int n, int q, cudaStream_t st) {
  int64_t tot = (int64_t)n * q;
  if (tot > 0) k_permute_out<<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(y, x, perm, n, q);
}
}  // namespace amp
