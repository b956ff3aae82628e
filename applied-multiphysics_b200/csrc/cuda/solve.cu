// Supernodal triangular solves on sm_100a (sparse.mjs solveNumeric :1261-1305, supernodalSolve :1200-1258).
//
// Multifrontal vector form, each sweep one launch over 64-row block tasks:
//   forward (tasks listed children before parents, the longest estimated path to the sweep's end first)
//     diagonal task (s, k)  block 0 first gathers v_s = [y(f .. f+nc); 0] + the children's pass-up vectors (extend-add
//                           in the reference's child order); then r_k = v_k - L[k, 0:k] y(0:k) (row-block dot products)
//                           and y_k = L_kk^-1 r_k as a 64 x 64 product with the precomputed inverse block
//     below task (s, j)     the pass-up vector u_j = v_j - L[j, 0:nc] y (read by the parent's gather)
//   backward (tasks listed parents before children, the same way; blocks of a supernode from the last down)
//     x_k = L_kk^-T (y_k - L[rows below k, k]^T x(rows)), the rows below the supernode gathered from the ancestors'
//     final values
// Every L element is read once per sweep. Persistent CTAs (3 per SM) take the next task with an atomic ticket (so a
// task only ever waits for tasks already taken by running or finished CTAs) and wait on per-block ready flags with a
// bounded spin; on time-out a CTA records AMP_DEVICE_TIMEOUT in the status word and returns. The L values a task
// needs from a block are loaded before it waits for that block's flag, so the dependency chain through a large
// supernode costs a flag round trip, 64 y values and a 64 x 64 product per block.
//
// The inverses of the diagonal blocks are computed once per factorization, after it (k_diag_inv, all blocks of the
// supernodes solved by block tasks (m > 32; the smaller ones are solved by one warp each, by substitution) in
// parallel): column j of X = L_kk^-1 by forward substitution, X(j, j) = 1 / L(j, j),
// X(i, j) = -(sum_{t=j}^{i-1} L(i, t) X(t, j)) X(i, i). Solving with X instead of by substitution changes the result
// by rounding only (the FP64 path stays within 1e-12 of the oracle).
#include <cuda_runtime.h>

#include <cstdint>

#include "../host/plan.hpp"
#include "devplan.cuh"
#include "solve_small.cuh"
#include "sync.cuh"

namespace amp {

constexpr int kSB = 64;  // solve block rows

// ---- inverses of the diagonal blocks -----------------------------------------------------------------------------
// One CTA per 64-column block b of the pivot columns (all supernodes): X = L_kk^-1, w x w column-major, lower part.
// The block's lower triangle is staged in shared memory (coalesced column loads); then a group of 4 lanes computes
// column j by forward substitution, X(j, j) = 1 / L(j, j), X(i, j) = -(sum_{t=j}^{i-1} L(i, t) X(t, j)) / L(i, i),
// lane p summing the terms t = j + p, j + p + 4, ... (two shuffles complete the sum) and keeping the entries X(t, j)
// of its own terms, so that the group needs no barrier between rows. Shared layouts: Ls[t][i] = L(i, t), 65 entries
// per column; Xs[j][t] = X(t, j), one 64-entry row per column (a group's lanes read consecutive entries).
// For a Bunch-Kaufman factor the stored block is
// X P_b (P_b the block's pivot order, a full w x w matrix): the forward sweep's r, taken in the original order of the
// block's rows, becomes y_b = X P_b r, and the backward sweep's x_b = (X P_b)^T r lands in that original order, so
// L's earlier columns keep the rows of later blocks in their original order (the interchanges are not applied to
// the left of a block) and the sweeps need no other change.
constexpr int kInvThreads = 4 * kSB;
template <class TL>
constexpr int diag_inv_smem() {
  return kSB * kSB * (int)sizeof(double) + kSB * (kSB + 1) * (int)sizeof(TL);
}
template <class TL>
__global__ void __launch_bounds__(kInvThreads) k_diag_inv(const int *__restrict__ blocks, DevPlan P,
                                                          const TL *__restrict__ Lx, TL *__restrict__ Inv) {
  extern __shared__ double inv_dyn[];
  double(*Xs)[kSB] = reinterpret_cast<double(*)[kSB]>(inv_dyn);
  TL(*Ls)[kSB + 1] = reinterpret_cast<TL(*)[kSB + 1]>(inv_dyn + kSB * kSB);
  __shared__ double dinv[kSB];
  __shared__ int kOf[kSB];
  const int b = blocks[blockIdx.x];
  int lo = 0, hi = P.nsuper;  // supernode s with blkOff[s] <= b < blkOff[s + 1]
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (P.blkOff[mid] <= b) lo = mid; else hi = mid;
  }
  const int s = lo, c0 = (b - P.blkOff[s]) * kSB;
  const int m = P.snM[s], w = min(kSB, P.snNc[s] - c0);
  const TL *Lb = Lx + P.snLxp[s] + (int64_t)c0 * m + c0;  // L_kk(i, t) = Lb[t m + i]
  const int tid = threadIdx.x;
  for (int e = tid; e < kSB * kSB; e += kInvThreads) {
    const int t = e >> 6, i = e & (kSB - 1);
    if (t < w && i >= t && i < w) Ls[t][i] = __ldg(Lb + (int64_t)t * m + i);
  }
  __syncthreads();
  if (tid < w) dinv[tid] = 1.0 / (double)Ls[tid][tid];
  __syncthreads();
  const int j = tid >> 2, p = tid & 3;
  if (j < w) {  // the 4 lanes of a group share j, so they take the same branches and trip counts
    const unsigned gmask = 0xfu << (threadIdx.x & 28);
    if (p == 0) Xs[j][j] = dinv[j];
    for (int i = j + 1; i < w; i++) {
      double acc = 0.0;
      for (int t = j + p; t < i; t += 4) acc += (double)Ls[t][i] * Xs[j][t];
      acc += __shfl_xor_sync(gmask, acc, 1);
      acc += __shfl_xor_sync(gmask, acc, 2);
      if (((i - j) & 3) == p) Xs[j][i] = -acc * dinv[i];  // read later by this lane only
    }
  }
  __syncthreads();
  TL *X = Inv + P.invOff[b];
  if (P.lpiv) {  // Bunch-Kaufman factor: X P_b, column piv(k) of it = column k of X (P_b r = r(piv(.)))
    if (tid < w) kOf[__ldg(P.lpiv + P.snF[s] + c0 + tid)] = tid;
    __syncthreads();
    for (int e = tid; e < w * w; e += kInvThreads) {
      const int i = e % w, k = kOf[e / w];
      X[e] = (TL)(i >= k ? Xs[k][i] : 0.0);
    }
    return;
  }
  for (int e = tid; e < w * w; e += kInvThreads) {
    const int i = e % w, jj = e / w;
    X[e] = (TL)(i >= jj ? Xs[jj][i] : 0.0);
  }
}

// ---- chain matrices ----------------------------------------------------------------------------------------------
// For consecutive 64-column diagonal blocks b - 1, b of a supernode (after the factorization, after k_diag_inv):
//   M_b = X_b L[b, b-1]   (w_b x 64): forward  y_b = X_b (v_b - P_b) - M_b y_{b-1}
//   G_b = L[b+1, b] X_b   (w_{b+1} x w_b): backward x_b = X_b^T (r_b - Q_b) - G_b^T x_{b+1}
// with P_b / Q_b the contributions of all other blocks, so that only one 64 x 64 product waits for the neighbouring
// block. Slots: supernode s's block b uses M slot blkOff[s] - s + b - 1 and G slot blkOff[s] - s + b (64 x 64,
// column-major), since a supernode with nb blocks has nb - 1 of each.
constexpr int kChainSmem = 2 * kSB * (kSB + 1) * (int)sizeof(double);
template <class TL>
__global__ void __launch_bounds__(256) k_chain_mats(const int2 *__restrict__ tasks, DevPlan P, const TL *__restrict__ Lx,
                                                    const TL *__restrict__ Inv, TL *__restrict__ Mch,
                                                    TL *__restrict__ Gch) {
  extern __shared__ double ch_dyn[];
  double(*Xs)[kSB + 1] = reinterpret_cast<double(*)[kSB + 1]>(ch_dyn);
  double(*Lt)[kSB + 1] = reinterpret_cast<double(*)[kSB + 1]>(ch_dyn + kSB * (kSB + 1));
  const int2 t = tasks[blockIdx.x];
  const int s = t.x, b = t.y;
  const int nc = P.snNc[s], m = P.snM[s], nb = (nc + kSB - 1) / kSB;
  const int c0 = b * kSB, w = min(kSB, nc - c0);
  const TL *Lp = Lx + P.snLxp[s];
  const TL *X = Inv + P.invOff[P.blkOff[s] + b];
  const int tid = threadIdx.x, i = tid & (kSB - 1), cg = tid >> 6;
  for (int e = tid; e < kSB * kSB; e += blockDim.x) {
    const int r = e & (kSB - 1), c = e >> 6;
    Xs[r][c] = (r < w && c < w) ? (double)X[c * w + r] : 0.0;  // X(r, c), lower
  }
  const int slotBase = P.blkOff[s] - s;
  if (b >= 1) {  // M(i, c) = sum_{j <= i} X(i, j) L(c0 + j, c0 - 64 + c)
    for (int e = tid; e < kSB * kSB; e += blockDim.x) {
      const int j = e & (kSB - 1), c = e >> 6;
      Lt[j][c] = j < w ? (double)Lp[(int64_t)(c0 - kSB + c) * m + c0 + j] : 0.0;
    }
    __syncthreads();
    TL *M = Mch + (int64_t)(slotBase + b - 1) * kSB * kSB;
    double a[16];  // M(i, cg 16 + u); each X(i, j) read once for the 16 columns (Lt[j][.] broadcast in the warp)
#pragma unroll
    for (int u = 0; u < 16; u++) a[u] = 0.0;
    for (int j = 0; j <= i && j < w; j++) {
      const double x = Xs[i][j];
#pragma unroll
      for (int u = 0; u < 16; u++) a[u] += x * Lt[j][cg * 16 + u];
    }
#pragma unroll
    for (int u = 0; u < 16; u++) M[(cg * 16 + u) * kSB + i] = (TL)a[u];
    __syncthreads();
  }
  if (b + 1 < nb) {  // G(r, c) = sum_{j >= c} L(c0 + 64 + r, c0 + j) X(j, c)
    const int wn = min(kSB, nc - c0 - kSB);
    for (int e = tid; e < kSB * kSB; e += blockDim.x) {
      const int r = e & (kSB - 1), j = e >> 6;
      Lt[r][j] = (r < wn && j < w) ? (double)Lp[(int64_t)(c0 + j) * m + c0 + kSB + r] : 0.0;
    }
    __syncthreads();
    TL *G = Gch + (int64_t)(slotBase + b) * kSB * kSB;
    double a[16];  // G(i, cg 16 + u) = sum over j >= c of L(i, j) X(j, c); each L(i, j) read once
#pragma unroll
    for (int u = 0; u < 16; u++) a[u] = 0.0;
    for (int j = cg * 16; j < w; j++) {
      const double l = Lt[i][j];
#pragma unroll
      for (int u = 0; u < 16; u++)
        if (j >= cg * 16 + u) a[u] += l * Xs[j][cg * 16 + u];
    }
#pragma unroll
    for (int u = 0; u < 16; u++) G[(cg * 16 + u) * kSB + i] = (TL)a[u];
  }
}

// ---- forward block tasks -----------------------------------------------------------------------------------------
constexpr int kChPre = 64;  // children located and waited for at once by a forward block task
// task: .x supernode, .y block, .z kind (0 diagonal, 1 below, 2 small supernodes, 3 whole supernode: one-vector list)
// One launch for the whole sweep: a supernode's tasks are listed after its children's, so every wait is on a task
// with an earlier ticket. Every task first waits for the supernode's children and gathers its own rows of the front vector
// v_s = [y(f .. f + nc); 0] + the children's pass-up vectors (in the reference's child order). A below task forms its
// part of the pass-up vector u_j = v_j - L[j, 0:nc] y and counts itself in done[s]; diagonal task b forms
// w_b = X_b (v_b - L[b, 0:(b-1) 64] y) while the earlier blocks finish, then waits for block b - 1 alone:
// y_b = w_b - M_b y_{b-1}.
template <class TL>
__global__ void __launch_bounds__(256, 3) k_fwd_blocks(const int4 *__restrict__ tasks, int ntasks, int *__restrict__ ticket,
                                                    DevPlan P, const TL *__restrict__ Lx, const TL *__restrict__ Inv,
                                                    const TL *__restrict__ Mch, double *__restrict__ y,
                                                    double *__restrict__ T, int *__restrict__ flags,
                                                    unsigned long long *__restrict__ hand, int epoch,
                                                    int *__restrict__ done, unsigned long long *status) {
  __shared__ int tk, waitOk;
  __shared__ unsigned hw[2 * kSB];
  __shared__ double red[4][kSB];
  __shared__ double rk[kSB];
  __shared__ double Xs[kSB][kSB + 1];
  __shared__ int2 chA[kChPre];
  __shared__ int64_t chMap[kChPre], chT[kChPre];
  __shared__ double vs[kWholeFront];
  // kind 3: the whole supernode s (nc <= 64, m <= kWholeFront): gather its front vector v (all m rows) in shared
  // memory, y = X v[0:nc), then u = v - L[rows below, :] y in 64-row chunks (L values loaded a chunk ahead, the first
  // chunk before the waits); the same arithmetic, term by term, as a diagonal task and its below tasks
  auto whole = [&](const int s) -> bool {
    const int f = P.snF[s], nc = P.snNc[s], m = P.snM[s], mu = m - nc;
    const TL *Lp = Lx + P.snLxp[s];
    const int tid = threadIdx.x, row = tid & (kSB - 1), part = tid >> 6;
    {
      const TL *X = Inv + P.invOff[P.blkOff[s]];
      for (int e = tid; e < nc * nc; e += blockDim.x) Xs[e % nc][e / nc] = (double)X[e];
    }
    TL lv[16];
    auto loadChunk = [&](int j, TL (&dst)[16]) {
      const int r = nc + j * kSB + row;
#pragma unroll
      for (int u = 0; u < 16; u++) {
        const int c = part + 4 * u;
        dst[u] = (r < m && c < nc) ? Lp[(int64_t)c * m + r] : (TL)0;
      }
    };
    loadChunk(0, lv);
    for (int r = tid; r < m; r += blockDim.x) vs[r] = r < nc ? y[f + r] : 0.0;
    // children: metadata and waits in parallel, kChPre at a time; whole pass-up vectors added in child order
    const int q0 = P.chPtr[s], q1 = P.chPtr[s + 1];
    for (int qb = q0; qb < q1; qb += kChPre) {
      const int nq = min(kChPre, q1 - qb);
      if (qb > q0) __syncthreads();  // the previous chunk's metadata is consumed
      int ok = 1;
      if (tid < nq) {
        const int c = P.chList[qb + tid];
        const int muc = P.snM[c] - P.snNc[c];
        chA[tid] = make_int2(0, muc);
        chMap[tid] = P.eaPtr[c];
        chT[tid] = P.snTOff[c];
        ok = wait_count(done + c, (muc + kSB - 1) / kSB, status, s, P.spin);
      }
      if (!__syncthreads_and(ok)) return false;  // block-uniform
      for (int q = 0; q < nq; q++) {
        const int *map = P.eaMap + chMap[q];
        const double *tc = T + chT[q];
        for (int a = tid; a < chA[q].y; a += blockDim.x) vs[map[a]] += __ldcg(tc + a);
        __syncthreads();
      }
    }
    if (q0 == q1) __syncthreads();
    {  // y = X v[0:nc): thread (row, part) sums columns part, part + 4, ... <= row
      double a2 = 0.0;
      const int cend = P.lpiv ? nc - 1 : row;  // X P_b is full for a Bunch-Kaufman factor
      if (row < nc)
        for (int c = part; c <= cend; c += 4) a2 += Xs[row][c] * vs[c];
      red[part][row] = a2;
    }
    __syncthreads();
    if (tid < kSB) {
      const double yv = tid < nc ? (red[0][tid] + red[1][tid]) + (red[2][tid] + red[3][tid]) : 0.0;
      rk[tid] = yv;
      if (tid < nc) y[f + tid] = yv;
    }
    __syncthreads();
    const int nch = (mu + kSB - 1) / kSB;
    for (int j = 0; j < nch; j++) {
      TL ln[16];
      loadChunk(j + 1, ln);
      double acc = 0.0;
#pragma unroll
      for (int u = 0; u < 16; u++) {
        const int c = part + 4 * u;
        if (c < nc) acc += (double)lv[u] * rk[c];
      }
      red[part][row] = acc;
      __syncthreads();
      const int r0 = nc + j * kSB;
      if (tid < min(kSB, m - r0))
        T[P.snTOff[s] + j * kSB + tid] = vs[r0 + tid] - ((red[0][tid] + red[1][tid]) + (red[2][tid] + red[3][tid]));
      __syncthreads();  // red is reused by the next chunk
#pragma unroll
      for (int u = 0; u < 16; u++) lv[u] = ln[u];
    }
    if (tid == 0) {  // after the barrier: the CTA's stores of y and T are ordered before both
      st_release(flags + P.blkOff[s], epoch);
      if (nch > 0) red_release_add(done + s, nch);
    }
    return true;
  };
  auto run = [&](const int tkv) -> bool {
    const int4 t = tasks[tkv];
    if (t.z == 3) return whole(t.x);
    if (t.z == 2) {  // up to kSolveGroup supernodes with m <= 32, one warp each
      const int warp = threadIdx.x >> 5;
      if (threadIdx.x == 0) waitOk = 1;
      __syncthreads();
      if (warp < t.y && !small_fwd_warp<TL>(P.solveSmall[t.x + warp], P, Lx, y, T, done, status, &red[0][0] + 32 * warp))
        waitOk = 0;
      __syncthreads();
      return waitOk != 0;
    }
    const int s = t.x, blk = t.y, below = t.z;
    const int f = P.snF[s], nc = P.snNc[s], m = P.snM[s], mu = m - nc;
    const TL *Lp = Lx + P.snLxp[s];
    const int r0 = below ? nc + blk * kSB : blk * kSB;
    const int rows = below ? min(kSB, mu - blk * kSB) : min(kSB, nc - blk * kSB);
    // with chain matrices (Cholesky) the diagonal task sums blocks 0 .. b - 2 before its last wait and applies M_b to
    // block b - 1; without them (LDL^T, whose inverse blocks can be large) it sums all blocks before b and applies X_b
    // last, as the reference's substitution does
    const bool chain = Mch != nullptr;
    const int ncols = below ? nc : max(0, chain ? blk - 1 : blk) * kSB;  // columns summed before the last product
    const int tid = threadIdx.x, row = tid & (kSB - 1), part = tid >> 6;
    const bool rowok = row < rows;
    int *myflags = flags + P.blkOff[s];
    if (!below) {
      const TL *X = Inv + P.invOff[P.blkOff[s] + blk];
      for (int e = tid; e < rows * rows; e += blockDim.x) Xs[e % rows][e / rows] = (double)X[e];
    }
    // this task's rows of v: pivot rows start from y; the children's entries mapping to rows [r0, r0 + rows) are added
    // in child order (the map is increasing, so they form one range per child). Up to kChPre children at a time, one
    // per thread: the thread locates the child's range (static) and then waits for the child, so that the searches
    // and the waits of all children overlap.
    if (tid < kSB) rk[tid] = (tid < rows && r0 + tid < nc) ? y[f + r0 + tid] : 0.0;
    const int q0 = P.chPtr[s], q1 = P.chPtr[s + 1];
    for (int qb = q0; qb < q1; qb += kChPre) {
      const int nq = min(kChPre, q1 - qb);
      if (qb > q0) __syncthreads();  // the previous chunk's ranges are consumed
      int ok = 1;
      if (tid < nq) {
        const int c = P.chList[qb + tid];
        const int muc = P.snM[c] - P.snNc[c];
        const int *map = P.eaMap + P.eaPtr[c];
        int lo = 0, hi = muc;
        while (lo < hi) {
          const int mid = (lo + hi) >> 1;
          if (map[mid] < r0) lo = mid + 1; else hi = mid;
        }
        const int a0 = lo;
        hi = muc;
        while (lo < hi) {
          const int mid = (lo + hi) >> 1;
          if (map[mid] < r0 + rows) lo = mid + 1; else hi = mid;
        }
        chA[tid] = make_int2(a0, lo);
        chMap[tid] = P.eaPtr[c];
        chT[tid] = P.snTOff[c];
        ok = wait_count(done + c, (muc + kSB - 1) / kSB, status, s, P.spin);
      }
      if (!__syncthreads_and(ok)) return false;  // block-uniform
      for (int q = 0; q < nq; q++) {
        const int *map = P.eaMap + chMap[q];
        const double *tc = T + chT[q];
        for (int a = chA[q].x + tid; a < chA[q].y; a += blockDim.x) rk[map[a] - r0] += __ldcg(tc + a);
        __syncthreads();
      }
    }
    if (q0 == q1) __syncthreads();
    const double vreg = tid < kSB ? rk[tid] : 0.0;
    // sums over the columns of the finished blocks; a block's L values are loaded before waiting for its flag
    double acc = 0.0;
    {
      const int ncb = (ncols + kSB - 1) / kSB;
      TL lv[16];
#pragma unroll
      for (int u = 0; u < 16; u++) {
        const int c = part + 4 * u;
        lv[u] = (rowok && c < ncols) ? Lp[(int64_t)c * m + r0 + row] : (TL)0;
      }
      for (int cb = 0; cb < ncb; cb++) {
        TL ln[16];
        const int cn = (cb + 1) * kSB;
#pragma unroll
        for (int u = 0; u < 16; u++) {
          const int c = cn + part + 4 * u;
          ln[u] = (rowok && c < ncols) ? Lp[(int64_t)c * m + r0 + row] : (TL)0;
        }
        if (tid == 0) waitOk = wait_flag(myflags + cb, epoch, status, s, P.spin);
        __syncthreads();
        if (!waitOk) return false;  // block-uniform
        const int cbase = cb * kSB;
#pragma unroll
        for (int u = 0; u < 16; u++) {
          const int c = cbase + part + 4 * u;
          if (c < ncols) acc += (double)lv[u] * __ldcg(y + f + c);
        }
#pragma unroll
        for (int u = 0; u < 16; u++) lv[u] = ln[u];
      }
    }
    // diagonal b >= 1: M_b(row, part + 4 u), loaded now (the tiles above are dead) and used after the last wait
    TL mv[16];
    if (!below && chain && blk > 0) {
      const TL *M = Mch + (int64_t)(P.blkOff[s] - s + blk - 1) * kSB * kSB;
#pragma unroll
      for (int u = 0; u < 16; u++) mv[u] = rowok ? M[(part + 4 * u) * kSB + row] : (TL)0;
    }
    red[part][row] = acc;
    __syncthreads();
    if (below) {
      if (tid < rows)
        T[P.snTOff[s] + blk * kSB + tid] = vreg - ((red[0][tid] + red[1][tid]) + (red[2][tid] + red[3][tid]));
      __syncthreads();
      if (tid == 0) red_release_add(done + s, 1);
      return true;
    }
    if (tid < kSB) rk[tid] = tid < rows ? vreg - ((red[0][tid] + red[1][tid]) + (red[2][tid] + red[3][tid])) : 0.0;
    __syncthreads();
    // w_b = X_b (v_b - the sums so far), X_b lower triangular: thread (row, part) sums columns part, part + 4, ... <= row
    {
      double a2 = 0.0;
      const int cend = P.lpiv ? rows - 1 : row;  // X P_b is full for a Bunch-Kaufman factor
      if (rowok)
        for (int c = part; c <= cend; c += 4) a2 += Xs[row][c] * rk[c];
      red[part][row] = a2;
    }
    __syncthreads();
    const double wv = tid < rows ? (red[0][tid] + red[1][tid]) + (red[2][tid] + red[3][tid]) : 0.0;
    double yv = wv;
    // the chain step: y_b = w_b - M_b y_{b-1}, with y_{b-1} taken from block b - 1's tagged words (hand, two per
    // value, slot of M_b) as soon as they carry this sweep's epoch, without waiting for its flag
    const int nb = (nc + kSB - 1) / kSB;
    const int64_t slot0 = P.blkOff[s] - s;  // this supernode's chain slots: slot0 + b for the pair (b, b + 1)
    if (chain && blk > 0) {
      int ok = 1;
      if (tid < 2 * kSB) {
        unsigned lo = 0;
        ok = wait_tagged(hand + (slot0 + blk - 1) * 2 * kSB + tid, epoch, status, s, lo, P.spin);
        hw[tid] = lo;
      }
      if (!__syncthreads_and(ok)) return false;  // block-uniform
      double a3 = 0.0;
#pragma unroll
      for (int u = 0; u < 16; u++) {
        const int k = part + 4 * u;
        a3 += (double)mv[u] * untag(hw[2 * k], hw[2 * k + 1]);
      }
      red[part][row] = a3;
      __syncthreads();
      if (tid < rows) yv = wv - ((red[0][tid] + red[1][tid]) + (red[2][tid] + red[3][tid]));
    }
    if (tid < rows) {
      if (chain && blk + 1 < nb) st_tagged(hand + (slot0 + blk) * 2 * kSB + 2 * tid, epoch, yv);
      y[f + r0 + tid] = yv;
    }
    // every reader of a forward flag acquires each block's flag it needs on its own (the chain step, which takes
    // y_{b-1} from the tagged words, is the one reader that does not), so block b's flag need not stand for b - 1
    __syncthreads();
    if (tid == 0) st_release(myflags + blk, epoch);  // after the barrier: the CTA's stores are ordered before it
    return true;
  };
  for (;;) {
    if (threadIdx.x == 0) tk = atomicAdd(ticket, 1);
    __syncthreads();
    const int mine = tk;
    __syncthreads();
    if (mine >= ntasks || !run(mine)) return;
  }
}

// ---- backward block tasks ----------------------------------------------------------------------------------------
// task: .x supernode, .y column block (tasks of a supernode listed from the last block down), .z 0 or 2 (small)
// r_b = y_b - L[rows below the block, b]^T x(rows): the rows below the supernode (ancestors, final once the parent's
// first pivot block is) and the pivot blocks b + 2 and later accumulate in registers (warps own columns, lanes walk
// rows) and give w_b = X_b^T (r_b without block b + 1); then, after block b + 1's flag, x_b = w_b - G_b^T x_{b+1} with
// G_b staged in shared memory beforehand.
constexpr int kBwdSmem = 2 * kSB * (kSB + 1) * (int)sizeof(double);
template <class TL>
__global__ void __launch_bounds__(256, 3) k_bwd_blocks(const int4 *__restrict__ tasks, int ntasks, int *__restrict__ ticket,
                                                    DevPlan P, const TL *__restrict__ Lx, const TL *__restrict__ Inv,
                                                    const TL *__restrict__ Gch, const double *__restrict__ Dpiv,
                                                    double *__restrict__ y, int *__restrict__ flags,
                                                    unsigned long long *__restrict__ hand, int epoch,
                                                    unsigned long long *status) {
  __shared__ int tk, waitOk;
  __shared__ unsigned hw[2 * kSB];
  __shared__ double red[4][kSB];
  __shared__ double red0[kSB];
  __shared__ double xs[kSB];
  __shared__ double rk[kSB];
  extern __shared__ double bwd_dyn[];
  double(*Xs)[kSB + 1] = reinterpret_cast<double(*)[kSB + 1]>(bwd_dyn);                    // X_b
  double(*Gt)[kSB + 1] = reinterpret_cast<double(*)[kSB + 1]>(bwd_dyn + kSB * (kSB + 1));  // G_b, [r][c]
  auto run = [&](const int tkv) -> bool {
    const int4 t = tasks[tkv];
    if (t.z == 2) {  // up to kSolveGroup supernodes with m <= 32, one warp each
      const int warp = threadIdx.x >> 5;
      if (threadIdx.x == 0) waitOk = 1;
      __syncthreads();
      if (warp < t.y && !small_bwd_warp<TL>(P.solveSmall[t.x + warp], P, Lx, Dpiv, y, flags, epoch, status))
        waitOk = 0;
      __syncthreads();
      return waitOk != 0;
    }
    const int s = t.x, blk = t.y;
    const int f = P.snF[s], nc = P.snNc[s], m = P.snM[s];
    const TL *Lp = Lx + P.snLxp[s];
    const int *rowsOf = P.Si + P.Sp[s];
    const int c0 = blk * kSB, w = min(kSB, nc - c0), nb = (nc + kSB - 1) / kSB;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    // with chain matrices (Cholesky) block b + 1 is applied last through G_b; without them (LDL^T) it is summed with
    // the other blocks before X_b^T is applied
    const bool chain = Gch != nullptr;
    const bool hasNext = chain && blk + 1 < nb;
    const int rn = (blk + 1) * kSB, wn = hasNext ? min(kSB, nc - rn) : 0;  // the next pivot block: rows [rn, rn + wn)
    const int rbLast = chain ? blk + 1 : blk;  // pivot blocks above rbLast are summed in registers
    int *myflags = flags + P.blkOff[s];
    {
      const TL *X = Inv + P.invOff[P.blkOff[s] + blk];
      for (int e = tid; e < w * w; e += blockDim.x) Xs[e % w][e / w] = (double)X[e];
      if (hasNext) {
        const TL *G = Gch + (int64_t)(P.blkOff[s] - s + blk) * kSB * kSB;
        for (int e = tid; e < kSB * kSB; e += blockDim.x) {
          const int r = e & (kSB - 1), c = e >> 6;
          Gt[r][c] = (r < wn && c < w) ? (double)G[c * kSB + r] : 0.0;
        }
      }
    }
    double acc[8];
#pragma unroll
    for (int u = 0; u < 8; u++) acc[u] = 0.0;
    // Rows of the supernode below its pivot columns (ancestors' rows, ascending), from the last down in chunks of 32
    // (lane = row; warps over the columns). One launch covers the whole sweep (parents listed first), and the parent's
    // pivot blocks become final from its last block down, each block's flag set only after the next one's (rows
    // above the parent's pivot columns are final before its last block is). So a chunk waits only for the parent's
    // block that holds its first row, and the chunks of rows in the parent's later blocks are summed while the
    // parent's earlier blocks are still being solved. Each warp waits on its own (lane 0, bounded).
    bool wok = true;
    const int mu = m - nc;
    if (mu > 0) {
      const int par = P.snParent[s];
      const int fp = P.snF[par], ncp = P.snNc[par], nbp = (ncp + kSB - 1) / kSB;
      const int *pflags = flags + P.blkOff[par];
      int ready = nbp;  // the parent's blocks >= ready are known final (warp-uniform)
      // the chunk's row indices and L values (static) are loaded one chunk ahead, so that a chunk waits for one load
      // round trip (its x values) after its flag
      int rb = nc + ((mu - 1) / 32) * 32;
      int idx = rb + lane < m ? rowsOf[rb + lane] : -1;
      TL lc[8];
#pragma unroll
      for (int u = 0; u < 8; u++) {
        const int c = warp + 8 * u;
        lc[u] = (idx >= 0 && c < w) ? Lp[(int64_t)(c0 + c) * m + rb + lane] : (TL)0;
      }
      for (; rb >= nc; rb -= 32) {
        const int rbn = rb - 32;  // the next chunk (rows below rb, all < m)
        const int idxn = rbn >= nc ? rowsOf[rbn + lane] : -1;
        TL ln[8];
#pragma unroll
        for (int u = 0; u < 8; u++) {
          const int c = warp + 8 * u;
          ln[u] = (idxn >= 0 && c < w) ? Lp[(int64_t)(c0 + c) * m + rbn + lane] : (TL)0;
        }
        // the chunk's first row, lane 0's (>= fp: every row below is a row of the parent's front)
        const int g0 = __shfl_sync(0xffffffffu, idx, 0);
        const int k = g0 < fp + ncp ? max(0, g0 - fp) / kSB : nbp - 1;
        if (k < ready && wok) {
          wok = warp_wait(pflags + k, epoch, true, status, s, P.spin);
          ready = k;
        }
        if (idx >= 0 && wok) {
          const double xr = __ldcg(y + idx);
#pragma unroll
          for (int u = 0; u < 8; u++) acc[u] += (double)lc[u] * xr;
        }
        idx = idxn;
#pragma unroll
        for (int u = 0; u < 8; u++) lc[u] = ln[u];
      }
    }
    if (!__syncthreads_and(wok)) return false;  // block-uniform
    // pivot blocks after the next one, as they become final; a block's L values are loaded before its wait
    TL lv[2][8];
    auto load_block = [&](int rb, TL (&dst)[2][8]) {
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const int r = rb * kSB + lane + 32 * h;
#pragma unroll
        for (int u = 0; u < 8; u++) {
          const int c = warp + 8 * u;
          dst[h][u] = (rb > rbLast && r < nc && c < w) ? Lp[(int64_t)(c0 + c) * m + r] : (TL)0;
        }
      }
    };
    load_block(nb - 1, lv);
    for (int rb = nb - 1; rb > rbLast; rb--) {
      TL ln[2][8];
      load_block(rb - 1, ln);
      if (tid == 0) waitOk = wait_flag(myflags + rb, epoch, status, s, P.spin);
      __syncthreads();
      if (!waitOk) return false;  // block-uniform
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const int r = rb * kSB + lane + 32 * h;
        const double xr = r < nc ? __ldcg(y + f + r) : 0.0;
#pragma unroll
        for (int u = 0; u < 8; u++) acc[u] += (double)lv[h][u] * xr;
      }
#pragma unroll
      for (int h = 0; h < 2; h++)
#pragma unroll
        for (int u = 0; u < 8; u++) lv[h][u] = ln[h][u];
    }
#pragma unroll
    for (int u = 0; u < 8; u++) {
      double v = acc[u];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
      if (lane == 0) red0[warp + 8 * u] = v;
    }
    __syncthreads();
    if (tid < kSB) {
      double yv = 0.0;  // LDL^T: y /= D before the backward sweep (ldlt.mjs:629)
      if (tid < w) yv = Dpiv ? y[f + c0 + tid] / Dpiv[f + c0 + tid] : y[f + c0 + tid];
      rk[tid] = tid < w ? yv - red0[tid] : 0.0;
    }
    __syncthreads();
    // w_b = X_b^T r: thread (i, part) sums X(j, i) r(j) over j = i + part, i + part + 4, ... < w
    {
      const int i = tid & (kSB - 1), part = tid >> 6;
      double a2 = 0.0;
      if (i < w)
        for (int j = (P.lpiv ? 0 : i) + part; j < w; j += 4) a2 += Xs[j][i] * rk[j];  // X P_b full (Bunch-Kaufman)
      red[part][i] = a2;
    }
    __syncthreads();
    const double wv = tid < w ? (red[0][tid] + red[1][tid]) + (red[2][tid] + red[3][tid]) : 0.0;
    double xv = wv;
    const int64_t slot0 = P.blkOff[s] - s;  // this supernode's chain slots: slot0 + b for the pair (b, b + 1)
    if (hasNext) {  // the chain step: x_b = w_b - G_b^T x_{b+1}, x_{b+1} from block b + 1's tagged words
      int ok = 1;
      if (tid < 2 * wn) {
        unsigned lo = 0;
        ok = wait_tagged(hand + (slot0 + blk) * 2 * kSB + tid, epoch, status, s, lo, P.spin);
        hw[tid] = lo;
      }
      if (!__syncthreads_and(ok)) return false;  // block-uniform
      if (tid < kSB) xs[tid] = tid < wn ? untag(hw[2 * tid], hw[2 * tid + 1]) : 0.0;
      __syncthreads();
      const int c = tid & (kSB - 1), part = tid >> 6;
      double a3 = 0.0;
#pragma unroll 4
      for (int r = part; r < wn; r += 4) a3 += Gt[r][c] * xs[r];
      red[part][c] = a3;
      __syncthreads();
      if (tid < w) xv = wv - ((red[0][tid] + red[1][tid]) + (red[2][tid] + red[3][tid]));
    }
    if (tid < w) {
      if (chain && blk > 0) st_tagged(hand + (slot0 + blk - 1) * 2 * kSB + 2 * tid, epoch, xv);
      y[f + c0 + tid] = xv;
    }
    // block b's flag stands for every later block (the children's rows-below waits rely on it): acquire block
    // b + 1's flag, taken above without an acquire, before releasing ours after the barrier
    int fok = 1;
    if (tid == 0 && hasNext) fok = wait_flag(myflags + blk + 1, epoch, status, s, P.spin);
    if (!__syncthreads_and(fok)) return false;  // block-uniform
    if (tid == 0) st_release(myflags + blk, epoch);
    return true;
  };
  for (;;) {
    if (threadIdx.x == 0) tk = atomicAdd(ticket, 1);
    __syncthreads();
    const int mine = tk;
    __syncthreads();
    if (mine >= ntasks || !run(mine)) return;
  }
}

// D solve of a Bunch-Kaufman factor between the sweeps (y /= D, ldlt.mjs:629, with its 2 x 2 pivots): q interleaved
// vectors (y[j q + k]); the first row of a 2 x 2 pivot (Doff[j] != 0) solves both rows with the inverse of bk_block.
__global__ void k_dsolve_bk(int n, int q, const double *__restrict__ D, const double *__restrict__ Doff,
                            double *__restrict__ y) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (int64_t)n * q) return;
  const int j = (int)(idx / q);
  const double e = Doff[j];
  if (j > 0 && Doff[j - 1] != 0.0) return;  // the second row of a 2 x 2 pivot
  if (e == 0.0) {
    y[idx] = y[idx] / D[j];
    return;
  }
  const double a = D[j] / e, c = D[j + 1] / e, te = (1.0 / (a * c - 1.0)) / e;
  const double y0 = y[idx], y1 = y[idx + q];
  y[idx] = te * (c * y0 - y1);
  y[idx + q] = te * (a * y1 - y0);
}
void launch_dsolve_bk(int n, int q, const double *D, const double *Doff, double *y, cudaStream_t st) {
  const int64_t tot = (int64_t)n * q;
  if (tot > 0) k_dsolve_bk<<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(n, q, D, Doff, y);
}

cudaError_t init_solve_attributes() {
  cudaError_t e = cudaFuncSetAttribute(k_bwd_blocks<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, kBwdSmem);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_bwd_blocks<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, kBwdSmem);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_chain_mats<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, kChainSmem);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_chain_mats<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, kChainSmem);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_diag_inv<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, diag_inv_smem<double>());
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_diag_inv<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, diag_inv_smem<float>());
  return e;
}

int num_sms();
// persistent solve grids: 3 CTAs per SM (the kernels' launch bounds)
static int solve_grid(int ntasks) { return ntasks < 3 * num_sms() ? ntasks : 3 * num_sms(); }

template <class TL>
void launch_diag_inv(const int *blocks, int nblocks, const DevPlan &P, const TL *Lx, TL *Inv, cudaStream_t st) {
  if (nblocks > 0) k_diag_inv<TL><<<nblocks, kInvThreads, diag_inv_smem<TL>(), st>>>(blocks, P, Lx, Inv);
}
template <class TL>
void launch_chain_mats(const int2 *tasks, int ntasks, const DevPlan &P, const TL *Lx, const TL *Inv, TL *Mch, TL *Gch,
                       cudaStream_t st) {
  if (ntasks > 0) k_chain_mats<TL><<<ntasks, 256, kChainSmem, st>>>(tasks, P, Lx, Inv, Mch, Gch);
}
template <class TL>
void launch_fwd_blocks(const int4 *tasks, int ntasks, int *ticket, const DevPlan &P, const TL *Lx, const TL *Inv,
                       const TL *Mch, double *y, double *T, int *flags, unsigned long long *hand, int epoch, int *done,
                       unsigned long long *status, cudaStream_t st) {
  if (ntasks > 0)
    k_fwd_blocks<TL><<<solve_grid(ntasks), 256, 0, st>>>(tasks, ntasks, ticket, P, Lx, Inv, Mch, y, T, flags, hand,
                                                         epoch, done, status);
}
template <class TL>
void launch_bwd_blocks(const int4 *tasks, int ntasks, int *ticket, const DevPlan &P, const TL *Lx, const TL *Inv,
                       const TL *Gch, const double *Dpiv, double *y, int *flags, unsigned long long *hand, int epoch,
                       unsigned long long *status, cudaStream_t st) {
  if (ntasks > 0)
    k_bwd_blocks<TL><<<solve_grid(ntasks), 256, kBwdSmem, st>>>(tasks, ntasks, ticket, P, Lx, Inv, Gch, Dpiv, y, flags,
                                                                 hand, epoch, status);
}
template void launch_diag_inv<double>(const int *, int, const DevPlan &, const double *, double *, cudaStream_t);
template void launch_diag_inv<float>(const int *, int, const DevPlan &, const float *, float *, cudaStream_t);
template void launch_chain_mats<double>(const int2 *, int, const DevPlan &, const double *, const double *, double *,
                                        double *, cudaStream_t);
template void launch_chain_mats<float>(const int2 *, int, const DevPlan &, const float *, const float *, float *,
                                       float *, cudaStream_t);
template void launch_fwd_blocks<double>(const int4 *, int, int *, const DevPlan &, const double *, const double *,
                                        const double *, double *, double *, int *, unsigned long long *, int, int *,
                                        unsigned long long *, cudaStream_t);
template void launch_fwd_blocks<float>(const int4 *, int, int *, const DevPlan &, const float *, const float *,
                                       const float *, double *, double *, int *, unsigned long long *, int, int *,
                                       unsigned long long *, cudaStream_t);
template void launch_bwd_blocks<double>(const int4 *, int, int *, const DevPlan &, const double *, const double *,
                                        const double *, const double *, double *, int *, unsigned long long *, int,
                                        unsigned long long *, cudaStream_t);
template void launch_bwd_blocks<float>(const int4 *, int, int *, const DevPlan &, const float *, const float *,
                                       const float *, const double *, double *, int *, unsigned long long *, int,
                                       unsigned long long *, cudaStream_t);

}  // namespace amp
