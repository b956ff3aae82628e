// Supernodal triangular solves with several right-hand sides at once (sparse.mjs solveNumericMulti :1261-1310,
// ldlt.mjs solveMany :595-643): the same task lists and ticket order as the one-vector sweeps (solve.cu), every task
// moving a slice of up to 16 of the q <= 64 vectors.
//
// Vectors are interleaved: entry i of vector k sits at y[i q + k] (and likewise the front vectors V and the pass-up
// buffers T), so a row of the solution is q contiguous doubles and the gathers through the extend-add maps and the
// row lists move whole rows.
//
// Vector slices of 16 (ns = ceil(q / 16)), each with its own ready flags (flags[slice * nflags + block]) and done
// counters (done[slice * nsuper + s]): the host expands the block tasks of supernodes with several pivot blocks into
// ns consecutive tasks, one per slice (int4 .w = the slice), so the slices' dependency chains run on different CTAs;
// a task with .w = -1 (a supernode of few pivot blocks) moves all vectors at once (below; compiled into the sweeps of
// the WIDE instantiation only, which the host launches for plans made mostly of such supernodes: the all-vector path
// holds more registers, and in the same kernel the sliced tasks would spill). The expanded order keeps every wait on a
// task with a smaller ticket, and a task never computes on absent vectors. The small supernodes (kind 2, one warp
// each, not expanded) solve all q vectors and count/release every slice.
//
// A task is a small GEMM on the FP64 tensor cores (mma.sync m16n8k16): out (64 rows x 16 vectors) = sum over a
// reduction index of A (64 x 32 chunk, FP32 factors widened on the shared-memory store) times B (32 x 16), 8 warps
// as 4 (16-row blocks) x 2 (16-wide halves of the chunk), the halves summed through shared memory at the end.
// Forward: A = L[block rows, pivot columns so far], B = y[those columns]. Backward: A = the block's columns of L over
// the rows below the block (transposed on load), B = x[those rows]. Then the 64 x 64 inverse of the diagonal block,
// prefetched into shared memory by cp.async when the task starts, is applied the same way.
//
// Backward order: the rows below the supernode are summed from the last chunk down, each chunk after the flags of the
// ancestor blocks that hold its rows (rowBlk), so a task works while its ancestors are still being solved (the
// highest ancestors, which hold the last rows, finish first); then the supernode's own later blocks, each after its
// flag.
#include <cuda_runtime.h>

#include <cstdint>

#include "../host/plan.hpp"
#include "devplan.cuh"
#include "solve_small.cuh"
#include "sync.cuh"

namespace amp {

constexpr int kMB = 64;              // rows of a block task
constexpr int kKC = 32;              // reduction chunk
constexpr int kQS = 16;              // vectors per slice (one slice per task)
constexpr int kMQ = 64;              // vectors per pass (the host splits larger sets)
constexpr int kLdKM = kMB + 4;       // A stored [k][m] (m contiguous): 68 doubles, == 4 mod 16 (conflict-free fragments)
constexpr int kLdMK = kKC + 4;       // A chunk stored [m][k]: 36
constexpr int kLdX = kMB + 4;        // inverse block stored [k][m] or [m][k], 64 x 64: 68
constexpr int kLdB = kQS + 4;        // B stored [k][n]: 20
constexpr int kMultiThreads = 256;
constexpr int kMultiCtas = 3;      // resident CTAs per SM of the persistent sweeps (registers capped at 80)
constexpr int kAElems = kMB * kLdMK;  // >= kKC * kLdKM; also the halves' reduction buffer (64 x 17)
static_assert(kAElems >= kKC * kLdKM && kAElems >= kMB * (kQS + 1), "A tile buffer");
template <class TL>
constexpr int multi_smem() {
  const int own = (kAElems + 2 * kMB * kLdB) * (int)sizeof(double) + kMB * kLdX * (int)sizeof(TL);
  const int small = kSolveGroup * 32 * kMQ * (int)sizeof(double);  // kind 2 tasks: 32 x 64 front vectors per warp
  const int wide = (2 * 32 + kMB) * 66 * (int)sizeof(double);        // all-vector tasks (kWideSmem)
  const int m1 = own > small ? own : small;
  return m1 > wide ? m1 : wide;
}

__device__ __forceinline__ void dmma16816(double (&c)[4], const double (&a)[8], const double (&b)[4]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7,%8,%9,%10,%11}, "
      "{%12,%13,%14,%15}, {%0,%1,%2,%3};\n"
      : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
      : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(a[4]), "d"(a[5]), "d"(a[6]), "d"(a[7]), "d"(b[0]), "d"(b[1]),
        "d"(b[2]), "d"(b[3]));
}

// Fragment layouts of the m16n8k16 FP64 MMA (g = lane / 4, t = lane % 4): A (m = g + 8 (v & 1), k = t + 4 (v >> 1)),
// B (n = g, k = t + 4 v), C (m = g + 8 (v >> 1), n = 2 t + (v & 1)).
// c[nb] += A[16 mw .. +16, k0 .. k0 + 16) B[k0 .. k0 + 16, 8 nb .. 8 nb + 8) for both n halves; A element (m, k) at
// A[k * lda + m] (KM) or A[m * lda + k] (MK), B element (k, n) at B[k * kLdB + n].
template <bool KM, class TA>
__device__ __forceinline__ void mma_k16(const TA *__restrict__ A, int lda, const double *__restrict__ B, int k0,
                                        int mw, int lane, double (&c)[2][4]) {
  const int g = lane >> 2, t = lane & 3;
  double a[8];
#pragma unroll
  for (int v = 0; v < 8; v++) {
    const int m = 16 * mw + g + 8 * (v & 1), k = k0 + t + 4 * (v >> 1);
    a[v] = (double)(KM ? A[k * lda + m] : A[m * lda + k]);
  }
#pragma unroll
  for (int nb = 0; nb < 2; nb++) {
    double b[4];
#pragma unroll
    for (int v = 0; v < 4; v++) b[v] = B[(k0 + t + 4 * v) * kLdB + 8 * nb + g];
    dmma16816(c[nb], a, b);
  }
}

// The two halves of the reduction index: warps 4-7 add their partial tile into warps 0-3's (red: 64 x 17 doubles).
// On return warps 0-3 hold the sum; red is free after the caller's next barrier.
__device__ __forceinline__ void halves_sum(double (&c)[2][4], double *red, int warp, int lane) {
  const int mw = warp & 3, g = lane >> 2, t = lane & 3;
  if (warp >= 4) {
#pragma unroll
    for (int nb = 0; nb < 2; nb++)
#pragma unroll
      for (int v = 0; v < 4; v++) red[(16 * mw + g + 8 * (v >> 1)) * (kQS + 1) + 8 * nb + 2 * t + (v & 1)] = c[nb][v];
  }
  __syncthreads();
  if (warp < 4) {
#pragma unroll
    for (int nb = 0; nb < 2; nb++)
#pragma unroll
      for (int v = 0; v < 4; v++) c[nb][v] += red[(16 * mw + g + 8 * (v >> 1)) * (kQS + 1) + 8 * nb + 2 * t + (v & 1)];
  }
}

// row / vector of accumulator element (nb, v) of this lane (warps 0-3)
__device__ __forceinline__ int acc_row(int warp, int lane, int v) { return 16 * (warp & 3) + (lane >> 2) + 8 * (v >> 1); }
__device__ __forceinline__ int acc_vec(int lane, int nb, int v) { return 8 * nb + 2 * (lane & 3) + (v & 1); }

__device__ __forceinline__ void cp_async_el(void *smem, const void *gmem, int bytes, bool valid) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  const int n = valid ? bytes : 0;  // zero-fill when out of range
  if (bytes == 8)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(sa), "l"(gmem), "r"(n) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(sa), "l"(gmem), "r"(n) : "memory");
}
__device__ __forceinline__ void cp_async_all() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

// persistent ticket loop shared by both sweeps
template <class Run>
__device__ __forceinline__ void ticket_loop(int *ticket, int ntasks, Run &&run) {
  __shared__ int tk;
  for (;;) {
    if (threadIdx.x == 0) tk = atomicAdd(ticket, 1);
    __syncthreads();
    const int mine = tk;
    __syncthreads();
    if (mine >= ntasks || !run(mine)) return;
  }
}

// This task's rows [r0, r0 + rows) of the front vector v_s = [y(f .. f + nc); 0] + the children's pass-up vectors,
// vectors [vb, vb + qs) of q, into Rs (row r at Rs[r LDR], QW >= qs columns; zero outside): the pivot rows from y,
// then each child's entries that map into these rows, in the reference's child order. Up to kGatherCh children at a
// time, one per thread: the thread locates the child's entries for these rows (the map is increasing, so they form
// one range) and waits for the child's pass-up vectors of slices [sl0, sl0 + nsl), so the searches and the waits of
// all children overlap and every task of the supernode gathers its own rows in parallel. false: a wait gave up.
constexpr int kGatherCh = 64;
template <int QW, int LDR>
__device__ bool gather_front_rows(const DevPlan &P, int s, int r0, int rows, const double *__restrict__ y,
                                  const double *__restrict__ T, int *done, int sl0, int nsl, int q, int vb, int qs,
                                  unsigned long long *status, double *Rs) {
  __shared__ int2 chA[kGatherCh];
  __shared__ int64_t chMap[kGatherCh], chT[kGatherCh];
  const int tid = threadIdx.x, f = P.snF[s], nc = P.snNc[s];
  for (int e = tid; e < kMB * QW; e += blockDim.x) {
    const int row = e / QW, k = e % QW;
    Rs[row * LDR + k] = (row < rows && k < qs && r0 + row < nc) ? y[(int64_t)(f + r0 + row) * q + vb + k] : 0.0;
  }
  const int q0 = P.chPtr[s], q1 = P.chPtr[s + 1];
  for (int qb = q0; qb < q1; qb += kGatherCh) {
    const int nq = min(kGatherCh, q1 - qb);
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
      const int need = (muc + kMB - 1) / kMB;
      for (int sl = sl0; sl < sl0 + nsl && ok; sl++) ok = wait_count(done + (int64_t)sl * P.nsuper + c, need, status, s, P.spin);
    }
    if (!__syncthreads_and(ok)) return false;  // block-uniform
    for (int qq = 0; qq < nq; qq++) {
      const int *map = P.eaMap + chMap[qq];
      const double *tc = T + chT[qq] * q + vb;
      const int a0 = chA[qq].x, na = chA[qq].y - a0;
      for (int e = tid; e < na * QW; e += blockDim.x) {
        const int a = a0 + e / QW, k = e % QW;
        if (k < qs) Rs[(map[a] - r0) * LDR + k] += __ldcg(tc + (int64_t)a * q + k);
      }
      __syncthreads();
    }
  }
  if (q0 == q1) __syncthreads();
  return true;
}

// ---- tasks of supernodes with few pivot blocks: all q vectors at once on the CUDA cores ----------------------------
// A task of a supernode with at most two pivot blocks (list entry .w = -1) moves all q <= 64 vectors together: out
// (64 rows x 64 vectors) = sum of A (64 x 32 L chunk) times B (32 x 64 vector chunk), both in shared memory, each
// thread accumulating a 4 x 4 register tile in FP64. Such a task has no chain worth splitting, and one pass over
// its L tile serves every vector. It waits for every slice of what another supernode provides (children's counts,
// the parent's flag) and releases every slice of its own flags and counts.
constexpr int kWKC = 32;  // reduction chunk
constexpr int kWLd = 66;  // shared tile row stride in doubles (even: 16-byte aligned double2 reads)
constexpr int kWideSmem = (2 * kWKC + kMB) * kWLd * (int)sizeof(double);
// acc[i][j] += sum over kk < kc of A[kk][4 ty + i] B[kk][4 tx + j]
__device__ __forceinline__ void mm_tile_w(const double *__restrict__ A, const double *__restrict__ B, int kc, int ty,
                                          int tx, double (&acc)[4][4]) {
#pragma unroll 4
  for (int kk = 0; kk < kc; kk++) {
    const double2 a0 = *reinterpret_cast<const double2 *>(A + kk * kWLd + 4 * ty);
    const double2 a1 = *reinterpret_cast<const double2 *>(A + kk * kWLd + 4 * ty + 2);
    const double2 b0 = *reinterpret_cast<const double2 *>(B + kk * kWLd + 4 * tx);
    const double2 b1 = *reinterpret_cast<const double2 *>(B + kk * kWLd + 4 * tx + 2);
    const double a[4] = {a0.x, a0.y, a1.x, a1.y}, b[4] = {b0.x, b0.y, b1.x, b1.y};
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
      for (int j = 0; j < 4; j++) acc[i][j] = fma(a[i], b[j], acc[i][j]);
  }
}

// forward: as the sliced task (diagonal y[block] = X (v[block] - L[block, 0:blk 64] y), below T[block] = v[block] -
// L[block, 0:nc] y), every vector
template <class TL>
__device__ __forceinline__ bool fwd_wide_task(const int4 t, const DevPlan &P, const TL *__restrict__ Lx, const TL *__restrict__ Inv,
                              double *__restrict__ y, double *__restrict__ T, int *flags,
                              int nflags, int epoch, int *done, int q, int ns, unsigned long long *status,
                              double *msm, int &waitOk) {
  double *As = msm, *Bs = msm + kWKC * kWLd, *Rs = msm + 2 * kWKC * kWLd;
  const int tid = threadIdx.x, ty = tid >> 4, tx = tid & 15;
  const int s = t.x, blk = t.y, below = t.z;
  const int f = P.snF[s], nc = P.snNc[s], m = P.snM[s], mu = m - nc;
  const TL *Lp = Lx + P.snLxp[s];
  const int r0 = below ? nc + blk * kMB : blk * kMB;
  const int rows = below ? min(kMB, mu - blk * kMB) : min(kMB, nc - blk * kMB);
  const int ncols = below ? nc : blk * kMB;
  int *myflags = flags + P.blkOff[s];  // the slice-0 set: this supernode releases every slice at once
  // this task's rows of v_s, every vector, into Rs (every slice of each child done)
  if (!gather_front_rows<kMQ, kWLd>(P, s, r0, rows, y, T, done, 0, ns, q, 0, q, status, Rs)) return false;
  double acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int j = 0; j < 4; j++) acc[i][j] = 0.0;
  // L tile of a chunk: As[c][row] = L(r0 + row, cb + c); thread elements e = tid + 256 u: row = e & 63, c = e >> 6
  TL lr[8];
  auto loadL = [&](int cb) {
#pragma unroll
    for (int u = 0; u < 8; u++) {
      const int e = tid + kMultiThreads * u, row = e & (kMB - 1), c = e >> 6;
      lr[u] = (row < rows && cb + c < ncols) ? Lp[(int64_t)(cb + c) * m + r0 + row] : (TL)0;
    }
  };
  const int nch = (ncols + kWKC - 1) / kWKC;
  if (nch > 0) loadL(0);
  for (int ch = 0; ch < nch; ch++) {
    const int cb = ch * kWKC, cw = min(kWKC, ncols - cb);
    if ((cb & (kMB - 1)) == 0) {  // first chunk of a pivot block: its y values final?
      if (tid == 0) waitOk = wait_flag(myflags + cb / kMB, epoch, status, s, P.spin);
      __syncthreads();
      if (!waitOk) return false;
    }
    for (int e = tid; e < kWKC * kMQ; e += kMultiThreads) {
      const int c = e >> 6, k = e & (kMQ - 1);
      Bs[c * kWLd + k] = (c < cw && k < q) ? __ldcg(y + (int64_t)(f + cb + c) * q + k) : 0.0;
    }
#pragma unroll
    for (int u = 0; u < 8; u++) {
      const int e = tid + kMultiThreads * u;
      As[(e >> 6) * kWLd + (e & (kMB - 1))] = (double)lr[u];
    }
    __syncthreads();
    if (ch + 1 < nch) loadL(cb + kWKC);
    mm_tile_w(As, Bs, cw, ty, tx, acc);
    __syncthreads();
  }
  // R = v[block] - acc (the task's rows of v in Rs)
  if (below) {
    double *to = T + (P.snTOff[s] + (int64_t)blk * kMB) * q;
#pragma unroll
    for (int i = 0; i < 4; i++) {
      const int row = 4 * ty + i;
      if (row >= rows) continue;
#pragma unroll
      for (int j = 0; j < 4; j++) {
        const int k = 4 * tx + j;
        if (k < q) to[(int64_t)row * q + k] = Rs[row * kWLd + k] - acc[i][j];
      }
    }
    __syncthreads();
    if (tid < ns) red_release_add(done + (int64_t)tid * P.nsuper + s, 1);  // one count per vector slice
    return true;
  }
#pragma unroll
  for (int i = 0; i < 4; i++) {
    const int row = 4 * ty + i;
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const int k = 4 * tx + j;
      Rs[row * kWLd + k] = (row < rows && k < q) ? Rs[row * kWLd + k] - acc[i][j] : 0.0;
      acc[i][j] = 0.0;
    }
  }
  // y[block] = X R, X = L_kk^-1 (rows x rows, column-major): As[jj][i] = X(i, jb + jj)
  const TL *X = Inv + P.invOff[P.blkOff[s] + blk];
  for (int jb = 0; jb < rows; jb += kWKC) {
    const int jw = min(kWKC, rows - jb);
    __syncthreads();
    for (int e = tid; e < kWKC * kMB; e += kMultiThreads) {
      const int i = e & (kMB - 1), jj = e >> 6;
      As[jj * kWLd + i] = (i < rows && jj < jw) ? (double)X[(int64_t)(jb + jj) * rows + i] : 0.0;
    }
    __syncthreads();
    mm_tile_w(As, Rs + jb * kWLd, jw, ty, tx, acc);
  }
#pragma unroll
  for (int i = 0; i < 4; i++) {
    const int row = 4 * ty + i;
    if (row >= rows) continue;
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const int k = 4 * tx + j;
      if (k < q) y[(int64_t)(f + r0 + row) * q + k] = acc[i][j];
    }
  }
  __syncthreads();
  if (tid < ns) st_release(flags + (int64_t)tid * nflags + P.blkOff[s] + blk, epoch);  // every vector slice
  return true;
}

// backward: as the sliced task, every vector (the rows below after the parent's every slice is final)
template <class TL>
__device__ __forceinline__ bool bwd_wide_task(const int4 t, const DevPlan &P, const TL *__restrict__ Lx, const TL *__restrict__ Inv,
                              const double *__restrict__ Dpiv, double *__restrict__ y, int *flags, int nflags,
                              int epoch, int q, int ns, unsigned long long *status, double *msm, int &waitOk) {
  double *As = msm, *Bs = msm + kWKC * kWLd, *Rs = msm + 2 * kWKC * kWLd;
  const int tid = threadIdx.x, ty = tid >> 4, tx = tid & 15;
  const int s = t.x, blk = t.y;
  const int f = P.snF[s], nc = P.snNc[s], m = P.snM[s];
  const TL *Lp = Lx + P.snLxp[s];
  const int *rowsOf = P.Si + P.Sp[s];
  const int c0 = blk * kMB, w = min(kMB, nc - c0), nb = (nc + kMB - 1) / kMB;
  int *myflags = flags + P.blkOff[s];  // the slice-0 set: this supernode releases every slice at once
  const int par = P.snParent[s];
  if (par >= 0) {  // the parent's every vector slice final
    if (tid == 0) {
      waitOk = 1;
      for (int sl = 0; sl < ns && waitOk; sl++)
        waitOk = wait_flag(flags + (int64_t)sl * nflags + P.blkOff[par], epoch, status, s, P.spin);
    }
    __syncthreads();
    if (!waitOk) return false;
  }
  double acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int j = 0; j < 4; j++) acc[i][j] = 0.0;
  // chunks: ancestors rows [nc, m) in kWKC steps, then pivot blocks nb - 1 .. blk + 1 (two chunks each)
  const int nanc = (m - nc + kWKC - 1) / kWKC;
  const int npiv = (nb - 1 - blk) * (kMB / kWKC);
  const int nch = nanc + npiv;
  // chunk ch -> first row and row count
  auto chunk = [&](int ch, int &rb, int &rw) {
    if (ch < nanc) {
      rb = nc + ch * kWKC;
      rw = min(kWKC, m - rb);
    } else {
      const int p = ch - nanc, pb = nb - 1 - p / 2;  // pivot block, from the last down
      rb = pb * kMB + (p & 1) * kWKC;
      rw = max(0, min(kWKC, nc - rb));
    }
  };
  // L tile: As[rr][c] = L(rb + rr, c0 + c); elements e = tid + 256 u: rr = e & 31, c = e >> 5
  TL lr[8];
  auto loadL = [&](int rb, int rw) {
#pragma unroll
    for (int u = 0; u < 8; u++) {
      const int e = tid + kMultiThreads * u, rr = e & (kWKC - 1), c = e >> 5;
      lr[u] = (rr < rw && c < w) ? Lp[(int64_t)(c0 + c) * m + rb + rr] : (TL)0;
    }
  };
  int rb = 0, rw = 0;
  if (nch > 0) {
    chunk(0, rb, rw);
    loadL(rb, rw);
  }
  for (int ch = 0; ch < nch; ch++) {
    const bool anc = ch < nanc;
    if (!anc && ((ch - nanc) & 1) == 0) {  // first chunk of a pivot block: its x values final?
      if (tid == 0) waitOk = wait_flag(myflags + rb / kMB, epoch, status, s, P.spin);
      __syncthreads();
      if (!waitOk) return false;
    }
    for (int e = tid; e < kWKC * kMQ; e += kMultiThreads) {
      const int rr = e >> 6, k = e & (kMQ - 1);
      double v = 0.0;
      if (rr < rw && k < q) {
        const int gi = anc ? rowsOf[rb + rr] : f + rb + rr;
        v = __ldcg(y + (int64_t)gi * q + k);
      }
      Bs[rr * kWLd + k] = v;
    }
#pragma unroll
    for (int u = 0; u < 8; u++) {
      const int e = tid + kMultiThreads * u;
      As[(e & (kWKC - 1)) * kWLd + (e >> 5)] = (double)lr[u];
    }
    __syncthreads();
    const int cw = rw;
    if (ch + 1 < nch) {
      chunk(ch + 1, rb, rw);
      loadL(rb, rw);
    }
    mm_tile_w(As, Bs, cw, ty, tx, acc);
    __syncthreads();
  }
  // R = y[block] (/ D) - acc
#pragma unroll
  for (int i = 0; i < 4; i++) {
    const int c = 4 * ty + i;
    const double d = (Dpiv && c < w) ? Dpiv[f + c0 + c] : 1.0;
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const int k = 4 * tx + j;
      double v = 0.0;
      if (c < w && k < q) {
        const double yv = y[(int64_t)(f + c0 + c) * q + k];
        v = (Dpiv ? yv / d : yv) - acc[i][j];  // LDL^T: y /= D before the backward sweep (ldlt.mjs:629)
      }
      Rs[c * kWLd + k] = v;
      acc[i][j] = 0.0;
    }
  }
  // x[block] = X^T R: As[jj][i] = X(jb + jj, i) = Inv[i w + jb + jj]
  const TL *X = Inv + P.invOff[P.blkOff[s] + blk];
  for (int jb = 0; jb < w; jb += kWKC) {
    const int jw = min(kWKC, w - jb);
    __syncthreads();
    for (int e = tid; e < kWKC * kMB; e += kMultiThreads) {
      const int jj = e & (kWKC - 1), i = e >> 5;
      As[jj * kWLd + i] = (i < w && jj < jw) ? (double)X[(int64_t)i * w + jb + jj] : 0.0;
    }
    __syncthreads();
    mm_tile_w(As, Rs + jb * kWLd, jw, ty, tx, acc);
  }
#pragma unroll
  for (int i = 0; i < 4; i++) {
    const int c = 4 * ty + i;
    if (c >= w) continue;
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const int k = 4 * tx + j;
      if (k < q) y[(int64_t)(f + c0 + c) * q + k] = acc[i][j];
    }
  }
  __syncthreads();
  if (tid < ns) st_release(flags + (int64_t)tid * nflags + P.blkOff[s] + blk, epoch);  // every vector slice
  return true;
}

// ---- forward ------------------------------------------------------------------------------------------------------
// task (s, blk, below) of slice sl: as k_fwd_blocks. Diagonal: y[block] = X (v[block] - L[block, 0:blk 64] y[0:blk 64]);
// below: T[block] = v[block] - L[block, 0:nc] y[0:nc], where v[block] is the task's rows of the front vector, gathered
// by the task itself (gather_front_rows). With the chain matrices of a Cholesky factor (Mch, see k_chain_mats), a
// diagonal task b >= 1 forms W = X (v[block] - L[block, 0:(b-1) 64] y) before its last wait and then, after block
// b - 1's flag, y[block] = W - M_b y[block b - 1]: one 64 x 64 product per chain step instead of the block's last
// chunk, the reduction and the inverse product.
template <class TL, bool WIDE>
__global__ void __launch_bounds__(kMultiThreads, kMultiCtas) k_fwd_multi(const int4 *__restrict__ tasks, int ntasks, int ns,
                                                                int *__restrict__ ticket, DevPlan P,
                                                                const TL *__restrict__ Lx, const TL *__restrict__ Inv,
                                                                const TL *__restrict__ Mch, double *__restrict__ y,
                                                                double *__restrict__ T, int *__restrict__ flags,
                                                                int nflags, int epoch, int *__restrict__ done, int q,
                                                                unsigned long long *status) {
  extern __shared__ double msm[];
  double *As = msm, *Bs = As + kAElems, *Rs = Bs + kMB * kLdB;
  TL *Xs = reinterpret_cast<TL *>(Rs + kMB * kLdB);
  __shared__ int waitOk;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, mw = warp & 3, kh = warp >> 2;
  auto bail = [] {  // a wait gave up: drain this thread's copies into shared memory before the CTA leaves
    cp_async_all();
    return false;
  };
  // one block task for vector slice sl
  auto run_slice = [&](const int4 t, const int sl) -> bool {
    const int s = t.x, blk = t.y, below = t.z;
    const int f = P.snF[s], nc = P.snNc[s], m = P.snM[s], mu = m - nc;
    const int vb = sl * kQS, qs = min(kQS, q - vb);
    const TL *Lp = Lx + P.snLxp[s];
    const int r0 = below ? nc + blk * kMB : blk * kMB;
    const int rows = below ? min(kMB, mu - blk * kMB) : min(kMB, nc - blk * kMB);
    const bool chain = Mch != nullptr && !below && blk > 0;  // block b - 1 enters through M_b after the last wait
    const int ncols = below ? nc : (chain ? blk - 1 : blk) * kMB;
    int *myflags = flags + (int64_t)sl * nflags + P.blkOff[s];
    int *mydone = done + (int64_t)sl * P.nsuper;
    if (!below) {  // the inverse of the diagonal block, [k][m], arrives while the task sums
      const TL *X = Inv + P.invOff[P.blkOff[s] + blk];
      for (int e = tid; e < kMB * kMB; e += kMultiThreads) {
        const int i = e & (kMB - 1), k = e >> 6;
        const bool ok = i < rows && k < rows;
        cp_async_el(Xs + k * kLdX + i, ok ? X + (int64_t)k * rows + i : X, (int)sizeof(TL), ok);
      }
      asm volatile("cp.async.commit_group;\n" ::: "memory");
    }
    // this task's rows of v_s (this slice) into Rs, gathered by every task of the supernode in parallel
    if (!gather_front_rows<kQS, kLdB>(P, s, r0, rows, y, T, done, sl, 1, q, vb, qs, status, Rs)) return bail();
    double c[2][4];
#pragma unroll
    for (int nb = 0; nb < 2; nb++)
#pragma unroll
      for (int v = 0; v < 4; v++) c[nb][v] = 0.0;
    // L chunk, [k][m]: As[cc][row] = L(r0 + row, cb + cc); thread elements e = tid + 256 u: row = e & 63, cc = e >> 6
    TL lr[8];
    auto loadL = [&](int cb) {
#pragma unroll
      for (int u = 0; u < 8; u++) {
        const int e = tid + kMultiThreads * u, row = e & (kMB - 1), cc = e >> 6;
        lr[u] = (row < rows && cb + cc < ncols) ? Lp[(int64_t)(cb + cc) * m + r0 + row] : (TL)0;
      }
    };
    const int nch = (ncols + kKC - 1) / kKC;
    if (nch > 0) loadL(0);
    for (int ch = 0; ch < nch; ch++) {
      const int cb = ch * kKC, cw = min(kKC, ncols - cb);
      const double *Bc = Bs + (cb & (kMB - 1)) * kLdB;  // this chunk's rows of the block's y values
      if ((cb & (kMB - 1)) == 0) {  // first chunk of a pivot block: its y values final? Then all 64 rows at once
        if (tid == 0) waitOk = wait_flag(myflags + cb / kMB, epoch, status, s, P.spin);
        __syncthreads();
        if (!waitOk) return bail();
        for (int e = tid; e < kMB * kQS; e += kMultiThreads) {
          const int k = e >> 4, n = e & (kQS - 1);
          Bs[k * kLdB + n] = (cb + k < ncols && n < qs) ? __ldcg(y + (int64_t)(f + cb + k) * q + vb + n) : 0.0;
        }
      }
#pragma unroll
      for (int u = 0; u < 8; u++) {
        const int e = tid + kMultiThreads * u;
        As[(e >> 6) * kLdKM + (e & (kMB - 1))] = (double)lr[u];
      }
      __syncthreads();
      if (ch + 1 < nch) loadL(cb + kKC);
      if (16 * kh < cw) mma_k16<true>(As, kLdKM, Bc, 16 * kh, mw, lane, c);
      __syncthreads();
    }
    halves_sum(c, As, warp, lane);
    // R = v[block] - acc (the task's rows of v in Rs)
    if (below) {
      if (warp < 4) {
        double *to = T + (P.snTOff[s] + (int64_t)blk * kMB) * q + vb;
#pragma unroll
        for (int nb = 0; nb < 2; nb++)
#pragma unroll
          for (int v = 0; v < 4; v++) {
            const int row = acc_row(warp, lane, v), n = acc_vec(lane, nb, v);
            if (row < rows && n < qs) to[(int64_t)row * q + n] = Rs[row * kLdB + n] - c[nb][v];
          }
      }
      __syncthreads();
      if (tid == 0) red_release_add(mydone + s, 1);
      return true;
    }
    if (warp < 4) {
#pragma unroll
      for (int nb = 0; nb < 2; nb++)
#pragma unroll
        for (int v = 0; v < 4; v++) {
          const int row = acc_row(warp, lane, v), n = acc_vec(lane, nb, v);
          Rs[row * kLdB + n] = (row < rows && n < qs) ? Rs[row * kLdB + n] - c[nb][v] : 0.0;
        }
    }
#pragma unroll
    for (int nb = 0; nb < 2; nb++)
#pragma unroll
      for (int v = 0; v < 4; v++) c[nb][v] = 0.0;
    cp_async_all();
    __syncthreads();
    // y[block] = X R: k = 0 .. 63 of X as four k16 steps, two per warp half
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const int k0 = 32 * h + 16 * kh;
      if (k0 < rows) mma_k16<true>(Xs, kLdX, Rs, k0, mw, lane, c);
    }
    halves_sum(c, As, warp, lane);
    if (chain) {
      // W stays in Rs (its R was consumed by the product); M_b arrives in Xs while the task waits for block b - 1
      if (warp < 4) {
#pragma unroll
        for (int nb = 0; nb < 2; nb++)
#pragma unroll
          for (int v = 0; v < 4; v++) {
            const int row = acc_row(warp, lane, v), n = acc_vec(lane, nb, v);
            Rs[row * kLdB + n] = c[nb][v];
          }
      }
#pragma unroll
      for (int nb = 0; nb < 2; nb++)
#pragma unroll
        for (int v = 0; v < 4; v++) c[nb][v] = 0.0;
      __syncthreads();  // every warp is done with X in Xs
      {  // M_b (rows x 64, column-major), [k][m] like X
        const TL *M = Mch + (int64_t)(P.blkOff[s] - s + blk - 1) * kMB * kMB;
        for (int e = tid; e < kMB * kMB; e += kMultiThreads) {
          const int i = e & (kMB - 1), k = e >> 6;
          const bool ok = i < rows;
          cp_async_el(Xs + k * kLdX + i, ok ? M + (int64_t)k * kMB + i : M, (int)sizeof(TL), ok);
        }
        asm volatile("cp.async.commit_group;\n" ::: "memory");
      }
      if (tid == 0) waitOk = wait_flag(myflags + blk - 1, epoch, status, s, P.spin);
      __syncthreads();
      if (!waitOk) return bail();
      const int cp = (blk - 1) * kMB;  // block b - 1: 64 columns (not the last block)
      for (int e = tid; e < kMB * kQS; e += kMultiThreads) {
        const int k = e >> 4, n = e & (kQS - 1);
        Bs[k * kLdB + n] = n < qs ? __ldcg(y + (int64_t)(f + cp + k) * q + vb + n) : 0.0;
      }
      cp_async_all();
      __syncthreads();
#pragma unroll
      for (int h = 0; h < 2; h++) mma_k16<true>(Xs, kLdX, Bs, 32 * h + 16 * kh, mw, lane, c);
      halves_sum(c, As, warp, lane);
      if (warp < 4) {
#pragma unroll
        for (int nb = 0; nb < 2; nb++)
#pragma unroll
          for (int v = 0; v < 4; v++) {
            const int row = acc_row(warp, lane, v), n = acc_vec(lane, nb, v);
            if (row < rows && n < qs) y[(int64_t)(f + r0 + row) * q + vb + n] = Rs[row * kLdB + n] - c[nb][v];
          }
      }
      __syncthreads();
      if (tid == 0) st_release(myflags + blk, epoch);
      return true;
    }
    if (warp < 4) {
#pragma unroll
      for (int nb = 0; nb < 2; nb++)
#pragma unroll
        for (int v = 0; v < 4; v++) {
          const int row = acc_row(warp, lane, v), n = acc_vec(lane, nb, v);
          if (row < rows && n < qs) y[(int64_t)(f + r0 + row) * q + vb + n] = c[nb][v];
        }
    }
    __syncthreads();
    if (tid == 0) st_release(myflags + blk, epoch);
    return true;
  };
  auto run = [&](const int tkv) -> bool {
    const int4 t = tasks[tkv];
    if (t.z == 2) {  // up to kSolveGroup supernodes with m <= 32, one warp each, all q vectors
      if (tid == 0) waitOk = 1;
      __syncthreads();
      if (warp < t.y && !small_fwd_warp_multi<TL>(P.solveSmall[t.x + warp], P, Lx, y, T, done, q, ns, status,
                                                  msm + 32 * kMQ * warp))
        waitOk = 0;
      __syncthreads();
      return waitOk != 0;
    }
    if constexpr (WIDE) {
      if (t.w < 0) return fwd_wide_task<TL>(t, P, Lx, Inv, y, T, flags, nflags, epoch, done, q, ns, status, msm, waitOk);
    }
    return run_slice(t, t.w);
  };
  ticket_loop(ticket, ntasks, run);
}

// ---- backward -----------------------------------------------------------------------------------------------------
// task (s, blk) of slice sl: x[block] = X^T (y[block] (/ D for LDL^T) - L[rows below the block, block columns]^T
// x[those rows]). With the chain matrices of a Cholesky factor (Gch), block b + 1 is left out of the sum and enters
// after its flag as x[block] = W - G_b^T x[block b + 1], W = X^T (y[block] - the other rows' terms).
template <class TL, bool WIDE>
__global__ void __launch_bounds__(kMultiThreads, kMultiCtas) k_bwd_multi(const int4 *__restrict__ tasks, int ntasks, int ns,
                                                                int *__restrict__ ticket, DevPlan P,
                                                                const TL *__restrict__ Lx, const TL *__restrict__ Inv,
                                                                const TL *__restrict__ Gch,
                                                                const double *__restrict__ Dpiv,
                                                                double *__restrict__ y, int *__restrict__ flags,
                                                                int nflags, int epoch, int q,
                                                                unsigned long long *status) {
  extern __shared__ double msm[];
  double *As = msm, *Bs = As + kAElems, *Rs = Bs + kMB * kLdB;
  TL *Xs = reinterpret_cast<TL *>(Rs + kMB * kLdB);
  __shared__ int waitOk;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, mw = warp & 3, kh = warp >> 2;
  auto bail = [] {  // a wait gave up: drain this thread's copies into shared memory before the CTA leaves
    cp_async_all();
    return false;
  };
  // one block task for vector slice sl
  auto run_slice = [&](const int4 t, const int sl) -> bool {
    const int s = t.x, blk = t.y;
    const int f = P.snF[s], nc = P.snNc[s], m = P.snM[s];
    const int vb = sl * kQS, qs = min(kQS, q - vb);
    const TL *Lp = Lx + P.snLxp[s];
    const int *rowsOf = P.Si + P.Sp[s];
    const int c0 = blk * kMB, w = min(kMB, nc - c0), nb = (nc + kMB - 1) / kMB;
    int *sflags = flags + (int64_t)sl * nflags;
    int *myflags = sflags + P.blkOff[s];
    {  // X^T: Xs[i][j] = X(j, i) = X[i w + j] ([m][k] with m = i), arriving while the task sums
      const TL *X = Inv + P.invOff[P.blkOff[s] + blk];
      for (int e = tid; e < kMB * kMB; e += kMultiThreads) {
        const int j = e & (kMB - 1), i = e >> 6;
        const bool ok = i < w && j < w;
        cp_async_el(Xs + i * kLdX + j, ok ? X + (int64_t)i * w + j : X, (int)sizeof(TL), ok);
      }
      asm volatile("cp.async.commit_group;\n" ::: "memory");
    }
    double c[2][4];
#pragma unroll
    for (int nb2 = 0; nb2 < 2; nb2++)
#pragma unroll
      for (int v = 0; v < 4; v++) c[nb2][v] = 0.0;
    // chunks: the rows below the supernode [nc, m) in kKC steps from the last down, then pivot blocks nb - 1 .. blk + 1
    // (two chunks each)
    const bool chain = Gch != nullptr && blk + 1 < nb;  // block b + 1 enters through G_b after its flag
    const int nanc = (m - nc + kKC - 1) / kKC;
    const int npiv = (nb - 1 - blk - (chain ? 1 : 0)) * (kMB / kKC);
    const int nch = nanc + npiv;
    auto chunk = [&](int ch, int &rb, int &rw) {
      if (ch < nanc) {
        rb = nc + (nanc - 1 - ch) * kKC;
        rw = min(kKC, m - rb);
      } else {
        const int p = ch - nanc, pb = nb - 1 - p / 2;  // pivot block, from the last down
        rb = pb * kMB + (p & 1) * kKC;
        rw = max(0, min(kKC, nc - rb));
      }
    };
    // L chunk, [m][k]: As[cc][rr] = L(rb + rr, c0 + cc); elements e = tid + 256 u: rr = e & 31, cc = e >> 5
    TL lr[8];
    auto loadL = [&](int rb, int rw) {
#pragma unroll
      for (int u = 0; u < 8; u++) {
        const int e = tid + kMultiThreads * u, rr = e & (kKC - 1), cc = e >> 5;
        lr[u] = (rr < rw && cc < w) ? Lp[(int64_t)(c0 + cc) * m + rb + rr] : (TL)0;
      }
    };
    int rb = 0, rw = 0;
    if (nch > 0) {
      chunk(0, rb, rw);
      loadL(rb, rw);
    }
    for (int ch = 0; ch < nch; ch++) {
      const bool anc = ch < nanc;
      if (anc) {  // the ancestor blocks holding this chunk's rows final? (one lane per row, each distinct block once)
        if (warp == 0) {
          const int fb = lane < rw ? P.rowBlk[rowsOf[rb + lane]] : -1;
          const int prev = __shfl_up_sync(0xffffffffu, fb, 1);
          int ok = 1;
          if (fb >= 0 && (lane == 0 || fb != prev)) ok = wait_flag(sflags + fb, epoch, status, s, P.spin);
          ok = __all_sync(0xffffffffu, ok);
          if (lane == 0) waitOk = ok;
        }
        __syncthreads();
        if (!waitOk) return bail();
      } else if (((ch - nanc) & 1) == 0) {  // first chunk of a pivot block: its x values final?
        if (tid == 0) waitOk = wait_flag(myflags + rb / kMB, epoch, status, s, P.spin);
        __syncthreads();
        if (!waitOk) return bail();
      }
      for (int e = tid; e < kKC * kQS; e += kMultiThreads) {
        const int rr = e >> 4, n = e & (kQS - 1);
        double v = 0.0;
        if (rr < rw && n < qs) {
          const int gi = anc ? rowsOf[rb + rr] : f + rb + rr;
          v = __ldcg(y + (int64_t)gi * q + vb + n);
        }
        Bs[rr * kLdB + n] = v;
      }
#pragma unroll
      for (int u = 0; u < 8; u++) {
        const int e = tid + kMultiThreads * u;
        As[(e >> 5) * kLdMK + (e & (kKC - 1))] = (double)lr[u];
      }
      __syncthreads();
      const int cw = rw;
      if (ch + 1 < nch) {
        chunk(ch + 1, rb, rw);
        loadL(rb, rw);
      }
      if (16 * kh < cw) mma_k16<false>(As, kLdMK, Bs, 16 * kh, mw, lane, c);
      __syncthreads();
    }
    halves_sum(c, As, warp, lane);
    // R = y[block] (/ D) - acc
    if (warp < 4) {
#pragma unroll
      for (int nb2 = 0; nb2 < 2; nb2++)
#pragma unroll
        for (int v = 0; v < 4; v++) {
          const int cc = acc_row(warp, lane, v), n = acc_vec(lane, nb2, v);
          double r = 0.0;
          if (cc < w && n < qs) {
            const double yv = y[(int64_t)(f + c0 + cc) * q + vb + n];
            r = (Dpiv ? yv / Dpiv[f + c0 + cc] : yv) - c[nb2][v];  // LDL^T: y /= D before the backward sweep (ldlt.mjs:629)
          }
          Rs[cc * kLdB + n] = r;
          c[nb2][v] = 0.0;
        }
    }
    if (warp >= 4) {
#pragma unroll
      for (int nb2 = 0; nb2 < 2; nb2++)
#pragma unroll
        for (int v = 0; v < 4; v++) c[nb2][v] = 0.0;
    }
    cp_async_all();
    __syncthreads();
    // x[block] = X^T R
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const int k0 = 32 * h + 16 * kh;
      if (k0 < w) mma_k16<false>(Xs, kLdX, Rs, k0, mw, lane, c);
    }
    halves_sum(c, As, warp, lane);
    if (chain) {
      // W stays in Rs; G_b^T arrives in Xs while the task waits for block b + 1
      const int rn = (blk + 1) * kMB, wn = min(kMB, nc - rn);
      if (warp < 4) {
#pragma unroll
        for (int nb2 = 0; nb2 < 2; nb2++)
#pragma unroll
          for (int v = 0; v < 4; v++) {
            const int cc = acc_row(warp, lane, v), n = acc_vec(lane, nb2, v);
            Rs[cc * kLdB + n] = c[nb2][v];
          }
      }
#pragma unroll
      for (int nb2 = 0; nb2 < 2; nb2++)
#pragma unroll
        for (int v = 0; v < 4; v++) c[nb2][v] = 0.0;
      __syncthreads();  // every warp is done with X^T in Xs
      {  // G_b^T ([m][k]): Xs[i][r] = G(r, i) = G[i 64 + r], G (wn x w, column-major)
        const TL *G = Gch + (int64_t)(P.blkOff[s] - s + blk) * kMB * kMB;
        for (int e = tid; e < kMB * kMB; e += kMultiThreads) {
          const int r = e & (kMB - 1), i = e >> 6;
          const bool ok = i < w && r < wn;
          cp_async_el(Xs + i * kLdX + r, ok ? G + (int64_t)i * kMB + r : G, (int)sizeof(TL), ok);
        }
        asm volatile("cp.async.commit_group;\n" ::: "memory");
      }
      if (tid == 0) waitOk = wait_flag(myflags + blk + 1, epoch, status, s, P.spin);
      __syncthreads();
      if (!waitOk) return bail();
      for (int e = tid; e < kMB * kQS; e += kMultiThreads) {
        const int r = e >> 4, n = e & (kQS - 1);
        Bs[r * kLdB + n] = (r < wn && n < qs) ? __ldcg(y + (int64_t)(f + rn + r) * q + vb + n) : 0.0;
      }
      cp_async_all();
      __syncthreads();
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const int k0 = 32 * h + 16 * kh;
        if (k0 < wn) mma_k16<false>(Xs, kLdX, Bs, k0, mw, lane, c);
      }
      halves_sum(c, As, warp, lane);
      if (warp < 4) {
#pragma unroll
        for (int nb2 = 0; nb2 < 2; nb2++)
#pragma unroll
          for (int v = 0; v < 4; v++) {
            const int cc = acc_row(warp, lane, v), n = acc_vec(lane, nb2, v);
            if (cc < w && n < qs) y[(int64_t)(f + c0 + cc) * q + vb + n] = Rs[cc * kLdB + n] - c[nb2][v];
          }
      }
      __syncthreads();
      if (tid == 0) st_release(myflags + blk, epoch);
      return true;
    }
    if (warp < 4) {
#pragma unroll
      for (int nb2 = 0; nb2 < 2; nb2++)
#pragma unroll
        for (int v = 0; v < 4; v++) {
          const int cc = acc_row(warp, lane, v), n = acc_vec(lane, nb2, v);
          if (cc < w && n < qs) y[(int64_t)(f + c0 + cc) * q + vb + n] = c[nb2][v];
        }
    }
    __syncthreads();
    if (tid == 0) st_release(myflags + blk, epoch);
    return true;
  };
  auto run = [&](const int tkv) -> bool {
    const int4 t = tasks[tkv];
    if (t.z == 2) {  // up to kSolveGroup supernodes with m <= 32, one warp each, all q vectors
      if (tid == 0) waitOk = 1;
      __syncthreads();
      if (warp < t.y && !small_bwd_warp_multi<TL>(P.solveSmall[t.x + warp], P, Lx, Dpiv, y, flags, nflags, epoch, q,
                                                  ns, status, msm + 32 * kMQ * warp))
        waitOk = 0;
      __syncthreads();
      return waitOk != 0;
    }
    if constexpr (WIDE) {
      if (t.w < 0) return bwd_wide_task<TL>(t, P, Lx, Inv, Dpiv, y, flags, nflags, epoch, q, ns, status, msm, waitOk);
    }
    return run_slice(t, t.w);
  };
  ticket_loop(ticket, ntasks, run);
}

// ---- layout and vector kernels -------------------------------------------------------------------------------------
// Yil[i q + k] = B[k n + i] through 32 x 32 shared tiles (both sides coalesced)
__global__ void k_to_interleaved(const double *__restrict__ B, double *__restrict__ Yil, int n, int q) {
  __shared__ double t[32][33];
  const int i0 = blockIdx.x * 32, k0 = blockIdx.y * 32;
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int k = k0 + r, i = i0 + threadIdx.x;
    if (k < q && i < n) t[r][threadIdx.x] = B[(int64_t)k * n + i];
  }
  __syncthreads();
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int i = i0 + r, k = k0 + threadIdx.x;
    if (i < n && k < q) Yil[(int64_t)i * q + k] = t[threadIdx.x][r];
  }
}
// X[k n + i] = Xil[i q + k]
__global__ void k_from_interleaved(const double *__restrict__ Xil, double *__restrict__ X, int n, int q) {
  __shared__ double t[32][33];
  const int i0 = blockIdx.x * 32, k0 = blockIdx.y * 32;
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int i = i0 + r, k = k0 + threadIdx.x;
    if (i < n && k < q) t[r][threadIdx.x] = Xil[(int64_t)i * q + k];
  }
  __syncthreads();
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int k = k0 + r, i = i0 + threadIdx.x;
    if (k < q && i < n) X[(int64_t)k * n + i] = t[threadIdx.x][r];
  }
}
// row gather / scatter of interleaved rows: y[i] = b[perm[i]] (in), x[perm[i]] = y[i] (out)
__global__ void k_rows_permute(const double *__restrict__ src, double *__restrict__ dst, const int *__restrict__ perm,
                               int n, int q, int scatter) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (int64_t)n * q) return;
  const int i = (int)(e / q), k = (int)(e - (int64_t)i * q);
  const int p = perm[i];
  if (scatter)
    dst[(int64_t)p * q + k] = src[e];
  else
    dst[e] = src[(int64_t)p * q + k];
}

// r = b - A x for q interleaved vectors, with the squared norms of r and b summed per (row group, vector):
// norms[2 (g q + k)] += ||r_k restricted to group g||^2, norms[2 (g q + k) + 1] += the same for b (zeroed by the
// caller). rowGroup == nullptr: one group. One warp per row, lane l holds vectors l and l + 32.
//   one group: rows grid-strided over the warps; the squares stay in registers and each block adds its sums with one
//              atomic pair per vector;
//   groups:    each warp takes a contiguous range of rows and adds its sums whenever the group changes.
__global__ void __launch_bounds__(256) k_residual_multi(int n, const int *__restrict__ rowptr,
                                                        const int *__restrict__ colidx, const double *__restrict__ val,
                                                        const double *__restrict__ x, const double *__restrict__ b,
                                                        double *__restrict__ r, double *__restrict__ norms, int q,
                                                        const int *__restrict__ rowGroup) {
  __shared__ double red[8][2 * kMQ];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int k0 = lane, k1 = lane + 32;
  const bool v0 = k0 < q, v1 = k1 < q;
  double rr0 = 0.0, rr1 = 0.0, bb0 = 0.0, bb1 = 0.0;
  auto row = [&](int64_t i) {
    double s0 = 0.0, s1 = 0.0;
    const int p1 = rowptr[i + 1];
#pragma unroll 4
    for (int p = rowptr[i]; p < p1; p++) {
      const double a = val[p];
      const double *xr = x + (int64_t)colidx[p] * q;
      if (v0) s0 = fma(a, xr[k0], s0);
      if (v1) s1 = fma(a, xr[k1], s1);
    }
    if (v0) {
      const double bi = b[i * q + k0], ri = bi - s0;
      r[i * q + k0] = ri;
      rr0 += ri * ri;
      bb0 += bi * bi;
    }
    if (v1) {
      const double bi = b[i * q + k1], ri = bi - s1;
      r[i * q + k1] = ri;
      rr1 += ri * ri;
      bb1 += bi * bi;
    }
  };
  if (rowGroup) {
    const int64_t nw = (int64_t)gridDim.x * 8, gw = (int64_t)blockIdx.x * 8 + warp;
    const int64_t per = (n + nw - 1) / nw, i0 = gw * per, i1 = min((int64_t)n, i0 + per);
    int g = i0 < i1 ? rowGroup[i0] : 0;
    auto flush = [&] {
      double *nb = norms + 2 * (int64_t)g * q;
      if (v0) {
        atomicAdd(nb + 2 * k0, rr0);
        atomicAdd(nb + 2 * k0 + 1, bb0);
      }
      if (v1) {
        atomicAdd(nb + 2 * k1, rr1);
        atomicAdd(nb + 2 * k1 + 1, bb1);
      }
      rr0 = rr1 = bb0 = bb1 = 0.0;
    };
    for (int64_t i = i0; i < i1; i++) {
      const int gi = rowGroup[i];
      if (gi != g) {
        flush();
        g = gi;
      }
      row(i);
    }
    if (i0 < i1) flush();
    return;
  }
  for (int64_t i = (int64_t)blockIdx.x * 8 + warp; i < n; i += (int64_t)gridDim.x * 8) row(i);
  red[warp][2 * k0] = rr0;
  red[warp][2 * k0 + 1] = bb0;
  red[warp][2 * k1] = rr1;
  red[warp][2 * k1 + 1] = bb1;
  __syncthreads();
  if (threadIdx.x < 2 * q) {
    double a = 0.0;
    for (int w = 0; w < 8; w++) a += red[w][threadIdx.x];
    atomicAdd(norms + threadIdx.x, a);
  }
}

template <class TL, bool WIDE>
static cudaError_t set_multi_smem() {
  cudaError_t e =
      cudaFuncSetAttribute(k_fwd_multi<TL, WIDE>, cudaFuncAttributeMaxDynamicSharedMemorySize, multi_smem<TL>());
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_bwd_multi<TL, WIDE>, cudaFuncAttributeMaxDynamicSharedMemorySize, multi_smem<TL>());
  return e;
}
cudaError_t init_solve_multi_attributes() {
  cudaError_t e = set_multi_smem<double, false>();
  if (e == cudaSuccess) e = set_multi_smem<double, true>();
  if (e == cudaSuccess) e = set_multi_smem<float, false>();
  return e == cudaSuccess ? set_multi_smem<float, true>() : e;
}

int num_sms();
int multi_max_vectors() { return kMQ; }
int multi_slices(int q) { return (q + kQS - 1) / kQS; }
static int multi_grid(int64_t ntasks) {
  return ntasks < kMultiCtas * num_sms() ? (int)ntasks : kMultiCtas * num_sms();
}

template <class TL>
void launch_fwd_multi(const int4 *tasks, int ntasks, bool wide, int *ticket, const DevPlan &P, const TL *Lx,
                      const TL *Inv, const TL *Mch, double *y, double *T, int *flags, int nflags, int epoch, int *done,
                      int q, unsigned long long *status, cudaStream_t st) {
  const int ns = multi_slices(q);
  if (ntasks <= 0) return;
  auto k = wide ? k_fwd_multi<TL, true> : k_fwd_multi<TL, false>;
  k<<<multi_grid(ntasks), kMultiThreads, multi_smem<TL>(), st>>>(tasks, ntasks, ns, ticket, P, Lx, Inv, Mch, y, T,
                                                                  flags, nflags, epoch, done, q, status);
}
template <class TL>
void launch_bwd_multi(const int4 *tasks, int ntasks, bool wide, int *ticket, const DevPlan &P, const TL *Lx,
                      const TL *Inv, const TL *Gch, const double *Dpiv, double *y, int *flags, int nflags, int epoch,
                      int q, unsigned long long *status, cudaStream_t st) {
  const int ns = multi_slices(q);
  if (ntasks <= 0) return;
  auto k = wide ? k_bwd_multi<TL, true> : k_bwd_multi<TL, false>;
  k<<<multi_grid(ntasks), kMultiThreads, multi_smem<TL>(), st>>>(tasks, ntasks, ns, ticket, P, Lx, Inv, Gch, Dpiv, y,
                                                                  flags, nflags, epoch, q, status);
}
void launch_to_interleaved(const double *B, double *Yil, int n, int q, cudaStream_t st) {
  if (n > 0 && q > 0) k_to_interleaved<<<dim3((n + 31) / 32, (q + 31) / 32), dim3(32, 8), 0, st>>>(B, Yil, n, q);
}
void launch_from_interleaved(const double *Xil, double *X, int n, int q, cudaStream_t st) {
  if (n > 0 && q > 0) k_from_interleaved<<<dim3((n + 31) / 32, (q + 31) / 32), dim3(32, 8), 0, st>>>(Xil, X, n, q);
}
void launch_rows_permute(const double *src, double *dst, const int *perm, int n, int q, bool scatter, cudaStream_t st) {
  const int64_t tot = (int64_t)n * q;
  if (tot > 0) k_rows_permute<<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(src, dst, perm, n, q, scatter ? 1 : 0);
}
void launch_residual_multi(int n, const int *rowptr, const int *colidx, const double *val, const double *x,
                           const double *b, double *r, double *norms, int q, const int *rowGroup, cudaStream_t st) {
  if (n <= 0 || q <= 0) return;
  const int64_t want = ((int64_t)n + 7) / 8;
  const int grid = (int)(want < 8 * num_sms() ? want : 8 * num_sms());
  k_residual_multi<<<grid, 256, 0, st>>>(n, rowptr, colidx, val, x, b, r, norms, q, rowGroup);
}
template void launch_fwd_multi<double>(const int4 *, int, bool, int *, const DevPlan &, const double *,
                                       const double *, const double *, double *, double *, int *, int, int, int *, int,
                                       unsigned long long *, cudaStream_t);
template void launch_fwd_multi<float>(const int4 *, int, bool, int *, const DevPlan &, const float *, const float *,
                                      const float *, double *, double *, int *, int, int, int *, int,
                                      unsigned long long *, cudaStream_t);
template void launch_bwd_multi<double>(const int4 *, int, bool, int *, const DevPlan &, const double *,
                                       const double *, const double *, const double *, double *, int *, int, int, int,
                                       unsigned long long *, cudaStream_t);
template void launch_bwd_multi<float>(const int4 *, int, bool, int *, const DevPlan &, const float *, const float *,
                                      const float *, const double *, double *, int *, int, int, int,
                                      unsigned long long *, cudaStream_t);

}  // namespace amp
