// Supernodal triangular solves with several right-hand sides at once (sparse.mjs solveNumericMulti :1261-1310,
// ldlt.mjs solveMany :595-643): the same task lists, flags and ticket order as the one-vector sweeps (solve.cu), but
// every task moves all q <= 64 vectors together, so each L element is read once per sweep instead of once per vector.
//
// Vectors are interleaved: entry i of vector k sits at y[i q + k] (and likewise the front vectors V and the pass-up
// buffers T), so a row of the solution is q contiguous doubles and the gathers through the extend-add maps and the
// row lists move whole rows.
//
// A task is a small GEMM: out (64 rows x q) = sum over a reduction index of A (64 x KC tile) times B (KC x q tile),
// both tiles staged in shared memory (FP64; FP32 factors are widened on load), each thread accumulating a 4 x 4
// register tile. Forward: A = L[block rows, pivot columns so far], B = y[those columns]. Backward: A = the block's
// columns of L over the rows below the block (transposed on load), B = x[those rows]. Then the 64 x 64 inverse of the
// diagonal block is applied the same way.
#include <cuda_runtime.h>

#include <cstdint>

#include "../host/plan.hpp"
#include "devplan.cuh"
#include "solve_small.cuh"
#include "sync.cuh"

namespace amp {

constexpr int kMB = 64;              // rows of a block task
constexpr int kKC = 32;              // reduction chunk
constexpr int kMQ = 64;              // vectors per pass (the host splits larger sets)
constexpr int kLdt = 66;             // shared tile row stride in doubles (even: 16-byte aligned double2 reads)
constexpr int kMultiThreads = 256;
constexpr int kMultiSmem = (2 * kKC + kMB) * kLdt * (int)sizeof(double);
static_assert(kSolveGroup * 32 * kMQ * (int)sizeof(double) <= kMultiSmem, "small-supernode tasks: front vectors");
// acc[i][j] += sum over kk < kc of A[kk][4 ty + i] B[kk][4 tx + j]
__device__ __forceinline__ void mm_tile(const double *__restrict__ A, const double *__restrict__ B, int kc, int ty,
                                        int tx, double (&acc)[4][4]) {
#pragma unroll 4
  for (int kk = 0; kk < kc; kk++) {
    const double2 a0 = *reinterpret_cast<const double2 *>(A + kk * kLdt + 4 * ty);
    const double2 a1 = *reinterpret_cast<const double2 *>(A + kk * kLdt + 4 * ty + 2);
    const double2 b0 = *reinterpret_cast<const double2 *>(B + kk * kLdt + 4 * tx);
    const double2 b1 = *reinterpret_cast<const double2 *>(B + kk * kLdt + 4 * tx + 2);
    const double a[4] = {a0.x, a0.y, a1.x, a1.y}, b[4] = {b0.x, b0.y, b1.x, b1.y};
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
      for (int j = 0; j < 4; j++) acc[i][j] = fma(a[i], b[j], acc[i][j]);
  }
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

// ---- forward ------------------------------------------------------------------------------------------------------
// task (s, blk, below): as k_fwd_blocks. Diagonal: y[block] = X (V[block] - L[block, 0:blk 64] y[0:blk 64]);
// below: T[block] = V[block] - L[block, 0:nc] y[0:nc].
template <class TL>
__global__ void __launch_bounds__(kMultiThreads, 3) k_fwd_multi(const int4 *__restrict__ tasks, int ntasks,
                                                                int *__restrict__ ticket, DevPlan P,
                                                                const TL *__restrict__ Lx, const TL *__restrict__ Inv,
                                                                double *__restrict__ y, double *__restrict__ V,
                                                                double *__restrict__ T, int *__restrict__ flags,
                                                                int epoch, int *__restrict__ done, int q,
                                                                unsigned long long *status) {
  extern __shared__ double msm[];
  double *As = msm, *Bs = msm + kKC * kLdt, *Rs = msm + 2 * kKC * kLdt;
  __shared__ int waitOk;
  const int tid = threadIdx.x, ty = tid >> 4, tx = tid & 15;
  auto run = [&](const int tkv) -> bool {
    const int4 t = tasks[tkv];
    if (t.z == 2) {  // up to kSolveGroup supernodes with m <= 32, one warp each (32 x 64 doubles of msm per warp)
      const int warp = tid >> 5;
      if (tid == 0) waitOk = 1;
      __syncthreads();
      if (warp < t.y &&
          !small_fwd_warp_multi<TL>(P.solveSmall[t.x + warp], P, Lx, y, T, done, q, status, msm + 32 * kMQ * warp))
        waitOk = 0;
      __syncthreads();
      return waitOk != 0;
    }
    const int s = t.x, blk = t.y, below = t.z;
    const int f = P.snF[s], nc = P.snNc[s], m = P.snM[s], mu = m - nc;
    const TL *Lp = Lx + P.snLxp[s];
    const int r0 = below ? nc + blk * kMB : blk * kMB;
    const int rows = below ? min(kMB, mu - blk * kMB) : min(kMB, nc - blk * kMB);
    const int ncols = below ? nc : blk * kMB;
    int *myflags = flags + P.blkOff[s];
    const int64_t vbase = (int64_t)P.Sp[s];
    if (!below && blk == 0) {
      for (int qq = P.chPtr[s]; qq < P.chPtr[s + 1]; qq++) {
        const int c = P.chList[qq];
        const int need = (P.snM[c] - P.snNc[c] + kMB - 1) / kMB;
        if (tid == 0) waitOk = wait_count(done + c, need, status, s, P.spin);
        __syncthreads();
        if (!waitOk) return false;
      }
      // v_s = [y(f .. f + nc); 0] + the children's pass-up vectors in the reference's child order
      for (int64_t e = tid; e < (int64_t)m * q; e += kMultiThreads) {
        const int r = (int)(e / q), k = (int)(e - (int64_t)r * q);
        V[(vbase + r) * q + k] = r < nc ? y[(int64_t)(f + r) * q + k] : 0.0;
      }
      __syncthreads();
      for (int qq = P.chPtr[s]; qq < P.chPtr[s + 1]; qq++) {
        const int c = P.chList[qq];
        const int muc = P.snM[c] - P.snNc[c];
        const int *map = P.eaMap + P.eaPtr[c];
        const double *tc = T + P.snTOff[c] * q;
        for (int64_t e = tid; e < (int64_t)muc * q; e += kMultiThreads) {
          const int a = (int)(e / q), k = (int)(e - (int64_t)a * q);
          V[(vbase + map[a]) * q + k] += __ldcg(tc + e);
        }
        __syncthreads();
      }
    }
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
    const int nch = (ncols + kKC - 1) / kKC;
    if (nch > 0) loadL(0);
    for (int ch = 0; ch < nch; ch++) {
      const int cb = ch * kKC, cw = min(kKC, ncols - cb);
      if ((cb & (kMB - 1)) == 0) {  // first chunk of a pivot block: its y values final?
        if (tid == 0) waitOk = wait_flag(myflags + cb / kMB, epoch, status, s, P.spin);
        __syncthreads();
        if (!waitOk) return false;
      }
      for (int e = tid; e < kKC * kMQ; e += kMultiThreads) {
        const int c = e >> 6, k = e & (kMQ - 1);
        Bs[c * kLdt + k] = (c < cw && k < q) ? __ldcg(y + (int64_t)(f + cb + c) * q + k) : 0.0;
      }
#pragma unroll
      for (int u = 0; u < 8; u++) {
        const int e = tid + kMultiThreads * u;
        As[(e >> 6) * kLdt + (e & (kMB - 1))] = (double)lr[u];
      }
      __syncthreads();
      if (ch + 1 < nch) loadL(cb + kKC);
      mm_tile(As, Bs, cw, ty, tx, acc);
      __syncthreads();
    }
    // R = V[block] - acc (V final once the supernode's first diagonal block is: waited above, or gathered here)
    if (below) {
      double *to = T + (P.snTOff[s] + (int64_t)blk * kMB) * q;
#pragma unroll
      for (int i = 0; i < 4; i++) {
        const int row = 4 * ty + i;
        if (row >= rows) continue;
#pragma unroll
        for (int j = 0; j < 4; j++) {
          const int k = 4 * tx + j;
          if (k < q) to[(int64_t)row * q + k] = __ldcg(V + (vbase + r0 + row) * q + k) - acc[i][j];
        }
      }
      __syncthreads();
      if (tid == 0) red_release_add(done + s, 1);
      return true;
    }
#pragma unroll
    for (int i = 0; i < 4; i++) {
      const int row = 4 * ty + i;
#pragma unroll
      for (int j = 0; j < 4; j++) {
        const int k = 4 * tx + j;
        Rs[row * kLdt + k] = (row < rows && k < q) ? __ldcg(V + (vbase + r0 + row) * q + k) - acc[i][j] : 0.0;
        acc[i][j] = 0.0;
      }
    }
    // y[block] = X R, X = L_kk^-1 (rows x rows, column-major): As[jj][i] = X(i, jb + jj)
    const TL *X = Inv + P.invOff[P.blkOff[s] + blk];
    for (int jb = 0; jb < rows; jb += kKC) {
      const int jw = min(kKC, rows - jb);
      __syncthreads();
      for (int e = tid; e < kKC * kMB; e += kMultiThreads) {
        const int i = e & (kMB - 1), jj = e >> 6;
        As[jj * kLdt + i] = (i < rows && jj < jw) ? (double)X[(int64_t)(jb + jj) * rows + i] : 0.0;
      }
      __syncthreads();
      mm_tile(As, Rs + jb * kLdt, jw, ty, tx, acc);
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
    if (tid == 0) st_release(myflags + blk, epoch);
    return true;
  };
  ticket_loop(ticket, ntasks, run);
}

// ---- backward -----------------------------------------------------------------------------------------------------
// task (s, blk): x[block] = X^T (y[block] (/ D for LDL^T) - L[rows below the block, block columns]^T x[those rows]).
// The rows below the supernode (ancestors, final once the parent's first pivot block is) go first, then the later
// pivot blocks of the supernode from the last one down, each after its flag.
template <class TL>
__global__ void __launch_bounds__(kMultiThreads, 3) k_bwd_multi(const int4 *__restrict__ tasks, int ntasks,
                                                                int *__restrict__ ticket, DevPlan P,
                                                                const TL *__restrict__ Lx, const TL *__restrict__ Inv,
                                                                const double *__restrict__ Dpiv,
                                                                double *__restrict__ y, int *__restrict__ flags,
                                                                int epoch, int q, unsigned long long *status) {
  extern __shared__ double msm[];
  double *As = msm, *Bs = msm + kKC * kLdt, *Rs = msm + 2 * kKC * kLdt;
  __shared__ int waitOk;
  const int tid = threadIdx.x, ty = tid >> 4, tx = tid & 15;
  auto run = [&](const int tkv) -> bool {
    const int4 t = tasks[tkv];
    if (t.z == 2) {  // up to kSolveGroup supernodes with m <= 32, one warp each (32 x 64 doubles of msm per warp)
      const int warp = tid >> 5;
      if (tid == 0) waitOk = 1;
      __syncthreads();
      if (warp < t.y && !small_bwd_warp_multi<TL>(P.solveSmall[t.x + warp], P, Lx, Dpiv, y, flags, epoch, q, status,
                                                  msm + 32 * kMQ * warp))
        waitOk = 0;
      __syncthreads();
      return waitOk != 0;
    }
    const int s = t.x, blk = t.y;
    const int f = P.snF[s], nc = P.snNc[s], m = P.snM[s];
    const TL *Lp = Lx + P.snLxp[s];
    const int *rowsOf = P.Si + P.Sp[s];
    const int c0 = blk * kMB, w = min(kMB, nc - c0), nb = (nc + kMB - 1) / kMB;
    int *myflags = flags + P.blkOff[s];
    const int par = P.snParent[s];
    if (par >= 0) {
      if (tid == 0) waitOk = wait_flag(flags + P.blkOff[par], epoch, status, s, P.spin);
      __syncthreads();
      if (!waitOk) return false;
    }
    double acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
      for (int j = 0; j < 4; j++) acc[i][j] = 0.0;
    // chunks: ancestors rows [nc, m) in kKC steps, then pivot blocks nb - 1 .. blk + 1 (two chunks each)
    const int nanc = (m - nc + kKC - 1) / kKC;
    const int npiv = (nb - 1 - blk) * (kMB / kKC);
    const int nch = nanc + npiv;
    // chunk ch -> first row and row count
    auto chunk = [&](int ch, int &rb, int &rw) {
      if (ch < nanc) {
        rb = nc + ch * kKC;
        rw = min(kKC, m - rb);
      } else {
        const int p = ch - nanc, pb = nb - 1 - p / 2;  // pivot block, from the last down
        rb = pb * kMB + (p & 1) * kKC;
        rw = max(0, min(kKC, nc - rb));
      }
    };
    // L tile: As[rr][c] = L(rb + rr, c0 + c); elements e = tid + 256 u: rr = e & 31, c = e >> 5
    TL lr[8];
    auto loadL = [&](int rb, int rw) {
#pragma unroll
      for (int u = 0; u < 8; u++) {
        const int e = tid + kMultiThreads * u, rr = e & (kKC - 1), c = e >> 5;
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
      for (int e = tid; e < kKC * kMQ; e += kMultiThreads) {
        const int rr = e >> 6, k = e & (kMQ - 1);
        double v = 0.0;
        if (rr < rw && k < q) {
          const int gi = anc ? rowsOf[rb + rr] : f + rb + rr;
          v = __ldcg(y + (int64_t)gi * q + k);
        }
        Bs[rr * kLdt + k] = v;
      }
#pragma unroll
      for (int u = 0; u < 8; u++) {
        const int e = tid + kMultiThreads * u;
        As[(e & (kKC - 1)) * kLdt + (e >> 5)] = (double)lr[u];
      }
      __syncthreads();
      const int cw = rw;
      if (ch + 1 < nch) {
        chunk(ch + 1, rb, rw);
        loadL(rb, rw);
      }
      mm_tile(As, Bs, cw, ty, tx, acc);
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
        Rs[c * kLdt + k] = v;
        acc[i][j] = 0.0;
      }
    }
    // x[block] = X^T R: As[jj][i] = X(jb + jj, i) = Inv[i w + jb + jj]
    const TL *X = Inv + P.invOff[P.blkOff[s] + blk];
    for (int jb = 0; jb < w; jb += kKC) {
      const int jw = min(kKC, w - jb);
      __syncthreads();
      for (int e = tid; e < kKC * kMB; e += kMultiThreads) {
        const int jj = e & (kKC - 1), i = e >> 5;
        As[jj * kLdt + i] = (i < w && jj < jw) ? (double)X[(int64_t)i * w + jb + jj] : 0.0;
      }
      __syncthreads();
      mm_tile(As, Rs + jb * kLdt, jw, ty, tx, acc);
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
    if (tid == 0) st_release(myflags + blk, epoch);
    return true;
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

cudaError_t init_solve_multi_attributes() {
  cudaError_t e = cudaFuncSetAttribute(k_fwd_multi<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMultiSmem);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_fwd_multi<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMultiSmem);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_bwd_multi<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMultiSmem);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_bwd_multi<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMultiSmem);
  return e;
}

int num_sms();
int multi_max_vectors() { return kMQ; }
static int multi_grid(int ntasks) { return ntasks < 3 * num_sms() ? ntasks : 3 * num_sms(); }

template <class TL>
void launch_fwd_multi(const int4 *tasks, int ntasks, int *ticket, const DevPlan &P, const TL *Lx, const TL *Inv,
                      double *y, double *V, double *T, int *flags, int epoch, int *done, int q,
                      unsigned long long *status, cudaStream_t st) {
  if (ntasks > 0)
    k_fwd_multi<TL><<<multi_grid(ntasks), kMultiThreads, kMultiSmem, st>>>(tasks, ntasks, ticket, P, Lx, Inv, y, V, T,
                                                                          flags, epoch, done, q, status);
}
template <class TL>
void launch_bwd_multi(const int4 *tasks, int ntasks, int *ticket, const DevPlan &P, const TL *Lx, const TL *Inv,
                      const double *Dpiv, double *y, int *flags, int epoch, int q, unsigned long long *status,
                      cudaStream_t st) {
  if (ntasks > 0)
    k_bwd_multi<TL><<<multi_grid(ntasks), kMultiThreads, kMultiSmem, st>>>(tasks, ntasks, ticket, P, Lx, Inv, Dpiv, y,
                                                                          flags, epoch, q, status);
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
template void launch_fwd_multi<double>(const int4 *, int, int *, const DevPlan &, const double *, const double *,
                                       double *, double *, double *, int *, int, int *, int, unsigned long long *,
                                       cudaStream_t);
template void launch_fwd_multi<float>(const int4 *, int, int *, const DevPlan &, const float *, const float *,
                                      double *, double *, double *, int *, int, int *, int, unsigned long long *,
                                      cudaStream_t);
template void launch_bwd_multi<double>(const int4 *, int, int *, const DevPlan &, const double *, const double *,
                                       const double *, double *, int *, int, int, unsigned long long *, cudaStream_t);
template void launch_bwd_multi<float>(const int4 *, int, int *, const DevPlan &, const float *, const float *,
                                      const double *, double *, int *, int, int, unsigned long long *, cudaStream_t);

}  // namespace amp
