// FP64 multifrontal numeric factorization (Cholesky) and supernodal solves on sm_100a.
//
// Per level of the supernodal tree (leaves first):
//   k_assemble  zero the front, scatter A's entries (sparse.mjs:965-973) and extend-add the children's update
//               matrices in the reference's child order (sparse.mjs:974-985). One CTA owns a block of 32 front
//               columns, so every entry has a single writer and the summation order is the reference's.
//   per pivot block of 64 columns:
//     k_panel   POTRF of the 64 x 64 diagonal block in shared memory (pivot test d > 0, sqrt, multiply by 1/dk as
//               sparse.mjs:1151-1156) and TRSM of 256 panel rows per CTA (rows held in registers).
//     k_update  trailing update F -= L21 L21^T on 64 x 64 lower tiles with FP64 tensor-core MMA (DMMA m8n8k4),
//               covering both the remaining pivot columns (in Lx) and the update block (in the U arena).
// The solves run the multifrontal vector form: forward per level bottom-up (each supernode passes one update vector
// of length mu to its parent, no atomics), backward per level top-down gathering ancestor values.
#include <cuda_runtime.h>

#include <cstdint>

#include "devplan.cuh"
#include "../host/plan.hpp"

namespace amp {

__device__ __forceinline__ double *front_addr(double *Lp, double *Up, int m, int nc, int i, int j) {
  // front entry (i, j), i >= j: first nc columns in the L panel (ld m), the rest in the U block (ld mu)
  return j < nc ? Lp + (int64_t)j * m + i : Up + (int64_t)(j - nc) * (m - nc) + (i - nc);
}

__device__ __forceinline__ bool failed(const unsigned long long *st) {
  return *(volatile const unsigned long long *)st != kStatusOk;
}

// ---------------------------------------------------------------------------------------------------------------
// Assembly + extend-add
// ---------------------------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_assemble(const AsmTask *__restrict__ tasks, DevPlan P,
                                                  const double *__restrict__ values, double *__restrict__ Lx,
                                                  double *__restrict__ U, const unsigned long long *status) {
  if (failed(status)) return;
  const AsmTask t = tasks[blockIdx.x];
  const int s = t.s, j0 = t.j0;
  const int f = P.snF[s], nc = P.snNc[s], m = P.snM[s];
  const int jend = min(j0 + kAsmCols, m);
  double *Lp = Lx + P.snLxp[s];
  double *Up = (m > nc) ? U + P.snUoff[s] : nullptr;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
  // 1. zero the lower part of the owned columns
  for (int j = j0 + warp; j < jend; j += nwarps)
    for (int i = j + lane; i < m; i += 32) *front_addr(Lp, Up, m, nc, i, j) = 0.0;
  __syncthreads();
  // 2. A's entries of the owned pivot columns (each (row, col) once)
  for (int j = j0 + warp; j < min(jend, nc); j += nwarps) {
    const int p0 = P.asmColPtr[f + j], p1 = P.asmColPtr[f + j + 1];
    for (int p = p0 + lane; p < p1; p += 32) Lp[P.asmDst[p]] += values[P.asmSrc[p]];
  }
  __syncthreads();
  // 3. children, one after another (stack order of the reference)
  for (int q = P.chPtr[s]; q < P.chPtr[s + 1]; q++) {
    const int c = P.chList[q];
    const int muc = P.snM[c] - P.snNc[c];
    if (muc <= 0) continue;
    const int *map = P.eaMap + P.eaPtr[c];
    const double *Uc = U + P.snUoff[c];
    // child columns b mapping into [j0, jend): map is increasing
    int lo = 0, hi = muc;
    while (lo < hi) {
      int mid = (lo + hi) >> 1;
      if (map[mid] < j0) lo = mid + 1; else hi = mid;
    }
    const int b0 = lo;
    hi = muc;
    while (lo < hi) {
      int mid = (lo + hi) >> 1;
      if (map[mid] < jend) lo = mid + 1; else hi = mid;
    }
    const int b1 = lo;
    for (int b = b0 + warp; b < b1; b += nwarps) {
      const int jj = map[b];
      const double *col = Uc + (int64_t)b * muc;
      for (int a = b + lane; a < muc; a += 32) *front_addr(Lp, Up, m, nc, map[a], jj) += col[a];
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------------------------------------------
// Panel: POTRF of the pivot block + TRSM of a chunk of rows below it
// ---------------------------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_panel(const PanelTask *__restrict__ tasks, DevPlan P, double *__restrict__ Lx,
                                               int *__restrict__ readers, unsigned long long *status) {
  if (failed(status)) return;
  const PanelTask t = tasks[blockIdx.x];
  const int s = t.s, c0 = t.c0;
  const int f = P.snF[s], nc = P.snNc[s], m = P.snM[s];
  const int w = min(kPanel, nc - c0);
  double *Lp = Lx + P.snLxp[s];
  __shared__ double D[kPanel][kPanel + 1];
  __shared__ double invd[kPanel];
  __shared__ int fail, lastReader;
  const int tid = threadIdx.x;
  if (tid == 0) fail = -1;
  for (int e = tid; e < w * w; e += blockDim.x) {
    int i = e % w, j = e / w;
    if (i >= j) D[i][j] = Lp[(int64_t)(c0 + j) * m + (c0 + i)];
  }
  __syncthreads();
  // Every row chunk factors its own copy of the pivot block; the last chunk to have read the unfactored block writes
  // the factored one back (no chunk waits for another).
  if (tid == 0) {
    __threadfence();
    lastReader = atomicAdd(readers + t.group, 1) == t.nchunks - 1;
  }
  for (int k = 0; k < w; k++) {
    if (tid == 0) {
      double d = D[k][k];
      if (!(d > 0.0)) {
        fail = k;
      } else {
        double dk = sqrt(d);
        D[k][k] = dk;
        invd[k] = 1.0 / dk;
      }
    }
    __syncthreads();
    if (fail >= 0) break;
    const double iv = invd[k];
    for (int i = k + 1 + tid; i < w; i += blockDim.x) D[i][k] *= iv;
    __syncthreads();
    const int r = w - k - 1;
    for (int e = tid; e < r * r; e += blockDim.x) {
      int i = k + 1 + e / r, j = k + 1 + e % r;
      if (j <= i) D[i][j] -= D[i][k] * D[j][k];
    }
    __syncthreads();
  }
  if (fail >= 0) {
    if (tid == 0) atomicMin(status, status_word(f + c0 + fail, 1, s));
    return;
  }
  if (lastReader) {
    for (int e = tid; e < w * w; e += blockDim.x) {
      int i = e % w, j = e / w;
      if (i >= j) Lp[(int64_t)(c0 + j) * m + (c0 + i)] = D[i][j];
    }
  }
  // TRSM: row r of the panel solves x L11^T = a, thread per row, the row in registers
  const int r = t.r0 + tid;
  if (r >= t.r1) return;
  double x[kPanel];
#pragma unroll
  for (int c = 0; c < kPanel; c++) x[c] = (c < w) ? Lp[(int64_t)(c0 + c) * m + r] : 0.0;
#pragma unroll
  for (int k = 0; k < kPanel; k++) {
    if (k < w) {
      x[k] *= invd[k];
#pragma unroll
      for (int c = k + 1; c < kPanel; c++)
        if (c < w) x[c] -= x[k] * D[c][k];
    }
  }
#pragma unroll
  for (int c = 0; c < kPanel; c++)
    if (c < w) Lp[(int64_t)(c0 + c) * m + r] = x[c];
}

// ---------------------------------------------------------------------------------------------------------------
// Trailing update: F[i0:i0+64, j0:j0+64] -= A B^T, A = panel rows i, B = panel rows j, K = pivot block width.
// 128 threads = 2 x 2 warps of 32 x 32; DMMA m8n8k4 (A row-major 8x4, B col-major 4x8, C 8x8 f64).
// ---------------------------------------------------------------------------------------------------------------
__device__ __forceinline__ void dmma_8x8x4(double (&c)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(c[0]), "+d"(c[1])
               : "d"(a), "d"(b));
}

constexpr int kLdT = kTile + 4;  // 68 doubles: conflict-free fragment loads

__global__ void __launch_bounds__(128) k_update(const TileTask *__restrict__ tasks, DevPlan P, double *__restrict__ Lx,
                                                double *__restrict__ U, const unsigned long long *status) {
  if (failed(status)) return;
  const TileTask t = tasks[blockIdx.x];
  const int s = t.s, c0 = t.c0, i0 = t.i0, j0 = t.j0;
  const int nc = P.snNc[s], m = P.snM[s];
  const int w = min(kPanel, nc - c0);
  const int wp = (w + 3) & ~3;
  double *Lp = Lx + P.snLxp[s];
  double *Up = (m > nc) ? U + P.snUoff[s] : nullptr;
  extern __shared__ double smem_upd[];
  double(*As)[kLdT] = reinterpret_cast<double(*)[kLdT]>(smem_upd);
  double(*Bs)[kLdT] = reinterpret_cast<double(*)[kLdT]>(smem_upd + kPanel * kLdT);
  const int tid = threadIdx.x;
  for (int e = tid; e < wp * kTile; e += blockDim.x) {
    const int k = e / kTile, i = e % kTile;
    const int ri = i0 + i, rj = j0 + i;
    const double *col = Lp + (int64_t)(c0 + k) * m;
    As[k][i] = (k < w && ri < m) ? col[ri] : 0.0;
    Bs[k][i] = (k < w && rj < m) ? col[rj] : 0.0;
  }
  __syncthreads();
  const int warp = tid >> 5, lane = tid & 31;
  const int wr = (warp >> 1) * 32, wc = (warp & 1) * 32;
  const int gid = lane >> 2, t4 = lane & 3;
  double acc[4][4][2];
#pragma unroll
  for (int a = 0; a < 4; a++)
#pragma unroll
    for (int b = 0; b < 4; b++) acc[a][b][0] = acc[a][b][1] = 0.0;
  for (int kk = 0; kk < wp; kk += 4) {
    double af[4], bf[4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
      af[q] = As[kk + t4][wr + 8 * q + gid];
      bf[q] = Bs[kk + t4][wc + 8 * q + gid];
    }
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
      for (int b = 0; b < 4; b++) dmma_8x8x4(acc[a][b], af[a], bf[b]);
  }
#pragma unroll
  for (int a = 0; a < 4; a++)
#pragma unroll
    for (int b = 0; b < 4; b++)
#pragma unroll
      for (int v = 0; v < 2; v++) {
        const int i = i0 + wr + 8 * a + gid, j = j0 + wc + 8 * b + 2 * t4 + v;
        if (i < m && j < m && i >= j) *front_addr(Lp, Up, m, nc, i, j) -= acc[a][b][v];
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

// Forward: one CTA per supernode of the level. V: per-supernode front vectors (offset Sp[s], length m, per RHS
// stride Vstride); T: pass-up vectors (offset snTOff[s], length mu, per RHS stride Tstride).
__global__ void __launch_bounds__(256) k_forward(const int *__restrict__ sns, DevPlan P, const double *__restrict__ Lx,
                                                 double *__restrict__ y, double *__restrict__ V, double *__restrict__ T,
                                                 int q, int64_t Vstride, int64_t Tstride) {
  const int s = sns[blockIdx.x];
  const int f = P.snF[s], nc = P.snNc[s], m = P.snM[s], mu = m - nc;
  const double *Lp = Lx + P.snLxp[s];
  for (int k = 0; k < q; k++) {
    double *v = V + (int64_t)k * Vstride + P.Sp[s];
    double *yk = y + (int64_t)k * P.n;
    for (int r = threadIdx.x; r < m; r += blockDim.x) v[r] = r < nc ? yk[f + r] : 0.0;
    __syncthreads();
    for (int qq = P.chPtr[s]; qq < P.chPtr[s + 1]; qq++) {
      const int c = P.chList[qq];
      const int muc = P.snM[c] - P.snNc[c];
      const int *map = P.eaMap + P.eaPtr[c];
      const double *tc = T + (int64_t)k * Tstride + P.snTOff[c];
      for (int a = threadIdx.x; a < muc; a += blockDim.x) v[map[a]] += tc[a];
      __syncthreads();
    }
    for (int c = 0; c < nc; c++) {
      const double *col = Lp + (int64_t)c * m;
      const double yc = v[c] / col[c];
      __syncthreads();
      if (threadIdx.x == 0) v[c] = yc;
      for (int r = c + 1 + threadIdx.x; r < m; r += blockDim.x) v[r] -= col[r] * yc;
      __syncthreads();
    }
    for (int r = threadIdx.x; r < nc; r += blockDim.x) yk[f + r] = v[r];
    double *ts = T + (int64_t)k * Tstride + P.snTOff[s];
    for (int r = threadIdx.x; r < mu; r += blockDim.x) ts[r] = v[nc + r];
    __syncthreads();
  }
}

// Backward: one CTA per supernode of the level (levels top-down); ancestors' x are final.
__global__ void __launch_bounds__(256) k_backward(const int *__restrict__ sns, DevPlan P, const double *__restrict__ Lx,
                                                  double *__restrict__ y, int q) {
  const int s = sns[blockIdx.x];
  const int f = P.snF[s], nc = P.snNc[s], m = P.snM[s];
  const double *Lp = Lx + P.snLxp[s];
  const int *rows = P.Si + P.Sp[s];
  __shared__ double red[256 / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int k = 0; k < q; k++) {
    double *yk = y + (int64_t)k * P.n;
    for (int c = nc - 1; c >= 0; c--) {
      const double *col = Lp + (int64_t)c * m;
      double part = 0.0;
      for (int r = c + 1 + threadIdx.x; r < m; r += blockDim.x) part += col[r] * yk[rows[r]];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) part += __shfl_down_sync(0xffffffffu, part, o);
      if (lane == 0) red[warp] = part;
      __syncthreads();
      if (threadIdx.x == 0) {
        double sum = 0.0;
        for (int wv = 0; wv < nw; wv++) sum += red[wv];
        yk[f + c] = (yk[f + c] - sum) / col[c];
      }
      __syncthreads();
    }
  }
}

// ---------------------------------------------------------------------------------------------------------------
// Launchers (host side)
// ---------------------------------------------------------------------------------------------------------------
void init_kernel_attributes() {
  cudaFuncSetAttribute(k_update, cudaFuncAttributeMaxDynamicSharedMemorySize, 2 * kPanel * kLdT * (int)sizeof(double));
}

void launch_assemble(const AsmTask *tasks, int64_t ntasks, const DevPlan &P, const double *values, double *Lx,
                     double *U, const unsigned long long *status, cudaStream_t st) {
  if (ntasks > 0) k_assemble<<<(unsigned)ntasks, 256, 0, st>>>(tasks, P, values, Lx, U, status);
}
void launch_panel(const PanelTask *tasks, int64_t ntasks, const DevPlan &P, double *Lx, int *readers,
                  unsigned long long *status, cudaStream_t st) {
  if (ntasks > 0) k_panel<<<(unsigned)ntasks, 256, 0, st>>>(tasks, P, Lx, readers, status);
}
void launch_update(const TileTask *tasks, int64_t ntasks, const DevPlan &P, double *Lx, double *U,
                   const unsigned long long *status, cudaStream_t st) {
  constexpr int smem = 2 * kPanel * kLdT * (int)sizeof(double);
  if (ntasks > 0) k_update<<<(unsigned)ntasks, 128, smem, st>>>(tasks, P, Lx, U, status);
}
void launch_permute_in(const double *b, double *y, const int *perm, int n, int q, cudaStream_t st) {
  int64_t tot = (int64_t)n * q;
  if (tot > 0) k_permute_in<<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(b, y, perm, n, q);
}
void launch_permute_out(const double *y, double *x, const int *perm, int n, int q, cudaStream_t st) {
  int64_t tot = (int64_t)n * q;
  if (tot > 0) k_permute_out<<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(y, x, perm, n, q);
}
void launch_forward(const int *sns, int count, const DevPlan &P, const double *Lx, double *y, double *V, double *T,
                    int q, int64_t Vstride, int64_t Tstride, cudaStream_t st) {
  if (count > 0) k_forward<<<count, 256, 0, st>>>(sns, P, Lx, y, V, T, q, Vstride, Tstride);
}
void launch_backward(const int *sns, int count, const DevPlan &P, const double *Lx, double *y, int q, cudaStream_t st) {
  if (count > 0) k_backward<<<count, 256, 0, st>>>(sns, P, Lx, y, q);
}

}  // namespace amp
