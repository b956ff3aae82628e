// Solves and the refinement residual of the complex-symmetric LDL^T (the reference's ComplexSupernodalLDLT.solve and
// complexSolveRefined, ldlt.mjs:802-900): A = L D L^T with L unit lower (no conjugation), D complex diagonal.
//
// The sweeps go level by level over the supernodal tree (one launch per level, one CTA per supernode of the level),
// each supernode in 64-column blocks:
//   forward   the block's unit lower triangle by one warp (column by column), then every row below the block
//             takes its block product (one thread per row, coalesced reads of L's columns): rows of the supernode
//             in place, rows of ancestors by atomic subtraction (the ancestors run at later levels);
//   diagonal  y_j = y_j / D_j, written as the reference writes it ((a dr + b di) / den, (b dr - a di) / den);
//   backward  levels top-down, blocks last to first: each column of the block gathers its rows below (final values:
//             later blocks of the supernode, ancestors from earlier launches) by a warp reduction, then the block's
//             unit upper triangle (L11^T) by one warp.
// Sums run in a different order from the reference's sequential loops (atomic subtraction in the forward sweep,
// warp reductions in the backward one), so results agree with it to round-off, not bit for bit.
#include <cuda_runtime.h>

#include <cstdint>

#include "cplx.cuh"
#include "devplan.cuh"

namespace amp {

__device__ __forceinline__ cplx cld(const cplx *p) {
  const double2 v = *reinterpret_cast<const double2 *>(p);
  return cplx(v.x, v.y);
}
__device__ __forceinline__ cplx warp_sum(cplx v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    v.re += __shfl_down_sync(0xffffffffu, v.re, o);
    v.im += __shfl_down_sync(0xffffffffu, v.im, o);
  }
  return v;
}

// y (permuted order, complex) = b[perm[i]] from the planar right-hand side (br, bi)
__global__ void k_cpermute_in(int n, const double *__restrict__ br, const double *__restrict__ bi,
                              const int *__restrict__ perm, cplx *__restrict__ y) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) y[i] = cplx(br[perm[i]], bi[perm[i]]);
}
// x[perm[i]] = y[i], planar
__global__ void k_cpermute_out(int n, const cplx *__restrict__ y, const int *__restrict__ perm,
                               double *__restrict__ xr, double *__restrict__ xi) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    xr[perm[i]] = y[i].re;
    xi[perm[i]] = y[i].im;
  }
}
// interleave the planar values (re, im) of the CSR slots
__global__ void k_cpack(int64_t nnz, const double *__restrict__ re, const double *__restrict__ im,
                        cplx *__restrict__ out) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p < nnz) out[p] = cplx(re[p], im[p]);
}

__global__ void __launch_bounds__(256) k_cfwd_level(const int *__restrict__ sn, DevPlan P, const cplx *__restrict__ Lx,
                                                    cplx *__restrict__ y) {
  const int s = sn[blockIdx.x];
  const int f = P.snF[s], nc = P.snNc[s], m = P.snM[s];
  const cplx *L = Lx + P.snLxp[s];
  const int *rows = P.Si + P.Sp[s];
  __shared__ cplx yb[64];
  const int tid = threadIdx.x, lane = tid & 31;
  for (int p0 = 0; p0 < nc; p0 += 64) {
    const int w = min(64, nc - p0);
    if (tid < w) yb[tid] = y[f + p0 + tid];
    __syncthreads();
    if (tid < 32) {  // the block's unit lower triangle, column by column
      for (int c = 0; c < w; c++) {
        const cplx yc = yb[c];
        for (int r = c + 1 + lane; r < w; r += 32) yb[r] -= cld(L + (int64_t)(p0 + c) * m + p0 + r) * yc;
        __syncwarp();
      }
    }
    __syncthreads();
    if (tid < w) y[f + p0 + tid] = yb[tid];
    for (int r = p0 + w + tid; r < m; r += blockDim.x) {  // rows below the block
      cplx t(0.0);
      for (int c = 0; c < w; c++) t += cld(L + (int64_t)(p0 + c) * m + r) * yb[c];
      if (r < nc) {
        y[f + r] -= t;
      } else {
        double *d = reinterpret_cast<double *>(y + rows[r]);
        atomicAdd(d, -t.re);
        atomicAdd(d + 1, -t.im);
      }
    }
    __syncthreads();
  }
}

__global__ void k_cdiag(int n, const cplx *__restrict__ D, cplx *__restrict__ y) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const double ar = D[j].re, ai = D[j].im, den = ar * ar + ai * ai, a = y[j].re, b = y[j].im;
  y[j] = cplx((a * ar + b * ai) / den, (b * ar - a * ai) / den);
}

__global__ void __launch_bounds__(256) k_cbwd_level(const int *__restrict__ sn, DevPlan P, const cplx *__restrict__ Lx,
                                                    cplx *__restrict__ y) {
  const int s = sn[blockIdx.x];
  const int f = P.snF[s], nc = P.snNc[s], m = P.snM[s];
  const cplx *L = Lx + P.snLxp[s];
  const int *rows = P.Si + P.Sp[s];
  __shared__ cplx yb[64], sb[64];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int nblk = (nc + 63) / 64;
  for (int bk = nblk - 1; bk >= 0; bk--) {
    const int p0 = bk * 64, w = min(64, nc - p0);
    for (int c = warp; c < w; c += blockDim.x / 32) {  // the rows below the block, one warp per column
      cplx t(0.0);
      for (int r = p0 + w + lane; r < m; r += 32)
        t += cld(L + (int64_t)(p0 + c) * m + r) * (r < nc ? y[f + r] : y[rows[r]]);
      t = warp_sum(t);
      if (lane == 0) sb[c] = t;
    }
    __syncthreads();
    if (tid < w) yb[tid] = y[f + p0 + tid] - sb[tid];
    __syncthreads();
    if (tid < 32) {  // the block's unit upper triangle L11^T, last column first
      for (int c = w - 1; c >= 0; c--) {
        cplx t(0.0);
        for (int r = c + 1 + lane; r < w; r += 32) t += cld(L + (int64_t)(p0 + c) * m + p0 + r) * yb[r];
        t = warp_sum(t);
        if (lane == 0) yb[c] -= t;
        __syncwarp();
      }
    }
    __syncthreads();
    if (tid < w) y[f + p0 + tid] = yb[tid];
    __syncthreads();
  }
}

// r = b - A x (complex values on the CSR slots), norms[0] += ||r||^2, norms[1] += ||b||^2. One warp per row.
__global__ void __launch_bounds__(256) k_cresidual(int n, const int *__restrict__ rowptr, const int *__restrict__ colidx,
                                                   const cplx *__restrict__ val, const cplx *__restrict__ x,
                                                   const cplx *__restrict__ b, cplx *__restrict__ r,
                                                   double *__restrict__ norms) {
  const int lane = threadIdx.x & 31;
  const int64_t row = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (row >= n) return;
  cplx t(0.0);
  for (int p = rowptr[row] + lane; p < rowptr[row + 1]; p += 32) t += cld(val + p) * cld(x + colidx[p]);
  t = warp_sum(t);
  if (lane == 0) {
    const cplx bi = b[row], ri = bi - t;
    r[row] = ri;
    atomicAdd(norms, ri.re * ri.re + ri.im * ri.im);
    atomicAdd(norms + 1, bi.re * bi.re + bi.im * bi.im);
  }
}

__global__ void k_cpermute_vec(int n, const cplx *__restrict__ src, const int *__restrict__ perm, cplx *__restrict__ dst,
                               int gather) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (gather)
    dst[i] = src[perm[i]];
  else
    dst[perm[i]] = src[i];
}
__global__ void k_caxpy(int n, cplx *__restrict__ x, const cplx *__restrict__ dx) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) x[i] += dx[i];
}

// planar copy of a complex vector
__global__ void k_cunpack(int n, const cplx *__restrict__ x, double *__restrict__ xr, double *__restrict__ xi) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    xr[i] = x[i].re;
    xi[i] = x[i].im;
  }
}

// tau = pivotTol * max_i hypot(A(i, i)) (1 when that maximum is 0 or not a number; diagScale, ldlt.mjs:419-424)
__global__ void __launch_bounds__(1024) k_ctau(const cplx *__restrict__ values, const int *__restrict__ diagSlot, int n,
                                               double *scal) {
  __shared__ double red[32];
  double mx = 0.0;
  bool nan = false;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const cplx a = values[diagSlot[i]];
    const double h = hypot(a.re, a.im);
    if (h != h) nan = true;
    mx = fmax(mx, h);
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

static unsigned nblocks(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

void launch_cunpack(int n, const cplx *x, double *xr, double *xi, cudaStream_t st) {
  if (n > 0) k_cunpack<<<nblocks(n, 256), 256, 0, st>>>(n, x, xr, xi);
}
void launch_ctau(const cplx *values, const DevPlan &P, double *scal, cudaStream_t st) {
  k_ctau<<<1, 1024, 0, st>>>(values, P.diagSlot, P.n, scal);
}

void launch_cpack(int64_t nnz, const double *re, const double *im, cplx *out, cudaStream_t st) {
  if (nnz > 0) k_cpack<<<nblocks(nnz, 256), 256, 0, st>>>(nnz, re, im, out);
}
void launch_cpermute_in(int n, const double *br, const double *bi, const int *perm, cplx *y, cudaStream_t st) {
  if (n > 0) k_cpermute_in<<<nblocks(n, 256), 256, 0, st>>>(n, br, bi, perm, y);
}
void launch_cpermute_out(int n, const cplx *y, const int *perm, double *xr, double *xi, cudaStream_t st) {
  if (n > 0) k_cpermute_out<<<nblocks(n, 256), 256, 0, st>>>(n, y, perm, xr, xi);
}
void launch_cpermute_vec(int n, const cplx *src, const int *perm, cplx *dst, bool gather, cudaStream_t st) {
  if (n > 0) k_cpermute_vec<<<nblocks(n, 256), 256, 0, st>>>(n, src, perm, dst, gather ? 1 : 0);
}
void launch_caxpy(int n, cplx *x, const cplx *dx, cudaStream_t st) {
  if (n > 0) k_caxpy<<<nblocks(n, 256), 256, 0, st>>>(n, x, dx);
}
// y (permuted, complex) := A^-1 y: forward levels leaves first, the diagonal, backward levels top-down
int launch_csolve_permuted(const DevPlan &P, const int *lvlPtr, int nlevels, const cplx *L, const cplx *D, cplx *y,
                           cudaStream_t st) {
  int launched = 0;
  for (int Lv = 0; Lv < nlevels; Lv++) {
    const int c = lvlPtr[Lv + 1] - lvlPtr[Lv];
    if (c > 0) k_cfwd_level<<<c, 256, 0, st>>>(P.lvlSn + lvlPtr[Lv], P, L, y), launched++;
  }
  k_cdiag<<<nblocks(P.n, 256), 256, 0, st>>>(P.n, D, y);
  launched++;
  for (int Lv = nlevels - 1; Lv >= 0; Lv--) {
    const int c = lvlPtr[Lv + 1] - lvlPtr[Lv];
    if (c > 0) k_cbwd_level<<<c, 256, 0, st>>>(P.lvlSn + lvlPtr[Lv], P, L, y), launched++;
  }
  return launched;
}
void launch_cresidual(int n, const int *rowptr, const int *colidx, const cplx *val, const cplx *x, const cplx *b,
                      cplx *r, double *norms, cudaStream_t st) {
  if (n > 0) k_cresidual<<<nblocks((int64_t)n * 32, 256), 256, 0, st>>>(n, rowptr, colidx, val, x, b, r, norms);
}

}  // namespace amp
