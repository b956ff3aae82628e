// FP64 CSR kernels for refinement: y = A x (matVec, sparse.mjs:219-228) and r = b - A x with per-vector squared
// norms (the residual of solveRefined, ldlt.mjs:262-269). One warp per row; q vectors stored one after another.
#include <cuda_runtime.h>

#include <cstdint>

namespace amp {

__global__ void k_matvec(int n, const int *__restrict__ rowptr, const int *__restrict__ colidx,
                         const double *__restrict__ val, const double *__restrict__ x, double *__restrict__ y, int q) {
  const int lane = threadIdx.x & 31;
  const int64_t row = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (row >= (int64_t)n * q) return;
  const int k = (int)(row / n), i = (int)(row % n);
  const double *xk = x + (int64_t)k * n;
  double s = 0.0;
  for (int p = rowptr[i] + lane; p < rowptr[i + 1]; p += 32) s += val[p] * xk[colidx[p]];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if (lane == 0) y[(int64_t)k * n + i] = s;
}

// r = b - A x; norms[2k] += ||r_k||^2, norms[2k+1] += ||b_k||^2 (zeroed by the caller). One warp per row; the
// squares are summed per block in shared memory and added with one atomic pair per block and vector.
__global__ void __launch_bounds__(256) k_residual(int n, const int *__restrict__ rowptr, const int *__restrict__ colidx,
                                                  const double *__restrict__ val, const double *__restrict__ x,
                                                  const double *__restrict__ b, double *__restrict__ r,
                                                  double *__restrict__ norms, int q) {
  __shared__ double rr[8], bb[8];
  __shared__ int kk[8];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t row = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  double ri2 = 0.0, bi2 = 0.0;
  int k = -1;
  if (row < (int64_t)n * q) {
    k = (int)(row / n);
    const int i = (int)(row % n);
    const double *xk = x + (int64_t)k * n;
    double s = 0.0;
    for (int p = rowptr[i] + lane; p < rowptr[i + 1]; p += 32) s += val[p] * xk[colidx[p]];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (lane == 0) {
      const double bi = b[(int64_t)k * n + i];
      const double ri = bi - s;
      r[(int64_t)k * n + i] = ri;
      ri2 = ri * ri;
      bi2 = bi * bi;
    }
  }
  if (lane == 0) {
    rr[warp] = ri2;
    bb[warp] = bi2;
    kk[warp] = k;
  }
  __syncthreads();
  if (threadIdx.x == 0) {  // consecutive rows: one atomic pair per run of rows of the same vector
    int cur = -1;
    double a = 0.0, c = 0.0;
    for (int w = 0; w < 8; w++) {
      if (kk[w] != cur) {
        if (cur >= 0) {
          atomicAdd(norms + 2 * cur, a);
          atomicAdd(norms + 2 * cur + 1, c);
        }
        cur = kk[w];
        a = c = 0.0;
      }
      a += rr[w];
      c += bb[w];
    }
    if (cur >= 0) {
      atomicAdd(norms + 2 * cur, a);
      atomicAdd(norms + 2 * cur + 1, c);
    }
  }
}

__global__ void k_axpy_inplace(double *__restrict__ x, const double *__restrict__ dx, int64_t len) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < len) x[i] += dx[i];
}

void launch_matvec(int n, const int *rowptr, const int *colidx, const double *val, const double *x, double *y, int q,
                   cudaStream_t st) {
  int64_t threads = (int64_t)n * q * 32;
  if (threads > 0) k_matvec<<<(unsigned)((threads + 255) / 256), 256, 0, st>>>(n, rowptr, colidx, val, x, y, q);
}
void launch_residual(int n, const int *rowptr, const int *colidx, const double *val, const double *x, const double *b,
                     double *r, double *norms, int q, cudaStream_t st) {
  int64_t threads = (int64_t)n * q * 32;
  if (threads > 0)
    k_residual<<<(unsigned)((threads + 255) / 256), 256, 0, st>>>(n, rowptr, colidx, val, x, b, r, norms, q);
}
void launch_axpy(double *x, const double *dx, int64_t len, cudaStream_t st) {
  if (len > 0) k_axpy_inplace<<<(unsigned)((len + 255) / 256), 256, 0, st>>>(x, dx, len);
}

}  // namespace amp
