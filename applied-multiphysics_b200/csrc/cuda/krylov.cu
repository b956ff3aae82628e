// Vector kernels of the restarted GMRES driver (gmres-real.mjs:31-105), FP64, deterministic: the reductions sum
// fixed per-block partials in a fixed order, so a solve repeats bit for bit.
#include <cuda_runtime.h>

#include <cstdint>

namespace amp {

constexpr int kDotBlocks = 256;  // partial sums per dot product
constexpr int kDotThreads = 256;

// partial[j * kDotBlocks + block] = sum over the block's slice of V[j] . w, for j < nv (V rows of length n, ld n)
__global__ void __launch_bounds__(kDotThreads) k_dots_partial(const double *__restrict__ V, int nv, int64_t n,
                                                             const double *__restrict__ w, double *__restrict__ partial) {
  __shared__ double red[kDotThreads / 32];
  for (int j = 0; j < nv; j++) {
    const double *vj = V + (int64_t)j * n;
    double s = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
      s += vj[i] * w[i];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int k = 0; k < kDotThreads / 32; k++) t += red[k];
      partial[(int64_t)j * gridDim.x + blockIdx.x] = t;
    }
    __syncthreads();
  }
}

// out[j] = sum of the partials of dot j, in block order
__global__ void k_dots_final(const double *__restrict__ partial, int nv, int nblocks, double *__restrict__ out) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= nv) return;
  double t = 0.0;
  for (int b = 0; b < nblocks; b++) t += partial[(int64_t)j * nblocks + b];
  out[j] = t;
}

// w -= sum_j h[j] V[j]
__global__ void k_gs_update(double *__restrict__ w, const double *__restrict__ V, const double *__restrict__ h, int nv,
                            int64_t n) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double s = w[i];
  for (int j = 0; j < nv; j++) s -= h[j] * V[(int64_t)j * n + i];
  w[i] = s;
}

// x += sum_j y[j] Z[j]
__global__ void k_combine_add(double *__restrict__ x, const double *__restrict__ Z, const double *__restrict__ y, int nv,
                              int64_t n) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double s = 0.0;
  for (int j = 0; j < nv; j++) s += y[j] * Z[(int64_t)j * n + i];
  x[i] += s;
}

// v = a w
__global__ void k_scale_to(double *__restrict__ v, const double *__restrict__ w, double a, int64_t n) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) v[i] = a * w[i];
}

// v = w / sqrt(norm2[0]) (the next Arnoldi vector; left unchanged when the norm is zero, where GMRES stops)
__global__ void k_scale_by_norm(double *__restrict__ v, const double *__restrict__ w, const double *__restrict__ norm2,
                                int64_t n) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const double q = *norm2;
  if (i < n && q > 0.0) v[i] = (1.0 / sqrt(q)) * w[i];
}

// r = b - y
__global__ void k_sub_from(double *__restrict__ r, const double *__restrict__ b, const double *__restrict__ y,
                           int64_t n) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) r[i] = b[i] - y[i];
}

static unsigned blocks_for(int64_t n) { return (unsigned)((n + 255) / 256); }

int launch_dots(const double *V, int nv, int64_t n, const double *w, double *partial, double *out, cudaStream_t st) {
  if (nv <= 0) return 0;
  k_dots_partial<<<kDotBlocks, kDotThreads, 0, st>>>(V, nv, n, w, partial);
  k_dots_final<<<(nv + 63) / 64, 64, 0, st>>>(partial, nv, kDotBlocks, out);
  return 2;
}
void launch_gs_update(double *w, const double *V, const double *h, int nv, int64_t n, cudaStream_t st) {
  if (n > 0 && nv > 0) k_gs_update<<<blocks_for(n), 256, 0, st>>>(w, V, h, nv, n);
}
void launch_combine_add(double *x, const double *Z, const double *y, int nv, int64_t n, cudaStream_t st) {
  if (n > 0 && nv > 0) k_combine_add<<<blocks_for(n), 256, 0, st>>>(x, Z, y, nv, n);
}
void launch_scale_to(double *v, const double *w, double a, int64_t n, cudaStream_t st) {
  if (n > 0) k_scale_to<<<blocks_for(n), 256, 0, st>>>(v, w, a, n);
}
void launch_scale_by_norm(double *v, const double *w, const double *norm2, int64_t n, cudaStream_t st) {
  if (n > 0) k_scale_by_norm<<<blocks_for(n), 256, 0, st>>>(v, w, norm2, n);
}
void launch_sub_from(double *r, const double *b, const double *y, int64_t n, cudaStream_t st) {
  if (n > 0) k_sub_from<<<blocks_for(n), 256, 0, st>>>(r, b, y, n);
}
int dot_partials() { return kDotBlocks; }

}  // namespace amp
