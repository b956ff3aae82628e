// amp_front_factor_noalloc: partial Cholesky of one dense front in place, without any device allocation.
//
// Some callers cannot call cudaMalloc: a host application that hands all device memory to its own pool at start-up
// (a physics worker that refactors every time step inside a fixed memory budget), or one that must not stall its
// other streams (cudaMalloc and cudaFree can synchronise the device). For them this entry point keeps its scratch --
// one status word and one reader counter per 64-column pivot block -- in a file-scope __device__ array, present on
// every GPU that loads the library until the process exits. The caller passes the front (input and output).
//
// The algorithm is the one of the multifrontal factor's dense kernels (pivot-block POTRF + TRSM, then the DMMA
// trailing update), for a single front stored as one m x m column-major array (ld = m, lower part used).
//
// Scratch rules: every call shares the array and it keeps the last call's contents, so each call first resets the
// status word and the counters of its pivot blocks. Calls that overlap on the GPU (from several host threads or
// streams) race on the array; callers must serialise them. The first call on a device looks up the array's device
// address (cudaGetSymbolAddress) with that device current and caches it; make that first call before relying on
// anything else about the call sequence on that device.
//
// After a pivot failure (*fail_column >= 0) F holds a partial result, as the reference's factorization leaves its
// front after ok = false: the pivot blocks before the failing one are factored, their trailing updates applied, and
// the failing block and everything right of it are left as the last completed update wrote them.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <mutex>
#include <string>

#include "../../../include/ampsolve.h"
#include "../host/plan.hpp"
#include "devplan.cuh"

namespace amp {
void set_last_error(const std::string &msg);

namespace {

constexpr int kNoAllocMaxFront = 16384;                  // largest front m this entry point accepts
constexpr int kNoAllocMaxDevices = 64;                   // device ordinals 0 .. 63
constexpr int kNaRows = 256;                             // panel rows per CTA (one thread per row)
constexpr int kNoAllocBlocks = kNoAllocMaxFront / kPanel; // pivot blocks of the largest front
// [0] status word, [1 + k] readers of pivot block k: (1 + 256) x 8 bytes
static __device__ __align__(256) unsigned long long g_front_scratch[1 + kNoAllocBlocks];

__device__ __forceinline__ bool na_failed(const unsigned long long *st) {
  return *(volatile const unsigned long long *)st != kStatusOk;
}

// One CTA per chunk of 256 rows below pivot block [c0, c0 + w): factor the block, solve the chunk; the last CTA to
// have read the unfactored block writes it back.
__global__ void __launch_bounds__(256) k_front_panel_na(double *__restrict__ F, int m, int nc, int c0,
                                                        unsigned long long *scratch) {
  unsigned long long *status = scratch;
  if (na_failed(status)) return;
  const int w = min(kPanel, nc - c0), c1 = c0 + w;
  const int nchunks = c1 < m ? (m - c1 + kNaRows - 1) / kNaRows : 1;
  const int r0 = c1 + blockIdx.x * kNaRows, r1 = min(r0 + kNaRows, m);
  __shared__ double D[kPanel][kPanel + 1];
  __shared__ double invd[kPanel];
  __shared__ int fail, lastReader;
  const int tid = threadIdx.x;
  if (tid == 0) fail = -1;
  for (int e = tid; e < w * w; e += blockDim.x) {
    int i = e % w, j = e / w;
    if (i >= j) D[i][j] = F[(int64_t)(c0 + j) * m + (c0 + i)];
  }
  __syncthreads();
  if (tid == 0) {
    __threadfence();
    lastReader = atomicAdd(scratch + 1 + c0 / kPanel, 1ull) == (unsigned long long)(nchunks - 1);
  }
  for (int k = 0; k < w; k++) {
    if (tid == 0) {
      double d = D[k][k];
      if (!(d > 0.0))
        fail = k;
      else {
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
    if (tid == 0) atomicMin(status, status_word(c0 + fail, 1, 0));
    return;
  }
  if (lastReader)
    for (int e = tid; e < w * w; e += blockDim.x) {
      int i = e % w, j = e / w;
      if (i >= j) F[(int64_t)(c0 + j) * m + (c0 + i)] = D[i][j];
    }
  const int r = r0 + tid;
  if (c1 >= m || r >= r1) return;
  double x[kPanel];  // the row in registers, solved against the factored block (same order as the factor's panel)
#pragma unroll
  for (int c = 0; c < kPanel; c++) x[c] = (c < w) ? F[(int64_t)(c0 + c) * m + r] : 0.0;
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
    if (c < w) F[(int64_t)(c0 + c) * m + r] = x[c];
}

__device__ __forceinline__ void na_dmma(double (&c)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(c[0]), "+d"(c[1])
               : "d"(a), "d"(b));
}

constexpr int kNaLd = kTile + 4;

// Trailing update after pivot block [c0, c0 + w): lower 64 x 64 tiles of [c1, m), tile (I, J) from blockIdx.
__global__ void __launch_bounds__(128) k_front_update_na(double *__restrict__ F, int m, int nc, int c0,
                                                         const unsigned long long *scratch) {
  if (na_failed(scratch)) return;
  const int w = min(kPanel, nc - c0), c1 = c0 + w, wp = (w + 3) & ~3;
  const int b = blockIdx.x;
  int I = (int)((sqrt(8.0 * b + 1.0) - 1.0) * 0.5);
  while ((I + 1) * (I + 2) / 2 <= b) I++;
  while (I * (I + 1) / 2 > b) I--;
  const int J = b - I * (I + 1) / 2;
  const int i0 = c1 + kTile * I, j0 = c1 + kTile * J;
  extern __shared__ double smem_na[];
  double(*As)[kNaLd] = reinterpret_cast<double(*)[kNaLd]>(smem_na);
  double(*Bs)[kNaLd] = reinterpret_cast<double(*)[kNaLd]>(smem_na + kPanel * kNaLd);
  const int tid = threadIdx.x;
  for (int e = tid; e < wp * kTile; e += blockDim.x) {
    const int k = e / kTile, i = e % kTile;
    const int ri = i0 + i, rj = j0 + i;
    const double *col = F + (int64_t)(c0 + k) * m;
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
    for (int q = 0; q < 4; q++) acc[a][q][0] = acc[a][q][1] = 0.0;
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
      for (int q = 0; q < 4; q++) na_dmma(acc[a][q], af[a], bf[q]);
  }
#pragma unroll
  for (int a = 0; a < 4; a++)
#pragma unroll
    for (int q = 0; q < 4; q++)
#pragma unroll
      for (int v = 0; v < 2; v++) {
        const int i = i0 + wr + 8 * a + gid, j = j0 + wc + 8 * q + 2 * t4 + v;
        if (i < m && j < m && i >= j) F[(int64_t)j * m + i] -= acc[a][q][v];
      }
}

}  // namespace
}  // namespace amp

extern "C" AMP_API int amp_front_factor_noalloc(double *F, int32_t m, int32_t nc, void *stream,
                                                int32_t *fail_column) {
  using namespace amp;
  if (!F || m <= 0 || nc <= 0 || nc > m) {
    set_last_error("amp_front_factor_noalloc: need a device front F and 0 < nc <= m");
    return AMP_INVALID;
  }
  if (m > kNoAllocMaxFront) {
    set_last_error("amp_front_factor_noalloc: front of " + std::to_string(m) + " rows exceeds the maximum of " +
                   std::to_string(kNoAllocMaxFront) + " (static scratch size)");
    return AMP_INVALID;
  }
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    set_last_error(std::string("amp_front_factor_noalloc: cudaGetDevice: ") + cudaGetErrorString(e));
    return AMP_CUDA_ERROR;
  }
  if (dev < 0 || dev >= kNoAllocMaxDevices) {
    set_last_error("amp_front_factor_noalloc: device ordinal " + std::to_string(dev) + " is outside the supported 0.." +
                   std::to_string(kNoAllocMaxDevices - 1));
    return AMP_INVALID;
  }
  // Set-up once per device, with that device current: the device address of the scratch array and the kernel's
  // dynamic shared memory limit (a per-device attribute). Host threads making first calls take turns.
  static std::mutex s_mu;
  static unsigned long long *s_addr[kNoAllocMaxDevices] = {nullptr};
  unsigned long long *scratch = nullptr;
  {
    std::lock_guard<std::mutex> lock(s_mu);
    if (!s_addr[dev]) {
      unsigned long long *ptr = nullptr;
      e = cudaGetSymbolAddress((void **)&ptr, g_front_scratch);
      if (e != cudaSuccess || !ptr) {
        set_last_error(std::string("amp_front_factor_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        return AMP_CUDA_ERROR;
      }
      e = cudaFuncSetAttribute(k_front_update_na, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               2 * kPanel * kNaLd * (int)sizeof(double));
      if (e != cudaSuccess) {
        set_last_error(std::string("amp_front_factor_noalloc: cudaFuncSetAttribute: ") + cudaGetErrorString(e));
        return AMP_CUDA_ERROR;
      }
      s_addr[dev] = ptr;
    }
    scratch = s_addr[dev];
  }
  cudaStream_t st = (cudaStream_t)stream;
  const int blocks = (nc + kPanel - 1) / kPanel;
  // the array keeps the last call's contents: reset the status word (all ones = no failure) and the counters
  e = cudaMemsetAsync(scratch, 0xff, sizeof(unsigned long long), st);
  if (e == cudaSuccess) e = cudaMemsetAsync(scratch + 1, 0, sizeof(unsigned long long) * blocks, st);
  for (int k = 0; k < blocks && e == cudaSuccess; k++) {
    const int c0 = k * kPanel, c1 = std::min(c0 + kPanel, nc);
    const int nchunks = c1 < m ? (m - c1 + kNaRows - 1) / kNaRows : 1;
    k_front_panel_na<<<nchunks, 256, 0, st>>>(F, m, nc, c0, scratch);
    const int T = (m - c1 + kTile - 1) / kTile;
    if (T > 0)
      k_front_update_na<<<T * (T + 1) / 2, 128, 2 * kPanel * kNaLd * (int)sizeof(double), st>>>(F, m, nc, c0,
                                                                                               scratch);
    e = cudaGetLastError();
  }
  unsigned long long status = kStatusOk;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&status, scratch, sizeof status, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    set_last_error(std::string("amp_front_factor_noalloc: ") + cudaGetErrorString(e));
    return AMP_CUDA_ERROR;
  }
  if (fail_column) *fail_column = status == kStatusOk ? -1 : (int32_t)(status >> 32);
  return AMP_OK;
}
