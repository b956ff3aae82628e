// Supernodal triangular solves on sm_100a (sparse.mjs solveNumeric :1261-1305, supernodalSolve :1200-1258).
//
// Multifrontal vector form, one level of the supernodal tree per launch:
//   forward (levels bottom-up)
//     k_fwd_gather  v_s = [y(f .. f+nc); 0] + the children's pass-up vectors (extend-add in the reference's child
//                   order; one CTA per supernode, so no atomics)
//     k_fwd_blocks  tasks over 64-row blocks: diagonal block k computes v_k - L[k, 0:k] y(0:k) (row-block dot
//                   products) and solves with L_kk; below block j computes the pass-up vector
//                   u_j = v_j - L[j, 0:nc] y (read by the parent's gather)
//   backward (levels top-down)
//     k_bwd_blocks  column block k (reverse order): x_k = L_kk^-T (y_k - L[rows below k, k]^T x(rows)), the rows below
//                   the supernode gathered from the ancestors' final values
// Every L element is read once per sweep. Tasks inside a launch depend on earlier blocks of the same supernode: a
// CTA takes the next task with an atomic ticket (so it only ever waits for tasks already taken by running or finished
// CTAs) and waits on per-block ready flags with a bounded spin; on time-out it records AMP_DEVICE_TIMEOUT in the
// status word and returns.
#include <cuda_runtime.h>

#include <cstdint>

#include "../host/plan.hpp"
#include "devplan.cuh"

namespace amp {

constexpr int kSB = 64;                 // solve block rows
constexpr long long kSpinLimit = 1ll << 24;  // ~ seconds with the back-off below

__device__ __forceinline__ int ld_acquire(const int *p) {
  int v;
  asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release(int *p, int v) {
  asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Wait until flag == epoch; false on time-out (status set).
__device__ bool wait_flag(const int *flag, int epoch, unsigned long long *status, int s) {
  long long spins = 0;
  while (ld_acquire(flag) != epoch) {
    if (++spins > kSpinLimit) {
      atomicMin(status, status_word(0x7fffffff, 3, s));
      return false;
    }
    __nanosleep(64);
  }
  return true;
}

// Wait until *cnt == need; false on time-out (status set).
__device__ bool wait_count(const int *cnt, int need, unsigned long long *status, int s) {
  long long spins = 0;
  while (ld_acquire(cnt) < need) {
    if (++spins > kSpinLimit) {
      atomicMin(status, status_word(0x7fffffff, 3, s));
      return false;
    }
    __nanosleep(64);
  }
  return true;
}

// ---- forward gather ----------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_fwd_gather(const int *__restrict__ sns, DevPlan P, const double *__restrict__ y,
                                                    double *__restrict__ V, const double *__restrict__ T, int q,
                                                    int64_t Vstride, int64_t Tstride) {
  const int s = sns[blockIdx.x];
  const int f = P.snF[s], nc = P.snNc[s], m = P.snM[s];
  for (int k = 0; k < q; k++) {
    double *v = V + (int64_t)k * Vstride + P.Sp[s];
    const double *yk = y + (int64_t)k * P.n;
    for (int r = threadIdx.x; r < m; r += blockDim.x) v[r] = r < nc ? yk[f + r] : 0.0;
  }
  __syncthreads();
  for (int qq = P.chPtr[s]; qq < P.chPtr[s + 1]; qq++) {
    const int c = P.chList[qq];
    const int muc = P.snM[c] - P.snNc[c];
    const int *map = P.eaMap + P.eaPtr[c];
    for (int k = 0; k < q; k++) {
      double *v = V + (int64_t)k * Vstride + P.Sp[s];
      const double *tc = T + (int64_t)k * Tstride + P.snTOff[c];
      for (int a = threadIdx.x; a < muc; a += blockDim.x) v[map[a]] += tc[a];
    }
    __syncthreads();
  }
}

// ---- forward block tasks -----------------------------------------------------------------------------------------
// task: .x supernode, .y block, .z kind (0 diagonal, 1 below)
// One launch for the whole sweep: tasks are listed level by level (leaves first), so every wait below is on a task
// with an earlier ticket. The first diagonal task of a supernode waits for its children's pass-up vectors (their
// below tasks count themselves in done[]) and gathers its front vector; every below task counts itself when its
// part of the pass-up vector is written.
template <class TL>
__global__ void __launch_bounds__(256) k_fwd_blocks(const int4 *__restrict__ tasks, int ntasks, int *__restrict__ ticket,
                                                    DevPlan P, const int *__restrict__ blkOff,
                                                    const TL *__restrict__ Lx, double *__restrict__ y,
                                                    double *__restrict__ V, double *__restrict__ T,
                                                    int *__restrict__ flags, int epoch, int *__restrict__ done,
                                                    int q, int64_t Vstride, int64_t Tstride,
                                                    unsigned long long *status) {
  __shared__ int tk, waitOk;
  __shared__ double red[4][kSB];
  __shared__ double Lkk[kSB][kSB + 1];
  if (threadIdx.x == 0) tk = atomicAdd(ticket, 1);
  __syncthreads();
  if (tk >= ntasks) return;
  const int4 t = tasks[tk];
  const int s = t.x, blk = t.y, below = t.z;
  const int f = P.snF[s], nc = P.snNc[s], m = P.snM[s], mu = m - nc;
  const TL *Lp = Lx + P.snLxp[s];
  const int r0 = below ? nc + blk * kSB : blk * kSB;
  const int rows = below ? min(kSB, mu - blk * kSB) : min(kSB, nc - blk * kSB);
  const int ncols = below ? nc : blk * kSB;  // columns of L to the left of the diagonal block / all pivot columns
  const int tid = threadIdx.x, row = tid & (kSB - 1), part = tid >> 6;
  int *myflags = flags + blkOff[s];
  if (!below && blk == 0) {
    // children's pass-up vectors complete?
    for (int qq = P.chPtr[s]; qq < P.chPtr[s + 1]; qq++) {
      const int c = P.chList[qq];
      const int need = (P.snM[c] - P.snNc[c] + kSB - 1) / kSB;
      if (tid == 0) waitOk = wait_count(done + c, need, status, s);
      __syncthreads();
      if (!waitOk) return;
    }
    // gather v_s = [y(f .. f + nc); 0] + children's pass-up vectors (the reference's child order)
    for (int k = 0; k < q; k++) {
      double *v = V + (int64_t)k * Vstride + P.Sp[s];
      const double *yk = y + (int64_t)k * P.n;
      for (int r = tid; r < m; r += blockDim.x) v[r] = r < nc ? yk[f + r] : 0.0;
    }
    __syncthreads();
    for (int qq = P.chPtr[s]; qq < P.chPtr[s + 1]; qq++) {
      const int c = P.chList[qq];
      const int muc = P.snM[c] - P.snNc[c];
      const int *map = P.eaMap + P.eaPtr[c];
      for (int k = 0; k < q; k++) {
        double *v = V + (int64_t)k * Vstride + P.Sp[s];
        const double *tc = T + (int64_t)k * Tstride + P.snTOff[c];
        for (int a = tid; a < muc; a += blockDim.x) v[map[a]] += __ldcg(tc + a);
      }
      __syncthreads();
    }
  }
  for (int k = 0; k < q; k++) {
    const double *yk = y + (int64_t)k * P.n + f;
    double acc = 0.0;
    // row-block dot products over the columns of the blocks this one depends on, waiting for each block
    for (int cb = 0; cb * kSB < ncols; cb++) {
      if (k == 0) {
        if (tid == 0) waitOk = wait_flag(myflags + cb, epoch, status, s);
        __syncthreads();
        if (!waitOk) return;  // block-uniform
      }
      const int c1 = min(ncols, (cb + 1) * kSB);
      if (row < rows)
        for (int c = cb * kSB + part; c < c1; c += 4) acc += (double)Lp[(int64_t)c * m + r0 + row] * __ldcg(yk + c);
    }
    red[part][row] = acc;
    __syncthreads();
    if (tid < kSB) {
      double sum = (red[0][tid] + red[1][tid]) + (red[2][tid] + red[3][tid]);
      const double *vk = V + (int64_t)k * Vstride + P.Sp[s];
      red[0][tid] = tid < rows ? __ldcg(vk + r0 + tid) - sum : 0.0;
    }
    __syncthreads();
    if (below) {
      double *tk_out = T + (int64_t)k * Tstride + P.snTOff[s];
      if (tid < rows) tk_out[blk * kSB + tid] = red[0][tid];
    } else {
      // solve L_kk y_k = v_k with one warp: lane i owns rows i and i + 32
      if (k == 0) {
        for (int e = tid; e < rows * rows; e += blockDim.x) {
          int i = e % rows, j = e / rows;
          if (i >= j) Lkk[i][j] = (double)Lp[(int64_t)(r0 + j) * m + r0 + i];
        }
        __syncthreads();
      }
      if (tid < 32) {
        double v0 = red[0][tid], v1 = red[0][tid + 32];
        for (int j = 0; j < rows; j++) {
          double vj = __shfl_sync(0xffffffffu, j < 32 ? v0 : v1, j & 31);
          double yj = vj / Lkk[j][j];
          if (tid == (j & 31)) {
            if (j < 32) v0 = yj; else v1 = yj;
          }
          if (tid > j && tid < rows) v0 -= Lkk[tid][j] * yj;
          if (tid + 32 > j && tid + 32 < rows) v1 -= Lkk[tid + 32][j] * yj;
        }
        double *yo = y + (int64_t)k * P.n + f + r0;
        if (tid < rows) yo[tid] = v0;
        if (tid + 32 < rows) yo[tid + 32] = v1;
      }
      __syncthreads();
    }
  }
  __syncthreads();
  if (tid == 0) {
    __threadfence();
    if (below)
      atomicAdd(done + s, 1);
    else
      st_release(myflags + blk, epoch);
  }
}

// ---- backward block tasks ----------------------------------------------------------------------------------------
// task: .x supernode, .y column block (tasks of a supernode listed from the last block down)
template <class TL>
__global__ void __launch_bounds__(256) k_bwd_blocks(const int4 *__restrict__ tasks, int ntasks, int *__restrict__ ticket,
                                                    DevPlan P, const int *__restrict__ blkOff,
                                                    const TL *__restrict__ Lx, double *__restrict__ y,
                                                    int *__restrict__ flags, int epoch, int q,
                                                    unsigned long long *status) {
  __shared__ int tk, waitOk;
  __shared__ double red[8][kSB];
  __shared__ double Lkk[kSB][kSB + 1];
  if (threadIdx.x == 0) tk = atomicAdd(ticket, 1);
  __syncthreads();
  if (tk >= ntasks) return;
  const int4 t = tasks[tk];
  const int s = t.x, blk = t.y;
  const int f = P.snF[s], nc = P.snNc[s], m = P.snM[s];
  const TL *Lp = Lx + P.snLxp[s];
  const int *rowsOf = P.Si + P.Sp[s];
  const int c0 = blk * kSB, w = min(kSB, nc - c0), nb = (nc + kSB - 1) / kSB;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  int *myflags = flags + blkOff[s];
  // one launch for the whole sweep (levels top-down): the rows below this supernode are final once its parent's
  // first pivot block (the parent's last backward task) is
  const int par = P.snParent[s];
  if (par >= 0) {
    if (tid == 0) waitOk = wait_flag(flags + blkOff[par], epoch, status, s);
    __syncthreads();
    if (!waitOk) return;
  }
  for (int k = 0; k < q; k++) {
    double *yk = y + (int64_t)k * P.n;
    // each warp owns columns c0 + warp, c0 + warp + 8, ...; lanes walk the rows below the diagonal block
    double acc[8];
#pragma unroll
    for (int u = 0; u < 8; u++) acc[u] = 0.0;
    // rows of the supernode below its pivot columns: ancestors, final
    for (int r = nc + lane; r < m; r += 32) {
      const double xr = __ldcg(yk + rowsOf[r]);
#pragma unroll
      for (int u = 0; u < 8; u++) {
        const int c = warp + 8 * u;
        if (c < w) acc[u] += (double)Lp[(int64_t)(c0 + c) * m + r] * xr;
      }
    }
    // later pivot blocks of this supernode, as they become final
    for (int rb = nb - 1; rb > blk; rb--) {
      if (k == 0) {
        if (tid == 0) waitOk = wait_flag(myflags + rb, epoch, status, s);
        __syncthreads();
        if (!waitOk) return;  // block-uniform
      }
      const int rr1 = min(nc, (rb + 1) * kSB);
      for (int r = rb * kSB + lane; r < rr1; r += 32) {
        const double xr = __ldcg(yk + f + r);
#pragma unroll
        for (int u = 0; u < 8; u++) {
          const int c = warp + 8 * u;
          if (c < w) acc[u] += (double)Lp[(int64_t)(c0 + c) * m + r] * xr;
        }
      }
    }
#pragma unroll
    for (int u = 0; u < 8; u++) {
      double v = acc[u];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
      if (lane == 0) red[0][warp + 8 * u] = v;
    }
    if (k == 0) {
      for (int e = tid; e < w * w; e += blockDim.x) {
        int i = e % w, j = e / w;
        if (i >= j) Lkk[i][j] = (double)Lp[(int64_t)(c0 + j) * m + c0 + i];
      }
    }
    __syncthreads();
    // x_k = L_kk^-T (y_k - sum): upper-triangular solve with one warp, rows i and i + 32 per lane
    if (tid < 32) {
      double *yb = yk + f + c0;
      double w0 = tid < w ? yb[tid] - red[0][tid] : 0.0;
      double w1 = tid + 32 < w ? yb[tid + 32] - red[0][tid + 32] : 0.0;
      for (int j = w - 1; j >= 0; j--) {
        double wj = __shfl_sync(0xffffffffu, j < 32 ? w0 : w1, j & 31);
        double xj = wj / Lkk[j][j];
        if (tid == (j & 31)) {
          if (j < 32) w0 = xj; else w1 = xj;
        }
        if (tid < j) w0 -= Lkk[j][tid] * xj;
        if (tid + 32 < j) w1 -= Lkk[j][tid + 32] * xj;
      }
      if (tid < w) yb[tid] = w0;
      if (tid + 32 < w) yb[tid + 32] = w1;
    }
    __syncthreads();
  }
  if (tid == 0) {
    __threadfence();
    st_release(myflags + blk, epoch);
  }
}

void launch_fwd_gather(const int *sns, int count, const DevPlan &P, const double *y, double *V, const double *T, int q,
                       int64_t Vstride, int64_t Tstride, cudaStream_t st) {
  if (count > 0) k_fwd_gather<<<count, 256, 0, st>>>(sns, P, y, V, T, q, Vstride, Tstride);
}
template <class TL>
void launch_fwd_blocks(const int4 *tasks, int ntasks, int *ticket, const DevPlan &P, const int *blkOff,
                       const TL *Lx, double *y, double *V, double *T, int *flags, int epoch, int *done, int q,
                       int64_t Vstride, int64_t Tstride, unsigned long long *status, cudaStream_t st) {
  if (ntasks > 0)
    k_fwd_blocks<TL><<<ntasks, 256, 0, st>>>(tasks, ntasks, ticket, P, blkOff, Lx, y, V, T, flags, epoch, done, q,
                                             Vstride, Tstride, status);
}
template <class TL>
void launch_bwd_blocks(const int4 *tasks, int ntasks, int *ticket, const DevPlan &P, const int *blkOff,
                       const TL *Lx, double *y, int *flags, int epoch, int q, unsigned long long *status,
                       cudaStream_t st) {
  if (ntasks > 0)
    k_bwd_blocks<TL><<<ntasks, 256, 0, st>>>(tasks, ntasks, ticket, P, blkOff, Lx, y, flags, epoch, q, status);
}
template void launch_fwd_blocks<double>(const int4 *, int, int *, const DevPlan &, const int *, const double *,
                                        double *, double *, double *, int *, int, int *, int, int64_t, int64_t,
                                        unsigned long long *, cudaStream_t);
template void launch_fwd_blocks<float>(const int4 *, int, int *, const DevPlan &, const int *, const float *, double *,
                                       double *, double *, int *, int, int *, int, int64_t, int64_t,
                                       unsigned long long *, cudaStream_t);
template void launch_bwd_blocks<double>(const int4 *, int, int *, const DevPlan &, const int *, const double *,
                                        double *, int *, int, int, unsigned long long *, cudaStream_t);
template void launch_bwd_blocks<float>(const int4 *, int, int *, const DevPlan &, const int *, const float *, double *,
                                       int *, int, int, unsigned long long *, cudaStream_t);

}  // namespace amp
