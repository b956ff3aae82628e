// Mixed-precision trailing / update-block tiles on the 5th-generation tensor cores (tcgen05, sm_100a), 128 x 256, or
// 128 x 128 / 128 x 64 for the look-ahead's next group when it is two pivot blocks (one block) wide.
//
// C[i0:i0+128, j0:j0+256] -= A B^T in FP32, where A and B are rows of the factored pivot columns of a front (for
// LDL^T, A holds those rows times the pivots, L21 D) and the product runs as BF16x3: every FP32 value x is carried
// as hi = bf16(x), lo = bf16(x - hi) (split once, by the panel kernel, into the split buffers) and
// A B^T ~= Ahi Bhi^T + Ahi Blo^T + Alo Bhi^T with FP32 accumulation in tensor memory (the dropped Alo Blo^T term is
// ~2^-16 relative).
//
// Persistent, one CTA per SM, warp-specialised:
//   warp 0      TMA producer: per 64-column K chunk, 12 boxes of 64 rows x 64 columns (A and B, hi and lo) from the
//               front's 2D tensor maps into one of two 96 KB shared-memory stages (128-byte swizzle, zero fill past
//               the front's rows and pivot columns), completing on the stage's `full` barrier;
//   warp 1      MMA issuer: 4 K-steps x 3 UMMAs (M = 128, N = 256, K = 16) per chunk into one of two TMEM
//               accumulators (2 x 256 columns), `empty` commit per stage, `accFull` commit per tile;
//   warps 2-9   epilogue: 4 lane quadrants x 2 column halves; tcgen05.ld the accumulator, release it (`accEmpty`),
//               then subtract it from the FP32 front (masked to the task's rows, columns and the lower triangle).
// The epilogue of tile t overlaps the loads and MMAs of tile t + 1. Every wait is bounded: on time-out the waiting
// role raises a shared abort flag and a device-timeout status, the other roles see the flag and leave, and before
// the tensor memory is freed the producer waits (bounded) for its own loads and the MMA warp for its own MMAs.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "../host/plan.hpp"
#include "devplan.cuh"
#include "umma.cuh"

namespace amp {

namespace {
constexpr int kM = 128, kK = 64;
constexpr int kBox = 64;                                  // rows per TMA box (128 bytes of BF16)
constexpr uint32_t kBoxBytes = kBox * kK * 2;             // 8 KB
constexpr uint32_t kABytes = kM * kK * 2;                 // 16 KB (hi or lo)
template <int N>
constexpr uint32_t b_bytes() { return N * kK * 2; }  // 32 KB for N = 256 (hi or lo)
template <int N>
constexpr uint32_t stage_bytes() { return 2 * kABytes + 2 * b_bytes<N>(); }  // 96 KB for N = 256
constexpr int kStages = 2;
constexpr uint32_t kLbo = kBoxBytes;                      // between 64-row MN blocks
constexpr uint32_t kSbo = 8 * 128;                        // between groups of 8 K rows
constexpr uint32_t kKStep = 16 * 128;                     // one K16 step (2 groups of 8 K rows)
constexpr int kEpiPerQuad = 2;                           // epilogue warps per TMEM lane quadrant
constexpr int kEpiWarps = 4 * kEpiPerQuad;
constexpr int kThreads = 32 * (2 + kEpiWarps);
constexpr long long kMxSpin = 1ll << 22;                  // default bound of a role's wait: ~0.5 s with back-off
}  // namespace

template <int N>
constexpr int mixed_smem() { return kStages * stage_bytes<N>() + 1024; }

struct MxShared {
  uint64_t full[kStages], empty[kStages], accFull[2], accEmpty[2], drain;
  uint32_t tmem;
  int abort;
};

// Bounded wait (at most `limit` polls) that also gives up when another role raised the abort flag. false: aborted
// or timed out. The drains before the tensor memory is freed keep their own bound (umma::mbar_wait), whatever limit.
__device__ __forceinline__ bool mx_wait(uint64_t *bar, uint32_t parity, MxShared &sh, unsigned long long *status,
                                        long long limit) {
  for (long long i = 0; i < limit; i++) {
    if (umma::mbar_try_wait(bar, parity)) return true;
    if (*(volatile int *)&sh.abort) return false;
    if (i > 64) __nanosleep(128);
  }
  *(volatile int *)&sh.abort = 1;
  atomicMin(status, status_word(0x7fffffff, 3, 0));
  return false;
}

// N: tile columns, 256 (the general tiles), or 128 / 64 (the next group of the look-ahead when it is that wide)
template <int N>
__global__ void __launch_bounds__(kThreads, 1) k_update_mx(const MixTask *__restrict__ tasks, int ntasks,
                                                           const CUtensorMap *__restrict__ maps,
                                                           float *__restrict__ L32, float *__restrict__ U32,
                                                           unsigned long long *status, long long spin) {
  constexpr uint32_t kBBytes = b_bytes<N>(), kStageBytes = stage_bytes<N>(), kTmemCols = 2 * N;
  constexpr uint32_t kIdesc = umma::idesc_bf16_f32_mn(kM, N);
  constexpr int kN = N;
  extern __shared__ __align__(1024) uint8_t smem_mx[];
  __shared__ MxShared sh;
  if (*(volatile unsigned long long *)status != kStatusOk) return;
  if ((int)blockIdx.x >= ntasks) return;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint8_t *stages = smem_mx + ((1024 - (umma::smem_u32(smem_mx) & 1023)) & 1023);  // 1 KB aligned (swizzle atom)
  if (warp == 1) umma::tmem_alloc(&sh.tmem, kTmemCols);
  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; s++) {
      umma::mbar_init(&sh.full[s], 1);
      umma::mbar_init(&sh.empty[s], 1);
    }
    for (int a = 0; a < 2; a++) {
      umma::mbar_init(&sh.accFull[a], 1);
      umma::mbar_init(&sh.accEmpty[a], kEpiWarps);
    }
    umma::mbar_init(&sh.drain, 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    sh.abort = 0;
  }
  umma::tc_fence_before();
  __syncthreads();
  umma::tc_fence_after();
  const uint32_t tmem = sh.tmem;

  if (warp == 0) {
    if (lane == 0) {  // ---- TMA producer
      int it = 0;
      for (int t = blockIdx.x; t < ntasks; t += gridDim.x) {
        const MixTask tk = tasks[t];
        const CUtensorMap *ahi = maps + 4 * tk.s, *alo = ahi + 1, *bhi = ahi + 2, *blo = ahi + 3;
        const int nch = (tk.w + kK - 1) / kK;
        bool ok = true;
        for (int c = 0; c < nch; c++, it++) {
          const int s = it % kStages;
          const uint32_t n = it / kStages;
          if (!mx_wait(&sh.empty[s], (n & 1) ^ 1, sh, status, spin)) {
            ok = false;
            break;
          }
          uint8_t *st = stages + s * kStageBytes;
          umma::mbar_arrive_expect_tx(&sh.full[s], kStageBytes);
          const int kc = tk.c0 + c * kK;
#pragma unroll
          for (int b = 0; b < kM / kBox; b++) {
            umma::tma_load_2d(st + b * kBoxBytes, ahi, tk.i0 + kBox * b, kc, &sh.full[s]);
            umma::tma_load_2d(st + kABytes + b * kBoxBytes, alo, tk.i0 + kBox * b, kc, &sh.full[s]);
          }
#pragma unroll
          for (int b = 0; b < kN / kBox; b++) {
            umma::tma_load_2d(st + 2 * kABytes + b * kBoxBytes, bhi, tk.j0 + kBox * b, kc, &sh.full[s]);
            umma::tma_load_2d(st + 2 * kABytes + kBBytes + b * kBoxBytes, blo, tk.j0 + kBox * b, kc, &sh.full[s]);
          }
        }
        if (!ok) break;
      }
      // let the last loads land before the CTA can exit (bounded, also after an abort)
      for (int q = it > kStages ? it - kStages : 0; q < it; q++)
        umma::mbar_wait(&sh.full[q % kStages], (q / kStages) & 1);
    }
    __syncwarp();
  } else if (warp == 1) {
    if (lane == 0) {  // ---- MMA issuer
      int it = 0, tl = 0;
      for (int t = blockIdx.x; t < ntasks; t += gridDim.x, tl++) {
        const MixTask tk = tasks[t];
        const int nch = (tk.w + kK - 1) / kK;
        const int a = tl & 1;
        if (!mx_wait(&sh.accEmpty[a], ((tl >> 1) & 1) ^ 1, sh, status, spin)) break;
        umma::tc_fence_after();
        const uint32_t d = tmem + a * kN;
        bool ok = true;
        for (int c = 0; c < nch; c++, it++) {
          const int s = it % kStages;
          if (!mx_wait(&sh.full[s], (it / kStages) & 1, sh, status, spin)) {
            ok = false;
            break;
          }
          umma::tc_fence_after();
          const uint32_t sa = umma::smem_u32(stages + s * kStageBytes);
          const int kw = min(kK, tk.w - c * kK);
          for (int kk = 0; kk * 16 < kw; kk++) {
            const uint64_t ahi = umma::smem_desc_sw128(sa + kk * kKStep, kLbo, kSbo);
            const uint64_t alo = umma::smem_desc_sw128(sa + kABytes + kk * kKStep, kLbo, kSbo);
            const uint64_t bhi = umma::smem_desc_sw128(sa + 2 * kABytes + kk * kKStep, kLbo, kSbo);
            const uint64_t blo = umma::smem_desc_sw128(sa + 2 * kABytes + kBBytes + kk * kKStep, kLbo, kSbo);
            umma::mma_bf16(d, ahi, bhi, kIdesc, c > 0 || kk > 0);
            umma::mma_bf16(d, ahi, blo, kIdesc, true);
            umma::mma_bf16(d, alo, bhi, kIdesc, true);
          }
          umma::mma_commit(&sh.empty[s]);  // the stage is free once these MMAs have read it
        }
        if (!ok) break;
        umma::mma_commit(&sh.accFull[a]);  // accumulator complete
      }
      umma::mma_commit(&sh.drain);  // all MMAs of this CTA done before the tensor memory is freed
      umma::mbar_wait(&sh.drain, 0);
    }
    __syncwarp();
  } else {  // ---- epilogue: quadrant q of the TMEM lanes (rows), column quarter h
    const int ew = warp - 2, q = warp & 3, h = ew >> 2;
    int tl = 0;
    for (int t = blockIdx.x; t < ntasks; t += gridDim.x, tl++) {
      const MixTask tk = tasks[t];
      const int a = tl & 1;
      bool ok = true;
      if (lane == 0) ok = mx_wait(&sh.accFull[a], (tl >> 1) & 1, sh, status, spin);
      if (!__shfl_sync(0xffffffffu, ok ? 1 : 0, 0)) break;
      umma::tc_fence_after();
      const int i = tk.i0 + 32 * q + lane, m = tk.m, nc = tk.nc, mu = m - nc;
      const bool rowok = i >= tk.ilo && i < m;
      float *Lp = L32 + tk.lp;
      float *Up = tk.up >= 0 ? U32 + tk.up : Lp;
      constexpr int kChunks = kN / kEpiPerQuad / 32;
#pragma unroll 1
      for (int cc = 0; cc < kChunks; cc++) {
        const int col0 = h * (kN / kEpiPerQuad) + cc * 32;
        float v[32];
        umma::tmem_ld32(tmem + a * kN + ((uint32_t)(32 * q) << 16) + col0, v);
        if (cc == kChunks - 1) {  // accumulator fully read: hand it back to the MMA warp
          umma::tc_fence_before();
          __syncwarp();
          if (lane == 0) umma::mbar_arrive(&sh.accEmpty[a]);
        }
        if (!rowok) continue;
        const int j0 = tk.j0 + col0;
        const int jl = max(tk.jlo, j0), jh = min(min(tk.jend, i + 1), j0 + 32);  // columns of this row to update
        if (jl >= jh) continue;
        const uint32_t msk = (jh - j0 == 32 ? 0xffffffffu : ((1u << (jh - j0)) - 1)) & ~((1u << (jl - j0)) - 1);
        auto addr = [&](int x) {
          const int j = j0 + x;
          return j < nc ? Lp + (int64_t)j * m + i : Up + (int64_t)(j - nc) * mu + (i - nc);
        };
        float c[32];
#pragma unroll
        for (int x = 0; x < 32; x++) c[x] = (msk >> x) & 1 ? *addr(x) : 0.f;
#pragma unroll
        for (int x = 0; x < 32; x++)
          if ((msk >> x) & 1) *addr(x) = c[x] - v[x];
      }
    }
  }
  umma::tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    umma::tc_fence_after();
    umma::tmem_dealloc(tmem, kTmemCols);
  }
}

cudaError_t init_mixed_attributes() {
  cudaError_t e = cudaFuncSetAttribute(k_update_mx<256>, cudaFuncAttributeMaxDynamicSharedMemorySize, mixed_smem<256>());
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_update_mx<128>, cudaFuncAttributeMaxDynamicSharedMemorySize, mixed_smem<128>());
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_update_mx<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, mixed_smem<64>());
  return e;
}

void launch_update_mx(const MixTask *tasks, int64_t ntasks, const CUtensorMap *maps, float *L32, float *U32,
                      unsigned long long *status, int num_sms, cudaStream_t st, int width, long long spin) {
  if (ntasks <= 0) return;
  const int grid = (int)(ntasks < num_sms ? ntasks : num_sms);
  if (spin <= 0) spin = kMxSpin;
  if (width == 64)
    k_update_mx<64><<<grid, kThreads, mixed_smem<64>(), st>>>(tasks, (int)ntasks, maps, L32, U32, status, spin);
  else if (width == 128)
    k_update_mx<128><<<grid, kThreads, mixed_smem<128>(), st>>>(tasks, (int)ntasks, maps, L32, U32, status, spin);
  else
    k_update_mx<256><<<grid, kThreads, mixed_smem<256>(), st>>>(tasks, (int)ntasks, maps, L32, U32, status, spin);
}

}  // namespace amp
