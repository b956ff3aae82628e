// Mixed-precision trailing / update-block tiles on the 5th-generation tensor cores (tcgen05, sm_100a).
//
// C[i0:i0+128, j0:j0+256] -= A B^T in FP32, where A and B are rows of the factored pivot columns of a front and the
// product runs as BF16x3: every FP32 value x is carried as hi = bf16(x), lo = bf16(x - hi) (split once, by the panel
// kernel, into the split buffers) and A B^T ~= Ahi Bhi^T + Ahi Blo^T + Alo Bhi^T with FP32 accumulation in tensor
// memory (the dropped Alo Blo^T term is ~2^-16 relative).
//
// One CTA per SM (persistent), 4 warps. Per (tile, 64-column K chunk) item all threads stream the chunk's hi/lo
// operands into one of two shared-memory stages with 16-byte cp.async (MN-major, no-swizzle UMMA layout); thread 0
// then issues 4 K-steps x 3 UMMAs (M = 128, N = 256, K = 16) and commits them to the stage's mbarrier, so the next
// chunk loads while the tensor core works. After a tile's last chunk every warp reads its 32 accumulator lanes from
// tensor memory (tcgen05.ld) and updates its 32 rows of C. Every mbarrier wait is bounded; on time-out the kernel
// records a device-timeout status and leaves (after waiting, bounded, for its own MMAs), freeing its tensor memory.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "../host/plan.hpp"
#include "devplan.cuh"
#include "umma.cuh"

namespace amp {

namespace {
constexpr int kM = 128, kN = 256, kK = 64;
// Layout per 16-column K step: [K step][MN core block][K half][8 rows x 16 bytes]. The two K halves of an MN block
// are adjacent (LBO = 128 B) and MN blocks are 256 B apart (SBO), so one MMA's operand stays inside its K-step slab.
constexpr uint32_t kLbo = 128, kSbo = 256;
constexpr uint32_t kStepA = (kM / 8) * 256, kStepB = (kN / 8) * 256;  // bytes per K step
constexpr int kBytesA = kM * kK * 2, kBytesB = kN * kK * 2;          // one of hi / lo
constexpr int kStageBytes = 2 * kBytesA + 2 * kBytesB;              // 96 KB
constexpr uint32_t kIdesc = umma::idesc_bf16_f32_mn(kM, kN);
}  // namespace

constexpr int kMixedSmem = 2 * kStageBytes + 1024;

__device__ __forceinline__ void mx_fill(const MixTask &t, int chunk, const __nv_bfloat16 *Shi,
                                        const __nv_bfloat16 *Slo, uint8_t *stage) {
  const int kc = t.c0 + chunk * kK, kw = min(kK, t.w - chunk * kK);
  const uint32_t sa = umma::smem_u32(stage);
  const int tid = threadIdx.x;
  // A: 16 row-units x 64 columns = 1024 16-byte units per hi / lo; unit u -> (mb = u % 16, k = u / 16)
#pragma unroll 2
  for (int u = tid; u < (kM / 8) * kK; u += 128) {
    const int mb = u & 15, k = u >> 4, r = t.i0 + 8 * mb;
    const bool ok = k < kw && r < t.ld;
    const int64_t g = t.sp + (int64_t)(kc + (ok ? k : 0)) * t.ld + (ok ? r : 0);
    const uint32_t off = (k >> 4) * kStepA + mb * kSbo + ((k >> 3) & 1) * kLbo + (k & 7) * 16;
    umma::cp_async16(sa + off, Shi + g, ok);
    umma::cp_async16(sa + kBytesA + off, Slo + g, ok);
  }
  // B: 32 row-units x 64 columns
#pragma unroll 2
  for (int u = tid; u < (kN / 8) * kK; u += 128) {
    const int nb = u & 31, k = u >> 5, r = t.j0 + 8 * nb;
    const bool ok = k < kw && r < t.ld;
    const int64_t g = t.sp + (int64_t)(kc + (ok ? k : 0)) * t.ld + (ok ? r : 0);
    const uint32_t off = (k >> 4) * kStepB + nb * kSbo + ((k >> 3) & 1) * kLbo + (k & 7) * 16;
    umma::cp_async16(sa + 2 * kBytesA + off, Shi + g, ok);
    umma::cp_async16(sa + 2 * kBytesA + kBytesB + off, Slo + g, ok);
  }
  asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
}

__global__ void __launch_bounds__(128, 1) k_update_mx(const MixTask *__restrict__ tasks, int ntasks,
                                                      float *__restrict__ L32, float *__restrict__ U32,
                                                      const __nv_bfloat16 *__restrict__ Shi,
                                                      const __nv_bfloat16 *__restrict__ Slo,
                                                      unsigned long long *status) {
  extern __shared__ __align__(1024) uint8_t smem_mx[];
  __shared__ uint64_t bar[2];
  __shared__ uint32_t tmem_slot;
  __shared__ int abort_flag;
  if (*(volatile unsigned long long *)status != kStatusOk) return;
  if ((int)blockIdx.x >= ntasks) return;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  uint8_t *stages = smem_mx + ((1024 - (umma::smem_u32(smem_mx) & 1023)) & 1023);  // 1 KB aligned
  if (warp == 0) umma::tmem_alloc(&tmem_slot, kN);
  if (tid == 0) {
    umma::mbar_init(&bar[0], 1);
    umma::mbar_init(&bar[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    abort_flag = 0;
  }
  umma::tc_fence_before();
  __syncthreads();
  umma::tc_fence_after();
  const uint32_t tmem = tmem_slot;
  uint32_t phase[2] = {0, 0};
  bool pending[2] = {false, false};
  int item = 0;
  bool failedWait = false;  // block-uniform
  auto consume = [&](int s) -> bool {  // wait for the MMAs committed on stage s (bounded)
    if (!pending[s]) return true;
    const bool ok = umma::mbar_wait(&bar[s], phase[s]);
    phase[s] ^= 1;
    pending[s] = false;
    return ok;
  };
  for (int t = blockIdx.x; t < ntasks && !failedWait; t += gridDim.x) {
    const MixTask tk = tasks[t];
    const int nch = (tk.w + kK - 1) / kK;
    for (int c = 0; c < nch; c++, item++) {
      const int s = item & 1;
      if (__syncthreads_or(!consume(s))) {  // block-uniform decision
        failedWait = true;
        break;
      }
      uint8_t *st = stages + s * kStageBytes;
      mx_fill(tk, c, Shi, Slo, st);
      umma::fence_async_smem();
      umma::tc_fence_before();
      __syncthreads();
      if (tid == 0) {
        umma::tc_fence_after();
        const uint32_t sa = umma::smem_u32(st);
        const int kw = min(kK, tk.w - c * kK);
        for (int kk = 0; kk * 16 < kw; kk++) {
          const uint32_t ao = kk * kStepA, bo = kk * kStepB;
          const uint64_t ahi = umma::smem_desc(sa + ao, kLbo, kSbo);
          const uint64_t alo = umma::smem_desc(sa + kBytesA + ao, kLbo, kSbo);
          const uint64_t bhi = umma::smem_desc(sa + 2 * kBytesA + bo, kLbo, kSbo);
          const uint64_t blo = umma::smem_desc(sa + 2 * kBytesA + kBytesB + bo, kLbo, kSbo);
          umma::mma_bf16(tmem, ahi, bhi, kIdesc, c > 0 || kk > 0);
          umma::mma_bf16(tmem, ahi, blo, kIdesc, true);
          umma::mma_bf16(tmem, alo, bhi, kIdesc, true);
        }
        umma::mma_commit(&bar[s]);
      }
      pending[s] = true;
    }
    if (failedWait) break;
    // all MMAs of the tile: the last commit covers every earlier one
    const int last = (item - 1) & 1;
    const bool ok1 = consume(last), ok2 = consume(last ^ 1);
    if (__syncthreads_or(!(ok1 && ok2))) {
      failedWait = true;
      break;
    }
    umma::tc_fence_after();
    // epilogue: warp w owns accumulator lanes (tile rows) 32w .. 32w + 31
    const int i = tk.i0 + 32 * warp + lane, m = tk.m, nc = tk.nc, mu = m - nc;
    float *Lp = L32 + tk.lp;
    float *Up = tk.up >= 0 ? U32 + tk.up : Lp;
    const bool rowok = i >= tk.ilo && i < m;
    for (int cc = 0; cc < kN / 32; cc++) {
      float v[32];
      umma::tmem_ld32(tmem + ((uint32_t)(32 * warp) << 16) + cc * 32, v);
      if (!rowok) continue;
#pragma unroll
      for (int x = 0; x < 32; x++) {
        const int j = tk.j0 + cc * 32 + x;
        if (j >= tk.jlo && j < tk.jend && i >= j) {
          float *p = j < nc ? Lp + (int64_t)j * m + i : Up + (int64_t)(j - nc) * mu + (i - nc);
          *p -= v[x];
        }
      }
    }
    umma::tc_fence_before();
    __syncthreads();  // accumulators read before the next tile's first MMA overwrites them
  }
  if (failedWait) {
    if (tid == 0) atomicMin(status, status_word(0x7fffffff, 3, 0));
    consume(0);  // bounded: let our own MMAs finish before freeing tensor memory
    consume(1);
  }
  umma::tc_fence_before();
  __syncthreads();
  if (warp == 0) umma::tmem_dealloc(tmem, kN);
}

void init_mixed_attributes() {
  cudaFuncSetAttribute(k_update_mx, cudaFuncAttributeMaxDynamicSharedMemorySize, kMixedSmem);
}

void launch_update_mx(const MixTask *tasks, int64_t ntasks, float *L32, float *U32, const __nv_bfloat16 *Shi,
                      const __nv_bfloat16 *Slo, unsigned long long *status, int num_sms, cudaStream_t st) {
  if (ntasks <= 0) return;
  const int grid = (int)(ntasks < num_sms ? ntasks : num_sms);
  k_update_mx<<<grid, 128, kMixedSmem, st>>>(tasks, (int)ntasks, L32, U32, Shi, Slo, status);
}

}  // namespace amp
