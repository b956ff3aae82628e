// C ABI of libampsolve.so (include/ampsolve.h): plan / factor handles, device memory, and the orchestration of the
// kernels on one CUDA stream per factor.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "../../include/ampsolve.h"
#include "cuda/launch.hpp"
#include "host/plan.hpp"
#include "host/symbolic.hpp"

namespace amp {
int launch_assemble_values(int kind, int64_t ne, const int *conn, const double *coords, const double *coef, double *Ke,
                           int64_t nnz, const int64_t *gptr, const uint32_t *gidx, double *values, cudaStream_t st);
void launch_matvec(int n, const int *rowptr, const int *colidx, const double *val, const double *x, double *y, int q,
                   cudaStream_t st);
void launch_residual(int n, const int *rowptr, const int *colidx, const double *val, const double *x, const double *b,
                     double *r, double *norms, int q, cudaStream_t st);
void launch_axpy(double *x, const double *dx, int64_t len, cudaStream_t st);
int launch_dots(const double *V, int nv, int64_t n, const double *w, double *partial, double *out, cudaStream_t st);
void launch_gs_update(double *w, const double *V, const double *h, int nv, int64_t n, cudaStream_t st);
void launch_combine_add(double *x, const double *Z, const double *y, int nv, int64_t n, cudaStream_t st);
void launch_scale_to(double *v, const double *w, double a, int64_t n, cudaStream_t st);
void launch_scale_by_norm(double *v, const double *w, const double *norm2, int64_t n, cudaStream_t st);
void launch_sub_from(double *r, const double *b, const double *y, int64_t n, cudaStream_t st);
int dot_partials();
}  // namespace amp

namespace {

thread_local std::string g_err;

int fail(int code, const std::string &msg) {
  g_err = msg;
  return code;
}

struct CudaError {
  int code;
};

void ck(cudaError_t e, const char *what) {
  if (e != cudaSuccess) {
    g_err = std::string(what) + ": " + cudaGetErrorString(e);
    throw CudaError{e == cudaErrorMemoryAllocation ? AMP_OOM : AMP_CUDA_ERROR};
  }
}

// Device buffer list owned by a handle.
struct DevMem {
  std::vector<void *> ptrs;
  int64_t bytes = 0;
  template <class T>
  T *alloc(size_t count) {
    void *p = nullptr;
    size_t b = sizeof(T) * (count ? count : 1);
    ck(cudaMalloc(&p, b), "cudaMalloc");
    ptrs.push_back(p);
    bytes += (int64_t)b;
    return (T *)p;
  }
  template <class T>
  T *upload(const std::vector<T> &v) {
    T *p = alloc<T>(v.size());
    if (!v.empty()) ck(cudaMemcpy(p, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice), "cudaMemcpy H2D");
    return p;
  }
  void release() {
    for (void *p : ptrs) cudaFree(p);
    ptrs.clear();
    bytes = 0;
  }
  DevMem() = default;
  DevMem(const DevMem &) = delete;
  DevMem &operator=(const DevMem &) = delete;
  ~DevMem() { release(); }
};

}  // namespace

namespace amp {
void set_last_error(const std::string &msg) { g_err = msg; }
}  // namespace amp

namespace {
// elements of the diagonal-block inverses (none for an empty pattern, whose plan has no per-block arrays)
// chain-matrix slots: nb - 1 per supernode with nb diagonal blocks, 64 x 64 each
size_t chain_elems(const amp::Plan &P) { return (size_t)std::max(0, P.nflags - P.nsuper) * 64 * 64; }

int64_t inv_elems(const amp::Plan &P) { return P.invOff.empty() ? 0 : P.invOff[P.nflags]; }

// TMA descriptors of the BF16 split columns, two per supernode that has mixed-precision update tiles (hi, lo): the
// front's m x nc column-major block (ld = round_up(m, 8)) as a 2D tensor {rows, columns}, 64 x 64 boxes with the
// 128-byte swizzle; reads past m rows or nc columns return zeros, which is how partial tiles and K chunks are padded.
// Four per supernode: the A operand (hi, lo) and the B operand (hi, lo); for Cholesky A and B are the same columns,
// for LDL^T A is the split of L21 D and B the split of L21.
std::vector<CUtensorMap> split_tensor_maps(const amp::Plan &P, const __nv_bfloat16 *Ahi, const __nv_bfloat16 *Alo,
                                           const __nv_bfloat16 *Bhi, const __nv_bfloat16 *Blo) {
  using Encode = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                              const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                              CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
  static Encode encode = nullptr;
  if (!encode) {
    void *fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    ck(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q), "cudaGetDriverEntryPoint");
    if (!fn || q != cudaDriverEntryPointSuccess) throw std::runtime_error("cuTensorMapEncodeTiled not available");
    encode = (Encode)fn;
  }
  std::vector<char> need(P.nsuper, 0);
  for (const auto *v : {&P.mixTiles, &P.mixUTasks})
    for (const amp::MixTask &t : *v) need[t.s] = 1;
  std::vector<CUtensorMap> maps(4 * (size_t)std::max(1, P.nsuper));
  std::memset(maps.data(), 0, sizeof(CUtensorMap) * maps.size());
  for (int s = 0; s < P.nsuper; s++) {
    if (!need[s]) continue;
    const int m = P.snM[s], nc = P.snNc[s], ld = (m + 7) & ~7;
    const cuuint64_t dims[2] = {(cuuint64_t)m, (cuuint64_t)nc};
    const cuuint64_t strides[1] = {(cuuint64_t)ld * 2};
    const cuuint32_t box[2] = {64, 64}, estr[2] = {1, 1};
    const __nv_bfloat16 *bases[4] = {Ahi, Alo, Bhi, Blo};
    for (int h = 0; h < 4; h++) {
      const __nv_bfloat16 *base = bases[h] + P.snSp[s];
      CUresult r = encode(&maps[4 * s + h], CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, (void *)base, dims, strides, box, estr,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
      if (r != CUDA_SUCCESS)
        throw std::runtime_error("cuTensorMapEncodeTiled failed for supernode " + std::to_string(s) + " (error " +
                                 std::to_string((int)r) + ")");
    }
  }
  return maps;
}
}  // namespace

constexpr int kSlices = 4;  // vector slices of the multi-vector sweeps: multi_max_vectors() / 16

struct amp_plan_s {
  amp::Symbolic S;
  amp::Plan P;
  std::string key;
  int device = 0;
  DevMem mem;
  amp::DevPlan dp{};
  amp::AsmTask *dAsm = nullptr;
  amp::ChildRange *dAsmCh = nullptr;
  amp::GroupItem *dGroupItems = nullptr;
  amp::StripTask *dStrips = nullptr;
  amp::TileTask *dTile = nullptr, *dUTile = nullptr;
  amp::MixTask *dMixTile = nullptr, *dMixU = nullptr;
  int4 *dFwdTasks = nullptr, *dBwdTasks = nullptr, *dBwdAll = nullptr;
  int4 *dFwdTasks1 = nullptr;  // the one-vector forward's list (with whole-supernode tasks)
  // the multi-vector lists with every block task expanded into ns vector slices, built on first use (index ns - 1)
  int4 *dFwdSl[kSlices] = {}, *dBwdSl[kSlices] = {};
  int nFwdSl[kSlices] = {}, nBwdSl[kSlices] = {};
  bool wideSl[kSlices] = {};  // the list holds all-vector tasks (.w = -1)
  std::mutex slMu;
  int *dTinySn = nullptr, *dSmallSn = nullptr;  // small fronts per level (whole fronts by one warp / one CTA)
  int2 *dChain = nullptr;                        // chain-matrix tasks {s, b}
  int *dInvBlocks = nullptr;                     // diagonal blocks whose inverses the solves use
  int *dRowptr = nullptr, *dColidx = nullptr;
  std::vector<int> rowptr, colidx;  // host copy of the pattern (uploaded with the schedule)
  bool uploaded = false;
  // the dense schedule of every front, for complex-symmetric factors (built and uploaded by the first of them)
  amp::DenseSched cx;
  bool cxUploaded = false;
  amp::AsmTask *dCxAsm = nullptr;
  amp::ChildRange *dCxAsmCh = nullptr;
  amp::GroupItem *dCxItems = nullptr;
  amp::StripTask *dCxStrips = nullptr;
  amp::TileTask *dCxTiles = nullptr, *dCxU = nullptr;
  ~amp_plan_s() { mem.release(); }
};

// mesh and element-slot gather map of the on-device assembly
struct amp_assembly_s {
  int kind = 0, device = 0, ncoef = 1, nd = 3;
  int64_t nelem = 0, nnz = 0;
  DevMem mem;
  int *dConn = nullptr;
  double *dCoords = nullptr, *dKe = nullptr, *dCoef = nullptr, *dValues = nullptr;
  int64_t *dGptr = nullptr;
  uint32_t *dGidx = nullptr;
};

struct amp_factor_s {
  amp_plan *plan = nullptr;
  int kind = AMP_CHOLESKY, precision = AMP_FP64;
  bool bk = false;  // LDL^T with Bunch-Kaufman pivots inside each pivot block (amp_factor_opts kind AMP_LDLT_BK)
  cudaStream_t stream = nullptr;
  cudaStream_t side = nullptr;                      // look-ahead: part B of the panel steps' updates
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  cudaEvent_t evPanel = nullptr, evSide = nullptr;  // look-ahead ordering between the two streams
  DevMem mem;
  double *dLx = nullptr, *dU = nullptr, *dD = nullptr, *dValues = nullptr;
  float *dL32 = nullptr, *dU32 = nullptr;           // mixed precision: FP32 factor and update arena
  double *dW = nullptr;                             // LDL^T: L21 D of every front (the update's A operand)
  double *dScal = nullptr;                          // LDL^T: pivotTol, tau
  int *dCounts = nullptr;                           // LDL^T: nNeg, nPerturbed
  double *dDoff = nullptr;                          // Bunch-Kaufman: D(j + 1, j) of each 2 x 2 pivot (else 0)
  int *dPiv = nullptr;                              // Bunch-Kaufman: pivot order inside each 64-column block
  double *dInv = nullptr;                           // inverses of the 64-column diagonal blocks (FP64 factor)
  float *dInv32 = nullptr;                          // the same for the FP32 factor
  double *dMch = nullptr, *dGch = nullptr;          // chain matrices of consecutive diagonal blocks (FP64 factor)
  float *dMch32 = nullptr, *dGch32 = nullptr;       // the same for the FP32 factor
  __nv_bfloat16 *dShi = nullptr, *dSlo = nullptr;   // BF16 split columns of the factored pivot blocks
  __nv_bfloat16 *dWhi = nullptr, *dWlo = nullptr;   // mixed LDL^T: BF16 split of L21 D
  CUtensorMap *dMaps = nullptr;                     // per supernode: TMA descriptors of the split A and B operands
  unsigned long long *dStatus = nullptr;
  int *dGroupFlags = nullptr;  // group panels: flags of every item, then the ticket counter of every group step
  long long waitSpins = 0;  // bound of the device waits in polls (0 = the kernels' defaults)
  bool ok = false, hasValues = false;
  // profiling: events around every launch while enabled
  bool profiling = false;
  struct Rec {
    int kind;
    cudaEvent_t a, b;
    double flops, bytes;
    int kernels;  // kernel launches between a and b
  };
  std::vector<Rec> recs;
  std::vector<cudaEvent_t> evPool;
  size_t evUsed = 0;
  // the factorization sequence captured once, replayed afterwards
  cudaGraphExec_t factorGraph = nullptr;
  // solve workspace (grown on demand)
  DevMem smem;
  int qcap = 0;
  double *dY = nullptr, *dT = nullptr, *dB = nullptr, *dX = nullptr, *dR = nullptr, *dDX = nullptr,
         *dNorms = nullptr;
  int *dFlags = nullptr, *dTickets = nullptr;  // solve block ready flags (epoch-stamped) and per-launch tickets
  unsigned long long *dHand = nullptr;          // chain hand-off of consecutive diagonal blocks (epoch-tagged words)
  int *dDone = nullptr;                         // forward: finished below tasks per supernode
  DevMem gmem;                                  // GMRES workspace (Krylov and preconditioned bases), grown on demand
  int gmresCap = 0;
  double *gV = nullptr, *gZ = nullptr, *gR = nullptr, *gW = nullptr, *gX = nullptr, *gB = nullptr, *gPart = nullptr,
         *gH = nullptr;
  unsigned long long *dSolveStatus = nullptr;
  int solveEpoch = 0;
  // refinement row groups (independent diagonal blocks): group id per row, or none
  int ngroups = 0;
  int *dRowGroup = nullptr;
  double *dGroupNorms = nullptr;  // 2 x groups x multi_max_vectors()
  DevMem groupMem;
  // complex-symmetric LDL^T (kind AMP_LDLT_COMPLEX): factor, update arena, L21 D, pivots, values, solve vectors
  amp::cplx *dLc = nullptr, *dUc = nullptr, *dWc = nullptr, *dDc = nullptr, *dValC = nullptr;
  amp::cplx *dYc = nullptr, *dBc = nullptr, *dXc = nullptr, *dRc = nullptr, *dDXc = nullptr;
  double *dBr = nullptr, *dBi = nullptr, *dXr = nullptr, *dXi = nullptr, *dNormsC = nullptr;
  int *dCxFlags = nullptr;
  // shift-invert eigen operator: M's values on the pattern; Krylov workspace (grown on demand)
  double *dMass = nullptr;
  DevMem massMem, eigMem;
  int64_t eigCap = 0;
  ~amp_factor_s() {
    eigMem.release();
    massMem.release();
    if (factorGraph) cudaGraphExecDestroy(factorGraph);
    for (auto e : evPool) cudaEventDestroy(e);
    smem.release();
    groupMem.release();
    mem.release();
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (evPanel) cudaEventDestroy(evPanel);
    if (evSide) cudaEventDestroy(evSide);
    if (side) cudaStreamDestroy(side);
    if (stream) cudaStreamDestroy(stream);
  }
};

namespace {

void upload_plan(amp_plan *pl) {
  const amp::Plan &P = pl->P;
  DevMem &m = pl->mem;
  amp::DevPlan &d = pl->dp;
  d.n = P.n;
  d.spin = amp::kSpinLimit;
  d.nsuper = P.nsuper;
  d.maxFront = P.maxFront;
  if (P.nsuper == 0) return;
  d.snF = m.upload(P.snF);
  d.snNc = m.upload(P.snNc);
  d.snM = m.upload(P.snM);
  d.snParent = m.upload(P.snParent);
  d.snLxp = m.upload(P.snLxp);
  d.snUoff = m.upload(P.snUoff);
  d.snTOff = m.upload(P.snTOff);
  d.snSp = m.upload(P.snSp);
  d.chPtr = m.upload(P.chPtr);
  d.chList = m.upload(P.chList);
  d.asmColPtr = m.upload(P.asmColPtr);
  d.asmDst = m.upload(P.asmDst);
  d.asmSrc = m.upload(P.asmSrc);
  d.eaPtr = m.upload(P.eaPtr);
  d.eaMap = m.upload(P.eaMap);
  d.lvlSn = m.upload(P.lvlSn);
  d.perm = m.upload(P.perm);
  d.Sp = m.upload(P.Sp);
  d.Si = m.upload(P.Si);
  d.blkOff = m.upload(P.blkOff);
  d.rowBlk = m.upload(P.rowBlk);
  d.invOff = m.upload(P.invOff);
  d.diagSlot = m.upload(P.diagSlot);
  d.solveSmall = m.upload(P.solveSmall);
  pl->dAsm = m.upload(P.asmTasks);
  pl->dAsmCh = m.upload(P.asmCh);
  pl->dGroupItems = m.upload(P.groupItems);
  pl->dStrips = m.upload(P.strips);
  pl->dTile = m.upload(P.tileTasks);
  pl->dUTile = m.upload(P.uTasks);
  pl->dMixTile = m.upload(P.mixTiles);
  pl->dMixU = m.upload(P.mixUTasks);
  pl->dFwdTasks = (int4 *)m.upload(P.fwdTasks);
  pl->dFwdTasks1 = (int4 *)m.upload(P.fwdTasks1);
  pl->dBwdTasks = (int4 *)m.upload(P.bwdTasks);
  pl->dBwdAll = (int4 *)m.upload(P.bwdAll);
  pl->dTinySn = m.upload(P.tinySn);
  pl->dSmallSn = m.upload(P.smallSn);
  pl->dChain = (int2 *)m.upload(P.chainTasks);
  pl->dInvBlocks = m.upload(P.invBlocks);
}

void ensure_solve_ws(amp_factor *f, int q) {
  if (q <= f->qcap) return;
  f->smem.release();
  const amp::Plan &P = f->plan->P;
  size_t n = (size_t)P.n;
  f->dY = f->smem.alloc<double>(n * q);
  f->dT = f->smem.alloc<double>((size_t)P.solveBufDoubles * q);
  f->dB = f->smem.alloc<double>(n * q);
  f->dX = f->smem.alloc<double>(n * q);
  f->dR = f->smem.alloc<double>(n * q);
  f->dDX = f->smem.alloc<double>(n * q);
  f->dNorms = f->smem.alloc<double>(2 * (size_t)q);
  f->qcap = q;
}

enum KernelKind {
  K_ASSEMBLE, K_PANEL, K_UPDATE, K_FORWARD, K_BACKWARD, K_PERMUTE, K_RESIDUAL, K_POTRF, K_DIAGINV, K_KRYLOV,
  K_FRONTS, K_CHAIN, K_NKINDS
};
const char *kKindNames[K_NKINDS] = {"assemble",      "group_panel", "update_syrk", "solve_forward",
                                    "solve_backward", "permute",    "residual_spmv", "potrf",
                                    "diag_inverse",  "krylov",     "small_fronts", "chain_mats"};

cudaEvent_t pool_event(amp_factor *f) {
  if (f->evUsed == f->evPool.size()) {
    cudaEvent_t e;
    ck(cudaEventCreate(&e), "cudaEventCreate");
    f->evPool.push_back(e);
  }
  return f->evPool[f->evUsed++];
}

// Run one launch; while profiling, bracket it with events and record its algorithmic work. launch() issues one
// kernel, or returns how many it issued.
template <class L>
void timed_on(amp_factor *f, cudaStream_t st, int kind, double flops, double bytes, L &&launch) {
  if (!f->profiling) {
    launch();
    return;
  }
  amp_factor_s::Rec r{kind, pool_event(f), pool_event(f), flops, bytes, 1};
  ck(cudaEventRecord(r.a, st), "event");
  if constexpr (std::is_void_v<decltype(launch())>)
    launch();
  else
    r.kernels = (int)launch();
  ck(cudaEventRecord(r.b, st), "event");
  f->recs.push_back(r);
}
template <class L>
void timed(amp_factor *f, int kind, double flops, double bytes, L &&launch) {
  timed_on(f, f->stream, kind, flops, bytes, launch);
}

// Look-ahead of the panel steps: part B of a step's update (the columns right of the next pivot block) runs on the
// side stream while the factor's stream factors the next pivot block (part A of the update, POTRF, TRSM). Part A of
// step k + 1 writes columns part B of step k also writes, so it waits for it; the level's update-block pass and
// the next level wait for all of it. Inside the captured graph these waits are the graph's edges.
struct LookAhead {
  amp_factor *f;
  bool pending = false;  // a part B was issued since the last join
  void trsm_done() { ck(cudaEventRecord(f->evPanel, f->stream), "event"); }
  void before_part_a() {
    if (pending) ck(cudaStreamWaitEvent(f->stream, f->evSide, 0), "wait");
  }
  template <class L>
  void part_b(int kind, double flops, L &&launch) {
    ck(cudaStreamWaitEvent(f->side, f->evPanel, 0), "wait");
    timed_on(f, f->side, kind, flops, 0.0, launch);
    ck(cudaEventRecord(f->evSide, f->side), "event");
    pending = true;
  }
  void join() {
    if (pending) ck(cudaStreamWaitEvent(f->stream, f->evSide, 0), "wait");
    pending = false;
  }
};

// the small fronts of level L (whole fronts, one warp or one CTA each)
template <class T>
void enqueue_small_fronts(amp_factor *f, int L, T *Lx, T *U, const amp::LdltArgs<T> &la) {
  const amp::Plan &P = f->plan->P;
  const int64_t t0 = P.tinyPtr[L], t1 = P.tinyPtr[L + 1], s0 = P.smallPtr[L], s1 = P.smallPtr[L + 1];
  if (t1 == t0 && s1 == s0) return;
  const double scale = sizeof(T) / 8.0;
  timed(f, K_FRONTS, 2.0 * P.frontLvlFlops[L], P.frontLvlBytes[L] * scale, [&] {
    return amp::launch_fronts_small<T>(f->plan->dTinySn + t0, (int)(t1 - t0), (int)(P.tinyMid[L] - t0),
                                       f->plan->dSmallSn + s0, (int)(s1 - s0), P.smallMaxM[L], f->plan->dp,
                                       f->dValues, Lx, U, f->dStatus, la, f->stream);
  });
}

// chain matrices of consecutive diagonal blocks for the one-vector sweeps (after the inverses)
template <class T>
void enqueue_chain_mats(amp_factor *f, const T *Lx, const T *Inv, T *Mch, T *Gch) {
  const amp::Plan &P = f->plan->P;
  const int nt = (int)(P.chainTasks.size() / 2);
  if (nt == 0 || f->kind == AMP_LDLT) return;  // LDL^T sweeps apply the inverse blocks last
  timed(f, K_CHAIN, 2.0 * 2.0 * 64.0 * 64.0 * 64.0 / 2.0 * nt, 3.0 * 64.0 * 64.0 * sizeof(T) * nt, [&] {
    amp::launch_chain_mats<T>(f->plan->dChain, nt, f->plan->dp, Lx, Inv, Mch, Gch, f->stream);
  });
}

void enqueue_factor(amp_factor *f) {
  const amp::Plan &P = f->plan->P;
  amp::DevPlan dp = f->plan->dp;
  if (f->waitSpins > 0) dp.spin = f->waitSpins;
  cudaStream_t st = f->stream;
  ck(cudaMemsetAsync(f->dStatus, 0xff, sizeof(unsigned long long), st), "memset status");
  if (P.nGroupFlags + P.nGroupTickets > 0)
    ck(cudaMemsetAsync(f->dGroupFlags, 0, sizeof(int) * (P.nGroupFlags + P.nGroupTickets), st), "memset flags");
  int *tickets = f->dGroupFlags + P.nGroupFlags;
  if (f->precision == AMP_MIXED) {
    amp::LdltArgs<float> ld32{};
    if (f->kind == AMP_LDLT) {
      ld32 = amp::LdltArgs<float>{f->dScal, f->dCounts, nullptr, f->dD, f->dWhi, f->dWlo};
      ck(cudaMemsetAsync(f->dCounts, 0, 2 * sizeof(int), st), "memset counts");
      amp::launch_ldlt_tau(f->dValues, dp, f->dScal, st);
    }
    for (int L = 0; L < P.nlevels; L++) {
      enqueue_small_fronts<float>(f, L, f->dL32, f->dU32, ld32);
      if (P.asmLvlPtr[L + 1] > P.asmLvlPtr[L])
        timed(f, K_ASSEMBLE, 0.0, P.asmLvlBytes[L] / 2, [&] {
          amp::launch_assemble<float>(f->plan->dAsm + P.asmLvlPtr[L], f->plan->dAsmCh, P.asmLvlPtr[L + 1] - P.asmLvlPtr[L], dp,
                                      f->dValues, f->dL32, f->dU32, f->dStatus, st);
        });
      LookAhead la{f};
      for (int k = P.lvlStepPtr[L]; k < P.lvlStepPtr[L + 1]; k++) {
        const amp::StepRange &sr = P.steps[k];
        timed(f, K_PANEL, sr.panelFlops, 0.0, [&] {
          amp::launch_group_panel<float>(f->plan->dGroupItems, f->plan->dStrips + sr.strip0,
                                         (int)(sr.strip1 - sr.strip0), tickets + sr.ticket, f->dGroupFlags, dp,
                                         f->dL32, f->dStatus, f->dShi, f->dSlo, ld32, st);
        });
        la.trsm_done();
        la.before_part_a();
        if (sr.mixMid > sr.mix0)
          timed(f, K_UPDATE, sr.updateFlopsA, 0.0, [&] {
            amp::launch_update_mx(f->plan->dMixTile + sr.mix0, sr.mixMid - sr.mix0, f->dMaps, f->dL32, f->dU32,
                                  f->dStatus, amp::num_sms(), st, sr.mixWidthA, f->waitSpins);
          });
        if (sr.mix1 > sr.mixMid)
          la.part_b(K_UPDATE, sr.updateFlopsB, [&] {
            amp::launch_update_mx(f->plan->dMixTile + sr.mixMid, sr.mix1 - sr.mixMid, f->dMaps, f->dL32, f->dU32,
                                  f->dStatus, amp::num_sms(), f->side, 256, f->waitSpins);
          });
      }
      la.join();
      const int64_t u0 = P.mixULvlPtr[L], u1 = P.mixULvlPtr[L + 1];
      if (u1 > u0)
        timed(f, K_UPDATE, P.uLvlFlops[L], 0.0, [&] {
          amp::launch_update_mx(f->plan->dMixU + u0, u1 - u0, f->dMaps, f->dL32, f->dU32, f->dStatus,
                                amp::num_sms(), st, 256, f->waitSpins);
        });
    }
    if (P.nflags)
      timed(f, K_DIAGINV, 0.0, 8.0 * (double)inv_elems(P),
            [&] {
              amp::launch_diag_inv<float>(f->plan->dInvBlocks, (int)P.invBlocks.size(), dp, f->dL32, f->dInv32, st);
            });
    enqueue_chain_mats<float>(f, f->dL32, f->dInv32, f->dMch32, f->dGch32);
    return;
  }
  const bool ldlt = f->kind == AMP_LDLT;
  amp::LdltArgs<double> ld = ldlt ? amp::LdltArgs<double>{f->dScal, f->dCounts, f->dW, f->dD, nullptr, nullptr}
                                  : amp::LdltArgs<double>{};
  if (f->bk) {  // Bunch-Kaufman pivots inside each pivot block: the small-front and group-panel kernels' BK variants
    ld.piv = f->dPiv;
    ld.Doff = f->dDoff;
    dp.lpiv = f->dPiv;  // the inverse blocks with each block's pivot order folded in
  }
  if (ldlt) {
    ck(cudaMemsetAsync(f->dCounts, 0, 2 * sizeof(int), st), "memset counts");
    amp::launch_ldlt_tau(f->dValues, dp, f->dScal, st);
  }
  for (int L = 0; L < P.nlevels; L++) {
    enqueue_small_fronts<double>(f, L, f->dLx, f->dU, ld);
    if (P.asmLvlPtr[L + 1] > P.asmLvlPtr[L])
      timed(f, K_ASSEMBLE, 0.0, P.asmLvlBytes[L], [&] {
        amp::launch_assemble<double>(f->plan->dAsm + P.asmLvlPtr[L], f->plan->dAsmCh, P.asmLvlPtr[L + 1] - P.asmLvlPtr[L], dp,
                                     f->dValues, f->dLx, f->dU, f->dStatus, st);
      });
    LookAhead la{f};
    for (int k = P.lvlStepPtr[L]; k < P.lvlStepPtr[L + 1]; k++) {
      const amp::StepRange &sr = P.steps[k];
      timed(f, K_PANEL, sr.panelFlops, 0.0, [&] {
        amp::launch_group_panel<double>(f->plan->dGroupItems, f->plan->dStrips + sr.strip0,
                                        (int)(sr.strip1 - sr.strip0), tickets + sr.ticket, f->dGroupFlags, dp, f->dLx,
                                        f->dStatus, nullptr, nullptr, ld, st);
      });
      la.trsm_done();
      la.before_part_a();
      if (sr.tileMid > sr.tile0)
        timed(f, K_UPDATE, sr.updateFlopsA, 0.0, [&] {
          amp::launch_update(f->plan->dTile + sr.tile0, sr.tileMid - sr.tile0, dp, f->dLx, f->dU, ld.W, f->dStatus,
                             st);
        });
      if (sr.tile1 > sr.tileMid)
        la.part_b(K_UPDATE, sr.updateFlopsB, [&] {
          amp::launch_update(f->plan->dTile + sr.tileMid, sr.tile1 - sr.tileMid, dp, f->dLx, f->dU, ld.W, f->dStatus,
                             f->side);
        });
    }
    la.join();
    if (P.uLvlPtr[L + 1] > P.uLvlPtr[L])
      timed(f, K_UPDATE, P.uLvlFlops[L], 0.0, [&] {
        amp::launch_update(f->plan->dUTile + P.uLvlPtr[L], P.uLvlPtr[L + 1] - P.uLvlPtr[L], dp, f->dLx, f->dU, ld.W,
                           f->dStatus, st);
      });
  }
  if (P.nflags)
    timed(f, K_DIAGINV, 0.0, 16.0 * (double)inv_elems(P),
          [&] {
            amp::launch_diag_inv<double>(f->plan->dInvBlocks, (int)P.invBlocks.size(), dp, f->dLx, f->dInv, st);
          });
  enqueue_chain_mats<double>(f, f->dLx, f->dInv, f->dMch, f->dGch);
}

// y (permuted order, q vectors) := A^-1 y in place
// the plan's device view with this factor's wait bound
amp::DevPlan solve_view(const amp_factor *f) {
  amp::DevPlan dp = f->plan->dp;
  if (f->waitSpins > 0) dp.spin = f->waitSpins;
  if (f->bk) dp.lpiv = f->dPiv;
  return dp;
}

void device_solve_permuted(amp_factor *f) {
  const amp::Plan &P = f->plan->P;
  const amp::DevPlan dp = solve_view(f);
  const double lbytes = (f->dL32 ? 4.0 : 8.0) * (double)P.nnzLStored;  // each sweep reads L once
  cudaStream_t st = f->stream;
  ck(cudaMemsetAsync(f->dTickets, 0, sizeof(int) * 2, st), "memset tickets");
  ck(cudaMemsetAsync(f->dDone, 0, sizeof(int) * std::max(1, P.nsuper), st), "memset done");
  ck(cudaMemsetAsync(f->dSolveStatus, 0xff, sizeof(unsigned long long), st), "memset status");
  const int efwd = 2 * (++f->solveEpoch) - 1, ebwd = 2 * f->solveEpoch;
  const int nf = (int)(P.fwdTasks1.size() / 4), nb = (int)(P.bwdAll.size() / 4);
  const bool ldlt = f->kind == AMP_LDLT;
  const double *Dp = ldlt && !f->bk ? f->dD : nullptr;  // a Bunch-Kaufman factor's D solve runs between the sweeps
  timed(f, K_FORWARD, 2.0 * (double)P.nnzLStored, lbytes, [&] {
    if (f->dL32)
      amp::launch_fwd_blocks<float>(f->plan->dFwdTasks1, nf, f->dTickets, dp, f->dL32, f->dInv32,
                                    ldlt ? nullptr : f->dMch32, f->dY, f->dT, f->dFlags, f->dHand, efwd, f->dDone,
                                    f->dSolveStatus, st);
    else
      amp::launch_fwd_blocks<double>(f->plan->dFwdTasks1, nf, f->dTickets, dp, f->dLx, f->dInv, ldlt ? nullptr : f->dMch,
                                     f->dY, f->dT, f->dFlags, f->dHand, efwd, f->dDone, f->dSolveStatus, st);
  });
  if (f->bk)
    timed(f, K_PERMUTE, (double)P.n, 24.0 * P.n, [&] { amp::launch_dsolve_bk(P.n, 1, f->dD, f->dDoff, f->dY, st); });
  timed(f, K_BACKWARD, 2.0 * (double)P.nnzLStored, lbytes, [&] {
    if (f->dL32)
      amp::launch_bwd_blocks<float>(f->plan->dBwdAll, nb, f->dTickets + 1, dp, f->dL32, f->dInv32,
                                    ldlt ? nullptr : f->dGch32, Dp, f->dY, f->dFlags, f->dHand, ebwd, f->dSolveStatus,
                                    st);
    else
      amp::launch_bwd_blocks<double>(f->plan->dBwdAll, nb, f->dTickets + 1, dp, f->dLx, f->dInv,
                                     ldlt ? nullptr : f->dGch, Dp, f->dY, f->dFlags, f->dHand, ebwd, f->dSolveStatus,
                                     st);
  });
}

// AMP_DEVICE_TIMEOUT when a bounded wait of the last solve gave up (the stream must be synchronised)
int solve_status(amp_factor *f) {
  unsigned long long stw = 0;
  ck(cudaMemcpy(&stw, f->dSolveStatus, sizeof stw, cudaMemcpyDeviceToHost), "copy solve status");
  if (stw != amp::kStatusOk) return fail(AMP_DEVICE_TIMEOUT, "solve: a device wait timed out");
  return AMP_OK;
}

// x = A^-1 b for one device vector (original order)
void device_solve(amp_factor *f, const double *dB, double *dX) {
  const amp::Plan &P = f->plan->P;
  const double pb = 20.0 * P.n;
  timed(f, K_PERMUTE, 0.0, pb, [&] { amp::launch_permute_in(dB, f->dY, f->plan->dp.perm, P.n, 1, f->stream); });
  device_solve_permuted(f);
  timed(f, K_PERMUTE, 0.0, pb, [&] { amp::launch_permute_out(f->dY, dX, f->plan->dp.perm, P.n, 1, f->stream); });
}

// ---- several right-hand sides: groups of up to multi_max_vectors() vectors, interleaved ([i q + k]) -------------
// The multi-vector task lists for ns vector slices: a block task (kind 0 / 1) is expanded into ns consecutive entries
// with .w = the slice (the slices' chains run on different CTAs); the small-supernode tasks (kind 2) stay single.
// When supernodes with at most kWideBlocks pivot blocks hold at least half of L (a plan of many small systems, like
// the batch) and there are two or more slices, those supernodes' tasks stay single with .w = -1
// and move all vectors at once (no chain to split, one pass over the L tile, a quarter of the tasks). Built and
// uploaded once per plan and ns.
constexpr int kWideBlocks = 2;
static std::vector<int> expand_slices(const amp::Plan &P, const std::vector<int> &tasks, size_t ntasks, int ns,
                                      bool wide) {
  std::vector<int> out;
  out.reserve(4 * ntasks * (size_t)ns);
  for (size_t i = 0; i < ntasks; i++) {
    const int *t = &tasks[4 * i];
    if (t[2] == 2 || (wide && (P.snNc[t[0]] + 63) / 64 <= kWideBlocks)) {
      out.insert(out.end(), {t[0], t[1], t[2], t[2] == 2 ? 0 : -1});
      continue;
    }
    for (int sl = 0; sl < ns; sl++) out.insert(out.end(), {t[0], t[1], t[2], sl});
  }
  return out;
}
static void slice_lists(amp_plan *pl, int ns) {
  std::lock_guard<std::mutex> lock(pl->slMu);
  if (pl->dFwdSl[ns - 1]) return;
  const amp::Plan &P = pl->P;
  const size_t nf = (size_t)P.fwdLvlPtr[P.nlevels];
  double lAll = 0, lSmall = 0;  // L entries (nc m per supernode): all, and in supernodes of few pivot blocks
  for (int sn = 0; sn < P.nsuper; sn++) {
    const double e = (double)P.snNc[sn] * P.snM[sn];
    lAll += e;
    if ((P.snNc[sn] + 63) / 64 <= kWideBlocks) lSmall += e;
  }
  const bool wide = ns > 1 && lAll > 0 && 2 * lSmall >= lAll;
  const std::vector<int> fw = expand_slices(P, P.fwdTasks, nf, ns, wide);
  const std::vector<int> bw = expand_slices(P, P.bwdAll, P.bwdAll.size() / 4, ns, wide);
  pl->wideSl[ns - 1] = wide;
  pl->dBwdSl[ns - 1] = (int4 *)pl->mem.upload(bw);
  pl->nBwdSl[ns - 1] = (int)(bw.size() / 4);
  pl->nFwdSl[ns - 1] = (int)(fw.size() / 4);
  pl->dFwdSl[ns - 1] = (int4 *)pl->mem.upload(fw);
}
// y (permuted order, interleaved) := A^-1 y in place
void device_solve_multi_permuted(amp_factor *f, int q) {
  const amp::Plan &P = f->plan->P;
  const amp::DevPlan dp = solve_view(f);
  const double lbytes = (f->dL32 ? 4.0 : 8.0) * (double)P.nnzLStored;  // each sweep reads L once for all q vectors
  const double flops = 2.0 * (double)P.nnzLStored * q;
  cudaStream_t st = f->stream;
  ck(cudaMemsetAsync(f->dTickets, 0, sizeof(int) * 2, st), "memset tickets");
  const int nfl = std::max(1, P.nflags);
  ck(cudaMemsetAsync(f->dDone, 0, sizeof(int) * kSlices * std::max(1, P.nsuper), st), "memset done");
  ck(cudaMemsetAsync(f->dSolveStatus, 0xff, sizeof(unsigned long long), st), "memset status");
  const int efwd = 2 * (++f->solveEpoch) - 1, ebwd = 2 * f->solveEpoch;
  const int ns = amp::multi_slices(q);
  slice_lists(f->plan, ns);
  const int nf = f->plan->nFwdSl[ns - 1], nb = f->plan->nBwdSl[ns - 1];
  int4 *fwdTasks = f->plan->dFwdSl[ns - 1], *bwdTasks = f->plan->dBwdSl[ns - 1];
  const bool wide = f->plan->wideSl[ns - 1];
  const double *Dp = f->kind == AMP_LDLT && !f->bk ? f->dD : nullptr;  // Bunch-Kaufman: D solve between the sweeps
  const bool chain = f->kind != AMP_LDLT;  // Cholesky: chain matrices of consecutive diagonal blocks
  timed(f, K_FORWARD, flops, lbytes, [&] {
    if (f->dL32)
      amp::launch_fwd_multi<float>(fwdTasks, nf, wide, f->dTickets, dp, f->dL32, f->dInv32, chain ? f->dMch32 : nullptr,
                                   f->dY, f->dT, f->dFlags,
                                   nfl, efwd, f->dDone, q, f->dSolveStatus, st);
    else
      amp::launch_fwd_multi<double>(fwdTasks, nf, wide, f->dTickets, dp, f->dLx, f->dInv, chain ? f->dMch : nullptr,
                                    f->dY, f->dT, f->dFlags,
                                    nfl, efwd, f->dDone, q, f->dSolveStatus, st);
  });
  if (f->bk)
    timed(f, K_PERMUTE, (double)P.n * q, 24.0 * P.n * q,
          [&] { amp::launch_dsolve_bk(P.n, q, f->dD, f->dDoff, f->dY, st); });
  timed(f, K_BACKWARD, flops, lbytes, [&] {
    if (f->dL32)
      amp::launch_bwd_multi<float>(bwdTasks, nb, wide, f->dTickets + 1, dp, f->dL32, f->dInv32,
                                   chain ? f->dGch32 : nullptr, Dp, f->dY, f->dFlags, nfl,
                                   ebwd, q, f->dSolveStatus, st);
    else
      amp::launch_bwd_multi<double>(bwdTasks, nb, wide, f->dTickets + 1, dp, f->dLx, f->dInv, chain ? f->dGch : nullptr,
                                    Dp, f->dY, f->dFlags, nfl,
                                    ebwd, q, f->dSolveStatus, st);
  });
}

// xil = A^-1 bil, interleaved vectors in the original order
void device_solve_il(amp_factor *f, const double *bil, double *xil, int q) {
  const amp::Plan &P = f->plan->P;
  const double pb = 20.0 * P.n * q;
  timed(f, K_PERMUTE, 0.0, pb,
        [&] { amp::launch_rows_permute(bil, f->dY, f->plan->dp.perm, P.n, q, false, f->stream); });
  if (q == 1)  // one vector: the interleaved layout is the plain one
    device_solve_permuted(f);
  else
    device_solve_multi_permuted(f, q);
  timed(f, K_PERMUTE, 0.0, pb,
        [&] { amp::launch_rows_permute(f->dY, xil, f->plan->dp.perm, P.n, q, true, f->stream); });
}

// x = A^-1 b for nrhs > 1 vectors stored one after another (host or device), refined in FP64 when o is given.
// Each group of up to multi_max_vectors() vectors is moved to the interleaved layout, solved (and refined) and moved
// back. stt receives the worst relative residual and the largest number of refinement steps over the groups.
int solve_many(amp_factor *f, const double *b, int nrhs, double *x, bool on_device, const amp_refine_opts *o,
               amp_refine_stats *stt) {
  const amp::Plan &P = f->plan->P;
  const int n = P.n, G = amp::multi_max_vectors();
  ensure_solve_ws(f, std::min(nrhs, G));
  cudaStream_t st = f->stream;
  double worst = 0;
  int maxSteps = 0;
  const int ng = std::max(1, f->ngroups);
  double *dNorms = f->ngroups > 0 ? f->dGroupNorms : f->dNorms;
  std::vector<double> norms(2 * (size_t)ng * G);
  for (int g0 = 0; g0 < nrhs; g0 += G) {
    const int qg = std::min(G, nrhs - g0);
    const size_t len = (size_t)n * qg, bytes = sizeof(double) * len;
    const double *bg = b + (size_t)g0 * n;
    double *xg = x + (size_t)g0 * n;
    if (!on_device) {
      ck(cudaMemcpyAsync(f->dDX, bg, bytes, cudaMemcpyHostToDevice, st), "copy b");
      amp::launch_to_interleaved(f->dDX, f->dB, n, qg, st);
    } else {
      amp::launch_to_interleaved(bg, f->dB, n, qg, st);
    }
    device_solve_il(f, f->dB, f->dX, qg);
    int steps = 0;
    double gw = 0;  // worst relative residual of this group of vectors at its last residual evaluation
    for (; o; steps++) {
      const size_t nn = (size_t)2 * ng * qg;
      ck(cudaMemsetAsync(dNorms, 0, sizeof(double) * nn, st), "memset");
      timed(f, K_RESIDUAL, 2.0 * P.patNnz * qg, 12.0 * P.patNnz + 24.0 * n * qg, [&] {
        amp::launch_residual_multi(n, f->plan->dRowptr, f->plan->dColidx, f->dValues, f->dX, f->dB, f->dR, dNorms, qg,
                                   f->ngroups > 0 ? f->dRowGroup : nullptr, st);
      });
      ck(cudaMemcpyAsync(norms.data(), dNorms, sizeof(double) * nn, cudaMemcpyDeviceToHost, st), "norms");
      ck(cudaStreamSynchronize(st), "residual");
      gw = 0;
      bool any = false;
      for (size_t e = 0; e < (size_t)ng * qg; e++) {  // (row group, vector) pairs
        double bn = std::sqrt(norms[2 * e + 1]);
        if (bn == 0 || std::isnan(bn)) bn = 1;
        const double rel = std::sqrt(norms[2 * e]) / bn;
        gw = std::max(gw, rel);
        if (!(rel < o->tol)) any = true;
      }
      if (!any || steps >= o->max_steps) break;
      device_solve_il(f, f->dR, f->dDX, qg);
      amp::launch_axpy(f->dX, f->dDX, (int64_t)len, st);
    }
    worst = std::max(worst, gw);
    maxSteps = std::max(maxSteps, steps);
    if (!on_device) {
      amp::launch_from_interleaved(f->dX, f->dDX, n, qg, st);
      ck(cudaMemcpyAsync(xg, f->dDX, bytes, cudaMemcpyDeviceToHost, st), "copy x");
    } else {
      amp::launch_from_interleaved(f->dX, xg, n, qg, st);
    }
  }
  ck(cudaGetLastError(), "kernel launch");
  ck(cudaStreamSynchronize(st), "solve");
  if (int rc = solve_status(f)) return rc;
  if (stt) {
    stt->rel_residual = worst;
    stt->steps = maxSteps;
  }
  return (int)AMP_OK;
}

// Kernel attributes (large dynamic shared memory) belong to each device's context: set them once per device, with
// that device current, the first time a factor is created on it. Host threads creating factors on the same device
// take turns.
void init_device_once(int dev) {
  static std::mutex mu;
  static std::vector<char> done;
  std::lock_guard<std::mutex> lock(mu);
  if (dev < 0) throw std::runtime_error("invalid device ordinal");
  if ((size_t)dev >= done.size()) done.resize(dev + 1, 0);
  if (done[dev]) return;
  ck(amp::init_kernel_attributes(), "cudaFuncSetAttribute");
  done[dev] = 1;
}

template <class F>
int guarded(F &&fn) {
  try {
    g_err.clear();
    return fn();
  } catch (const CudaError &e) {
    return e.code;
  } catch (const std::bad_alloc &) {
    return fail(AMP_OOM, "host allocation failed");
  } catch (const std::exception &e) {
    return fail(AMP_INVALID, e.what());
  }
}

}  // namespace


// ---- shift-invert eigen operator and the device block Lanczos / Arnoldi (eigen.ts:116-175, arnoldi.mjs:36-200) ----
namespace {

// Y = A^-1 (M X) for m device vectors (one after another); T: n m scratch. Synchronises; returns an amp_status.
int device_shift_invert(amp_factor *f, const double *dX, int m, double *dY, double *dT) {
  const amp::Plan &P = f->plan->P;
  cudaStream_t st = f->stream;
  amp::launch_matvec(P.n, f->plan->dRowptr, f->plan->dColidx, f->dMass, dX, dT, m, st);
  if (m > 1) return solve_many(f, dT, m, dY, true, nullptr, nullptr);
  ensure_solve_ws(f, 1);
  device_solve(f, dT, dY);
  ck(cudaGetLastError(), "kernel launch");
  ck(cudaStreamSynchronize(st), "shift-invert");
  return solve_status(f);
}

// Eigen-decomposition of a symmetric p x p matrix S (row-major) by cyclic Jacobi rotations: S = Q diag(w) Q^T,
// Q row-major (column c of Q is the eigenvector of w[c]).
void jacobi_eigen(int p, std::vector<double> S, std::vector<double> &w, std::vector<double> &Q) {
  Q.assign((size_t)p * p, 0.0);
  for (int i = 0; i < p; i++) Q[(size_t)i * p + i] = 1.0;
  for (int sweep = 0; sweep < 100; sweep++) {
    double off = 0.0, tot = 0.0;
    for (int i = 0; i < p; i++)
      for (int j = 0; j < p; j++) {
        const double v = S[(size_t)i * p + j] * S[(size_t)i * p + j];
        tot += v;
        if (i != j) off += v;
      }
    if (off <= 1e-30 * tot || off == 0.0) break;
    for (int a = 0; a < p - 1; a++)
      for (int c = a + 1; c < p; c++) {
        const double sac = S[(size_t)a * p + c];
        if (sac == 0.0) continue;
        const double theta = (S[(size_t)c * p + c] - S[(size_t)a * p + a]) / (2.0 * sac);
        const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
        const double cs = 1.0 / std::sqrt(t * t + 1.0), sn = t * cs;
        for (int k = 0; k < p; k++) {  // S <- S J (columns a, c)
          const double ska = S[(size_t)k * p + a], skc = S[(size_t)k * p + c];
          S[(size_t)k * p + a] = cs * ska - sn * skc;
          S[(size_t)k * p + c] = sn * ska + cs * skc;
        }
        for (int k = 0; k < p; k++) {  // S <- J^T S (rows a, c)
          const double sak = S[(size_t)a * p + k], sck = S[(size_t)c * p + k];
          S[(size_t)a * p + k] = cs * sak - sn * sck;
          S[(size_t)c * p + k] = sn * sak + cs * sck;
        }
        for (int k = 0; k < p; k++) {  // Q <- Q J
          const double qka = Q[(size_t)k * p + a], qkc = Q[(size_t)k * p + c];
          Q[(size_t)k * p + a] = cs * qka - sn * qkc;
          Q[(size_t)k * p + c] = sn * qka + cs * qkc;
        }
      }
  }
  w.resize(p);
  for (int i = 0; i < p; i++) w[i] = S[(size_t)i * p + i];
}

struct EigenWork {
  amp_factor *f;
  int64_t n;
  double *part, *dh;
  std::vector<double> h;
  // h[j] = A_j . w for the nv device vectors A (n each), synchronised
  const std::vector<double> &dots(const double *A, int nv, const double *w) {
    cudaStream_t st = f->stream;
    h.resize(std::max(nv, 1));
    amp::launch_dots(A, nv, n, w, part, dh, st);
    ck(cudaMemcpyAsync(h.data(), dh, sizeof(double) * nv, cudaMemcpyDeviceToHost, st), "dots");
    ck(cudaStreamSynchronize(st), "dots");
    return h;
  }
  // out = sum_j c[j] A_j (nv device vectors A); out is overwritten
  void combine(double *out, const double *A, const std::vector<double> &c, int nv) {
    cudaStream_t st = f->stream;
    ck(cudaMemsetAsync(out, 0, sizeof(double) * n, st), "zero");
    ck(cudaMemcpyAsync(dh, c.data(), sizeof(double) * nv, cudaMemcpyHostToDevice, st), "coefficients");
    amp::launch_combine_add(out, A, dh, nv, n, st);
    ck(cudaStreamSynchronize(st), "combine");  // dh is reused by the next call
  }
};

}  // namespace

// ---- complex-symmetric LDL^T (ldlt.mjs:648-900) --------------------------------------------------------------------
namespace {

void upload_cx(amp_plan *pl) {
  if (pl->cxUploaded) return;
  amp::build_dense_all(pl->P, pl->cx);
  DevMem &m = pl->mem;
  pl->dCxAsm = m.upload(pl->cx.asmTasks);
  pl->dCxAsmCh = m.upload(pl->cx.asmCh);
  pl->dCxItems = m.upload(pl->cx.groupItems);
  pl->dCxStrips = m.upload(pl->cx.strips);
  pl->dCxTiles = m.upload(pl->cx.tileTasks);
  pl->dCxU = m.upload(pl->cx.uTasks);
  pl->cxUploaded = true;
}

// the complex factorization: per level, assembly, the group steps (group panel, then the group's update of the
// columns right of it: the next group's columns, then the rest), the update blocks
void enqueue_cfactor(amp_factor *f) {
  const amp::Plan &P = f->plan->P;
  const amp::DenseSched &D = f->plan->cx;
  amp::DevPlan dp = f->plan->dp;
  if (f->waitSpins > 0) dp.spin = f->waitSpins;
  cudaStream_t st = f->stream;
  ck(cudaMemsetAsync(f->dStatus, 0xff, sizeof(unsigned long long), st), "memset status");
  ck(cudaMemsetAsync(f->dCounts, 0, 2 * sizeof(int), st), "memset counts");
  if (D.nGroupFlags + D.nGroupTickets > 0)
    ck(cudaMemsetAsync(f->dCxFlags, 0, sizeof(int) * (D.nGroupFlags + D.nGroupTickets), st), "memset flags");
  int *tickets = f->dCxFlags + D.nGroupFlags;
  amp::launch_ctau(f->dValC, dp, f->dScal, st);
  const amp::LdltArgs<amp::cplx> ld{f->dScal, f->dCounts, f->dWc, f->dDc, nullptr, nullptr};
  for (int L = 0; L < P.nlevels; L++) {
    if (D.asmLvlPtr[L + 1] > D.asmLvlPtr[L])
      timed(f, K_ASSEMBLE, 0.0, 0.0, [&] {
        amp::launch_assemble<amp::cplx>(f->plan->dCxAsm + D.asmLvlPtr[L], f->plan->dCxAsmCh, D.asmLvlPtr[L + 1] - D.asmLvlPtr[L], dp,
                                        f->dValC, f->dLc, f->dUc, f->dStatus, st);
      });
    for (int k = D.lvlStepPtr[L]; k < D.lvlStepPtr[L + 1]; k++) {
      const amp::StepRange &sr = D.steps[k];
      timed(f, K_PANEL, 4.0 * sr.panelFlops, 0.0, [&] {
        amp::launch_group_panel<amp::cplx>(f->plan->dCxItems, f->plan->dCxStrips + sr.strip0,
                                           (int)(sr.strip1 - sr.strip0), tickets + sr.ticket, f->dCxFlags, dp,
                                           f->dLc, f->dStatus, nullptr, nullptr, ld, st);
      });
      if (sr.tile1 > sr.tile0)
        timed(f, K_UPDATE, 4.0 * (sr.updateFlopsA + sr.updateFlopsB), 0.0, [&] {
          amp::launch_update_c(f->plan->dCxTiles + sr.tile0, sr.tile1 - sr.tile0, f->dLc, f->dUc, f->dWc, f->dStatus,
                               st);
        });
    }
    if (D.uLvlPtr[L + 1] > D.uLvlPtr[L])
      timed(f, K_UPDATE, 0.0, 0.0, [&] {
        amp::launch_update_c(f->plan->dCxU + D.uLvlPtr[L], D.uLvlPtr[L + 1] - D.uLvlPtr[L], f->dLc, f->dUc, f->dWc,
                             f->dStatus, st);
      });
  }
}

// y (permuted order) := A^-1 y
void csolve_permuted(amp_factor *f, amp::cplx *y) {
  const amp::Plan &P = f->plan->P;
  timed(f, K_FORWARD, 8.0 * (double)P.nnzLStored, 16.0 * (double)P.nnzLStored, [&] {
    return amp::launch_csolve_permuted(f->plan->dp, P.lvlPtr.data(), P.nlevels, f->dLc, f->dDc, y, f->stream);
  });
}

int require_complex(const amp_factor *f) {
  if (!f) return fail(AMP_INVALID, "null handle");
  if (f->kind != AMP_LDLT_COMPLEX) return fail(AMP_INVALID, "a real factor: use the real-valued entry points");
  return AMP_OK;
}

}  // namespace

extern "C" {

const char *amp_last_error(void) { return g_err.c_str(); }

int amp_amd_order(int32_t n, const int32_t *rowptr, const int32_t *colidx, double dense_factor, int32_t *perm) {
  return guarded([&] {
    if (n < 0 || (n > 0 && (!rowptr || !colidx || !perm))) return fail(AMP_INVALID, "amdOrder: invalid arguments");
    if (!amp::amd_order({n, rowptr, colidx}, dense_factor, perm))
      return fail(AMP_INVALID, "amdOrder: internal error");
    return (int)AMP_OK;
  });
}

int amp_nd_order(int32_t n, const int32_t *rowptr, const int32_t *colidx, const double *x, const double *y,
                 int32_t leaf, int32_t *perm) {
  return guarded([&] {
    if (n > 0 && (!x || !y)) return fail(AMP_NEED_COORDS, "analyze: ordering nd needs node coordinates x and y of length n");
    amp::nd_order({n, rowptr, colidx}, x, y, leaf > 0 ? leaf : 48, perm);
    return (int)AMP_OK;
  });
}

int amp_nd3_order(int32_t n, const int32_t *rowptr, const int32_t *colidx, const double *x, const double *y,
                  const double *z, int32_t leaf, int32_t *perm) {
  return guarded([&] {
    if (n > 0 && (!x || !y || !z)) return fail(AMP_NEED_COORDS, "nd3Order: needs DOF coordinates x, y and z of length n");
    amp::nd3_order({n, rowptr, colidx}, x, y, z, leaf > 0 ? leaf : 2000, perm);
    return (int)AMP_OK;
  });
}

int amp_pattern_fingerprint(int32_t n, const int32_t *rowptr, const int32_t *colidx, char *buf, int32_t buflen) {
  return guarded([&] {
    std::string k = amp::pattern_key({n, rowptr, colidx});
    if (!buf || buflen <= (int32_t)k.size()) return fail(AMP_INVALID, "fingerprint buffer too small");
    std::memcpy(buf, k.c_str(), k.size() + 1);
    return (int)AMP_OK;
  });
}

int amp_analyze(int32_t n, const int32_t *rowptr, const int32_t *colidx, const amp_analyze_opts *opts,
                amp_plan **out) {
  return guarded([&] {
    if (!out || n < 0 || !rowptr || (n > 0 && !colidx)) return fail(AMP_INVALID, "analyze: invalid arguments");
    *out = nullptr;
    amp_analyze_opts o{};
    o.relax = 1;
    if (opts) o = *opts;
    amp::Pattern A{n, rowptr, colidx};
    const int32_t *perm = nullptr;
    int ordering = 0;
    if (o.ordering == AMP_ORDER_GIVEN) {
      if (!o.perm) return fail(AMP_BAD_LENGTH, "analyze: perm has length 0, pattern has " + std::to_string(n) + " rows");
      perm = o.perm;
    } else if (o.ordering == AMP_ORDER_ND) {
      if (n > 0 && (!o.x || !o.y)) return fail(AMP_NEED_COORDS, "analyze: ordering nd needs node coordinates x and y of length n");
      ordering = 1;
    } else if (o.ordering == AMP_ORDER_ND3) {
      if (n > 0 && (!o.x || !o.y || !o.z)) return fail(AMP_NEED_COORDS, "nd3Order: needs DOF coordinates x, y and z of length n");
      ordering = 2;
    } else if (o.ordering != AMP_ORDER_AMD)
      return fail(AMP_INVALID, "analyze: unknown ordering");
    auto *pl = new amp_plan_s();
    pl->device = o.device;
    try {
      std::vector<int> permBuf;
      if (ordering == 1 && o.leaf > 0 && o.leaf != 48) {
        permBuf.resize(n);
        amp::nd_order(A, o.x, o.y, o.leaf, permBuf.data());
        perm = permBuf.data();
      } else if (ordering == 2 && o.leaf > 0 && o.leaf != 2000) {
        permBuf.resize(n);
        amp::nd3_order(A, o.x, o.y, o.z, o.leaf, permBuf.data());
        perm = permBuf.data();
      }
      amp::analyze(A, perm, perm ? 3 : ordering, o.x, o.y, o.z, o.relax != 0, pl->S);
      amp::Tuning tune;
      if (o.group_blocks > 0) tune.groupBlocks = o.group_blocks;
      if (o.small_front > 0) tune.smallCut = o.small_front;
      if (o.defer_updates > 0) tune.deferB = o.defer_updates;
      amp::build_plan(pl->S, pl->P, tune);
      pl->key = amp::pattern_key(A);
      pl->rowptr.assign(rowptr, rowptr + n + 1);
      pl->colidx.assign(colidx, colidx + (n ? rowptr[n] : 0));
    } catch (...) {
      delete pl;
      throw;
    }
    *out = pl;
    return (int)AMP_OK;
  });
}

int amp_plan_get_info(const amp_plan *pl, amp_plan_info *info) {
  if (!pl || !info) return fail(AMP_INVALID, "null handle");
  const amp::Symbolic &S = pl->S;
  info->n = S.n;
  info->nsuper = S.nsuper;
  info->max_front = S.maxFront;
  info->nlevels = pl->P.nlevels;
  info->nnz_l = S.nnzL;
  info->nnz_a = S.nnzA;
  info->nnz_l_stored = S.nnzLStored;
  info->pattern_nnz = S.patNnz;
  info->fill = S.fill;
  info->flops = S.flops;
  info->ordering_ms = S.ordering_ms;
  info->symbolic_ms = S.symbolic_ms;
  info->device_bytes = 8 * (pl->P.nnzLStored + pl->P.arenaDoubles + pl->P.patNnz + S.n) + 4 * (int64_t)(
      pl->P.asmDst.size() * 2 + pl->P.eaMap.size() + pl->P.Si.size() + pl->rowptr.size() + pl->colidx.size()) +
      (int64_t)(sizeof(amp::TileTask) * pl->P.tileTasks.size() + sizeof(amp::StripTask) * pl->P.strips.size());
  return AMP_OK;
}

int amp_plan_array(const amp_plan *pl, int field, void *dst, int64_t len, int64_t *out_len) {
  if (!pl) return fail(AMP_INVALID, "null handle");
  const amp::Symbolic &S = pl->S;
  const std::vector<int> *v = nullptr;
  switch (field) {
    case AMP_F_PERM: v = &S.perm; break;
    case AMP_F_PINV: v = &S.pinv; break;
    case AMP_F_PARENT: v = &S.parent; break;
    case AMP_F_COLCOUNT: v = &S.colCount; break;
    case AMP_F_LOWERP: v = &S.lowerP; break;
    case AMP_F_LOWERI: v = &S.lowerI; break;
    case AMP_F_LOWERSRC: v = &S.lowerSrc; break;
    case AMP_F_SUPERSTART: v = &S.superStart; break;
    case AMP_F_COLSUPER: v = &S.colSuper; break;
    case AMP_F_SUPERPARENT: v = &S.superParent; break;
    case AMP_F_CHILDHEAD: v = &S.childHead; break;
    case AMP_F_CHILDNEXT: v = &S.childNext; break;
    case AMP_F_SP: v = &S.Sp; break;
    case AMP_F_SI: v = &S.Si; break;
    case AMP_F_LEVEL_PTR: v = &pl->P.lvlPtr; break;
    case AMP_F_LEVEL_SUPERNODES: v = &pl->P.lvlSn; break;
    case AMP_F_FWD_TASKS: v = &pl->P.fwdTasks1; break;
    case AMP_F_FWD_TASKS_MULTI: v = &pl->P.fwdTasks; break;
    case AMP_F_BWD_TASKS: v = &pl->P.bwdAll; break;
    case AMP_F_SOLVE_SMALL: v = &pl->P.solveSmall; break;
    case AMP_F_TINY_FRONTS: v = &pl->P.tinySn; break;
    case AMP_F_LXP:
    case AMP_F_TINY_PTR:
    case AMP_F_TINY_MID: {
      const std::vector<int64_t> &w =
          field == AMP_F_LXP ? S.Lxp : field == AMP_F_TINY_PTR ? pl->P.tinyPtr : pl->P.tinyMid;
      if (out_len) *out_len = (int64_t)w.size();
      if (dst) std::memcpy(dst, w.data(), sizeof(int64_t) * std::min<int64_t>(len, w.size()));
      return AMP_OK;
    }
    default: return fail(AMP_INVALID, "unknown field");
  }
  if (out_len) *out_len = (int64_t)v->size();
  if (dst) std::memcpy(dst, v->data(), sizeof(int) * std::min<int64_t>(len, v->size()));
  return AMP_OK;
}

int amp_plan_autotune(amp_plan *pl, const double *values, int64_t nvalues, int values_on_device, int kind,
                      int precision, amp_tune_result *res) {
  return guarded([&] {
    if (!pl || !res) return fail(AMP_INVALID, "null handle");
    if (pl->uploaded) return fail(AMP_INVALID, "autotune: the plan already has a factor (tune before the first one)");
    if (nvalues != pl->P.patNnz)
      return fail(AMP_BAD_LENGTH, "factorNumeric: " + std::to_string(nvalues) + " values for a pattern with " +
                                      std::to_string(pl->P.patNnz) + " entries");
    static std::mutex mu;
    static std::map<std::string, amp::Tuning> cache;
    const std::string key = pl->key + ":" + std::to_string(kind) + ":" + std::to_string(precision);
    amp_tune_result r{};
    {
      std::lock_guard<std::mutex> lock(mu);
      auto it = cache.find(key);
      if (it != cache.end()) {
        amp::build_plan(pl->S, pl->P, it->second);
        r.group_blocks = it->second.groupBlocks;
        r.small_front = it->second.smallCut;
        r.defer_updates = it->second.deferB;
        r.cached = 1;
        *res = r;
        return (int)AMP_OK;
      }
    }
    const int groups[4] = {4, 2, 8, 1}, smalls[2] = {128, 64}, defers[3] = {2, 4, 8};  // the default first
    amp_factor_opts fo{kind, precision};
    double best = 0.0;
    amp::Tuning bestT;
    std::vector<amp::Tuning> cands;
    for (int g : groups)
      for (int sc : smalls) {
        amp::Tuning t;
        t.groupBlocks = g;
        t.smallCut = sc;
        cands.push_back(t);
      }
    // the group and whole-front candidates, then the deferrals of the update beyond the next group with the best
    for (size_t ci = 0; ci < cands.size() + 3; ci++) {
      amp::Tuning t;
      if (ci < cands.size()) {
        t = cands[ci];
      } else {
        t = bestT;
        t.deferB = defers[ci - cands.size()];
      }
      {
        const int g = t.groupBlocks, sc = t.smallCut;
        amp::build_plan(pl->S, pl->P, t);
        amp_factor *f = nullptr;
        int rc = amp_factor_create(pl, &fo, &f);
        double ms = 0.0;
        if (rc == AMP_OK) {
          amp_factor_result fr{};
          for (int rep = 0; rep < 3 && rc == AMP_OK; rep++) {  // the first run captures the graph; time the third
            rc = amp_factor_numeric(f, values, nvalues, values_on_device, 1e-13, &fr);
            ms = fr.ms;
          }
          amp_factor_destroy(f);
        }
        pl->mem.release();  // the next candidate uploads its own schedule
        pl->uploaded = false;
        pl->cxUploaded = false;
        if (rc != AMP_OK) return rc;
        r.candidates++;
        if (g == 4 && sc == 128 && t.deferB == 1) r.ms_default = ms;
        if (r.candidates == 1 || ms < best) {
          best = ms;
          bestT = t;
        }
      }
    }
    amp::build_plan(pl->S, pl->P, bestT);
    {
      std::lock_guard<std::mutex> lock(mu);
      cache[key] = bestT;
    }
    r.group_blocks = bestT.groupBlocks;
    r.small_front = bestT.smallCut;
    r.defer_updates = bestT.deferB;
    r.ms_best = best;
    *res = r;
    return (int)AMP_OK;
  });
}

int amp_plan_fingerprint(const amp_plan *pl, char *buf, int32_t buflen) {
  if (!pl || !buf || buflen <= (int32_t)pl->key.size()) return fail(AMP_INVALID, "fingerprint buffer too small");
  std::memcpy(buf, pl->key.c_str(), pl->key.size() + 1);
  return AMP_OK;
}

int amp_plan_check_pattern(const amp_plan *pl, int32_t n, const int32_t *rowptr, const int32_t *colidx) {
  if (!pl) return fail(AMP_INVALID, "null handle");
  if (n != pl->S.n || amp::pattern_key({n, rowptr, colidx}) != pl->key)
    return fail(AMP_PATTERN_MISMATCH, "symbolic analysis is for a different sparsity pattern");
  return AMP_OK;
}

void amp_plan_destroy(amp_plan *pl) { delete pl; }

int amp_factor_create(amp_plan *pl, const amp_factor_opts *opts, amp_factor **out) {
  return guarded([&] {
    if (!pl || !out) return fail(AMP_INVALID, "null handle");
    *out = nullptr;
    amp_factor_opts o{AMP_CHOLESKY, AMP_FP64};
    if (opts) o = *opts;
    if (o.kind != AMP_CHOLESKY && o.kind != AMP_LDLT && o.kind != AMP_LDLT_BK)
      return fail(AMP_INVALID, "unknown factor kind");
    if (o.precision != AMP_FP64 && o.precision != AMP_MIXED) return fail(AMP_INVALID, "unknown precision");
    if (o.kind == AMP_LDLT_BK && o.precision != AMP_FP64)
      return fail(AMP_INVALID, "Bunch-Kaufman LDL^T: FP64 precision only");
    ck(cudaSetDevice(pl->device), "cudaSetDevice");
    if (!pl->uploaded) {  // the device schedule is uploaded once, by the first factor of the plan
      upload_plan(pl);
      pl->dRowptr = pl->mem.upload(pl->rowptr);
      pl->dColidx = pl->mem.upload(pl->colidx);
      pl->uploaded = true;
    }
    auto *f = new amp_factor_s();
    f->plan = pl;
    f->kind = o.kind == AMP_LDLT_BK ? AMP_LDLT : o.kind;
    f->bk = o.kind == AMP_LDLT_BK;
    f->precision = o.precision;
    try {
      ck(cudaStreamCreateWithFlags(&f->stream, cudaStreamNonBlocking), "cudaStreamCreate");
      ck(cudaStreamCreateWithFlags(&f->side, cudaStreamNonBlocking), "cudaStreamCreate");
      ck(cudaEventCreateWithFlags(&f->evPanel, cudaEventDisableTiming), "cudaEventCreate");
      ck(cudaEventCreateWithFlags(&f->evSide, cudaEventDisableTiming), "cudaEventCreate");
      ck(cudaEventCreate(&f->ev0), "cudaEventCreate");
      ck(cudaEventCreate(&f->ev1), "cudaEventCreate");
      const amp::Plan &P = pl->P;
      if (o.precision == AMP_FP64) {
        f->dLx = f->mem.alloc<double>((size_t)P.nnzLStored);
        f->dU = f->mem.alloc<double>((size_t)P.arenaDoubles);
        f->dInv = f->mem.alloc<double>((size_t)inv_elems(P));
        f->dMch = f->mem.alloc<double>(chain_elems(P));
        f->dGch = f->mem.alloc<double>(chain_elems(P));
        if (f->kind == AMP_LDLT) {
          f->dW = f->mem.alloc<double>((size_t)P.nnzLStored);
          f->dScal = f->mem.alloc<double>(2);
          f->dCounts = f->mem.alloc<int>(2);
        }
        if (f->bk) {
          f->dDoff = f->mem.alloc<double>((size_t)std::max(1, P.n));
          f->dPiv = f->mem.alloc<int>((size_t)std::max(1, P.n));
        }
      } else {
        f->dL32 = f->mem.alloc<float>((size_t)P.nnzLStored);
        f->dU32 = f->mem.alloc<float>((size_t)P.arenaDoubles);
        f->dInv32 = f->mem.alloc<float>((size_t)inv_elems(P));
        f->dMch32 = f->mem.alloc<float>(chain_elems(P));
        f->dGch32 = f->mem.alloc<float>(chain_elems(P));
        f->dShi = f->mem.alloc<__nv_bfloat16>((size_t)P.splitElems);
        f->dSlo = f->mem.alloc<__nv_bfloat16>((size_t)P.splitElems);
        if (o.kind == AMP_LDLT) {
          f->dWhi = f->mem.alloc<__nv_bfloat16>((size_t)P.splitElems);
          f->dWlo = f->mem.alloc<__nv_bfloat16>((size_t)P.splitElems);
          f->dScal = f->mem.alloc<double>(2);
          f->dCounts = f->mem.alloc<int>(2);
          f->dMaps = f->mem.upload(split_tensor_maps(P, f->dWhi, f->dWlo, f->dShi, f->dSlo));
        } else {
          f->dMaps = f->mem.upload(split_tensor_maps(P, f->dShi, f->dSlo, f->dShi, f->dSlo));
        }
      }
      f->dD = f->mem.alloc<double>((size_t)P.n);
      f->dValues = f->mem.alloc<double>((size_t)P.patNnz);
      f->dStatus = f->mem.alloc<unsigned long long>(1);
      f->dFlags = f->mem.alloc<int>((size_t)kSlices * std::max(1, P.nflags));  // one set per vector slice
      ck(cudaMemset(f->dFlags, 0, sizeof(int) * kSlices * std::max(1, P.nflags)), "memset flags");
      {  // two tagged words per value of a 64-row block, one slot per pair of consecutive diagonal blocks
        const size_t hw = std::max<size_t>(1, (size_t)std::max(0, P.nflags - P.nsuper) * 128);
        f->dHand = f->mem.alloc<unsigned long long>(hw);
        ck(cudaMemset(f->dHand, 0, sizeof(unsigned long long) * hw), "memset hand-off");
      }
      f->dTickets = f->mem.alloc<int>(2);
      f->dGroupFlags = f->mem.alloc<int>((size_t)std::max(1, P.nGroupFlags + P.nGroupTickets));
      f->dDone = f->mem.alloc<int>((size_t)kSlices * std::max(1, P.nsuper));
      f->dSolveStatus = f->mem.alloc<unsigned long long>(1);
      init_device_once(pl->device);
    } catch (...) {
      delete f;
      throw;
    }
    *out = f;
    return (int)AMP_OK;
  });
}

int amp_factor_numeric(amp_factor *f, const double *values, int64_t nvalues, int values_on_device, double pivot_tol,
                       amp_factor_result *res) {
  return guarded([&] {
    if (!f) return fail(AMP_INVALID, "null handle");
    if (f->kind == AMP_LDLT_COMPLEX) return fail(AMP_INVALID, "a complex-symmetric factor: use the amp_c* entry points");
    const amp::Plan &P = f->plan->P;
    if (nvalues != P.patNnz)
      return fail(AMP_BAD_LENGTH, "factorNumeric: " + std::to_string(nvalues) + " values for a pattern with " +
                                      std::to_string(P.patNnz) + " entries");
    ck(cudaSetDevice(f->plan->device), "cudaSetDevice");
    f->ok = false;
    amp_factor_result r{};
    r.fail_column = -1;
    if (P.n == 0) {
      f->ok = true;
      r.ok = 1;
      if (res) *res = r;
      return (int)AMP_OK;
    }
    cudaStream_t st = f->stream;
    if (nvalues > 0)
      ck(cudaMemcpyAsync(f->dValues, values, sizeof(double) * nvalues,
                         values_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st),
         "copy values");
    f->hasValues = true;
    if (f->kind == AMP_LDLT)  // read by the tau kernel at the start of the captured sequence
      ck(cudaMemcpyAsync(f->dScal, &pivot_tol, sizeof(double), cudaMemcpyHostToDevice, st), "copy pivotTol");
    ck(cudaEventRecord(f->ev0, st), "event");
    if (f->profiling) {
      enqueue_factor(f);
    } else {
      if (!f->factorGraph) {  // capture the whole sequence once per factor object
        cudaGraph_t g;
        ck(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "begin capture");
        enqueue_factor(f);
        ck(cudaStreamEndCapture(st, &g), "end capture");
        ck(cudaGraphInstantiate(&f->factorGraph, g, 0), "graph instantiate");
        cudaGraphDestroy(g);
      }
      ck(cudaGraphLaunch(f->factorGraph, st), "graph launch");
    }
    ck(cudaGetLastError(), "kernel launch");
    ck(cudaEventRecord(f->ev1, st), "event");
    unsigned long long status = 0;
    int counts[2] = {0, 0};
    ck(cudaMemcpyAsync(&status, f->dStatus, sizeof status, cudaMemcpyDeviceToHost, st), "copy status");
    if (f->kind == AMP_LDLT)
      ck(cudaMemcpyAsync(counts, f->dCounts, sizeof counts, cudaMemcpyDeviceToHost, st), "copy counts");
    ck(cudaStreamSynchronize(st), "factor");
    r.n_neg = counts[0];
    r.n_perturbed = counts[1];
    float ms = 0;
    cudaEventElapsedTime(&ms, f->ev0, f->ev1);
    r.ms = ms;
    if (status == amp::kStatusOk) {
      r.ok = 1;
      f->ok = true;
    } else if (((status >> 24) & 0xff) == 3) {  // a bounded device wait gave up: not a numerical result
      if (res) *res = r;
      return fail(AMP_DEVICE_TIMEOUT, "factorNumeric: a device wait timed out");
    } else {
      r.ok = 0;
      r.fail_column = (int32_t)(status >> 32);
    }
    if (res) *res = r;
    return (int)AMP_OK;
  });
}

int amp_solve(amp_factor *f, const double *b, int32_t nrhs, double *x, int on_device) {
  return guarded([&] {
    if (!f) return fail(AMP_INVALID, "null handle");
    if (f->kind == AMP_LDLT_COMPLEX) return fail(AMP_INVALID, "a complex-symmetric factor: use the amp_c* entry points");
    if (!f->ok) return fail(AMP_NO_FACTOR, "solveNumeric: no successful numeric factorization");
    const amp::Plan &P = f->plan->P;
    if (nrhs <= 0 || P.n == 0) return (int)AMP_OK;
    ck(cudaSetDevice(f->plan->device), "cudaSetDevice");
    if (nrhs > 1) return solve_many(f, b, nrhs, x, on_device != 0, nullptr, nullptr);
    ensure_solve_ws(f, nrhs);
    size_t bytes = sizeof(double) * (size_t)P.n * nrhs;
    const double *dB = b;
    double *dX = x;
    if (!on_device) {
      ck(cudaMemcpyAsync(f->dB, b, bytes, cudaMemcpyHostToDevice, f->stream), "copy b");
      dB = f->dB;
      dX = f->dX;
    }
    device_solve(f, dB, dX);
    ck(cudaGetLastError(), "kernel launch");
    if (!on_device) ck(cudaMemcpyAsync(x, dX, bytes, cudaMemcpyDeviceToHost, f->stream), "copy x");
    ck(cudaStreamSynchronize(f->stream), "solve");
    return solve_status(f);
  });
}

int amp_solve_refined(amp_factor *f, const double *b, int32_t nrhs, double *x, int on_device,
                      const amp_refine_opts *opts, amp_refine_stats *stats) {
  return guarded([&] {
    if (!f) return fail(AMP_INVALID, "null handle");
    if (f->kind == AMP_LDLT_COMPLEX) return fail(AMP_INVALID, "a complex-symmetric factor: use the amp_c* entry points");
    if (!f->ok) return fail(AMP_NO_FACTOR, "solveNumeric: no successful numeric factorization");
    const amp::Plan &P = f->plan->P;
    amp_refine_opts o{3, 1e-14};
    if (opts) o = *opts;
    amp_refine_stats stt{0.0, 0};
    if (nrhs <= 0 || P.n == 0) {
      if (stats) *stats = stt;
      return (int)AMP_OK;
    }
    ck(cudaSetDevice(f->plan->device), "cudaSetDevice");
    if (nrhs > 1 || f->ngroups > 0) {
      const int rc = solve_many(f, b, nrhs, x, on_device != 0, &o, &stt);
      if (rc == AMP_OK && stats) *stats = stt;
      return rc;
    }
    ensure_solve_ws(f, nrhs);
    const int n = P.n;
    size_t len = (size_t)n * nrhs, bytes = sizeof(double) * len;
    cudaStream_t st = f->stream;
    const double *dB = b;
    double *dX = x;
    if (!on_device) {
      ck(cudaMemcpyAsync(f->dB, b, bytes, cudaMemcpyHostToDevice, st), "copy b");
      dB = f->dB;
      dX = f->dX;
    }
    device_solve(f, dB, dX);
    std::vector<double> norms(2 * (size_t)nrhs);
    std::vector<char> active(nrhs, 1);
    double worst = 0;
    int steps = 0;
    for (;; steps++) {
      ck(cudaMemsetAsync(f->dNorms, 0, sizeof(double) * 2 * nrhs, st), "memset");
      timed(f, K_RESIDUAL, 2.0 * P.patNnz * nrhs, (12.0 * P.patNnz + 24.0 * n) * nrhs, [&] {
        amp::launch_residual(n, f->plan->dRowptr, f->plan->dColidx, f->dValues, dX, dB, f->dR, f->dNorms, nrhs, st);
      });
      ck(cudaMemcpyAsync(norms.data(), f->dNorms, sizeof(double) * 2 * nrhs, cudaMemcpyDeviceToHost, st), "norms");
      ck(cudaStreamSynchronize(st), "residual");
      worst = 0;
      bool any = false;
      for (int k = 0; k < nrhs; k++) {
        double bn = std::sqrt(norms[2 * k + 1]);
        if (bn == 0 || std::isnan(bn)) bn = 1;
        double rel = std::sqrt(norms[2 * k]) / bn;
        worst = std::max(worst, rel);
        if (!(rel < o.tol)) any = true;
      }
      if (!any || steps >= o.max_steps) break;
      device_solve(f, f->dR, f->dDX);
      amp::launch_axpy(dX, f->dDX, (int64_t)len, st);
    }
    ck(cudaGetLastError(), "kernel launch");
    if (!on_device) ck(cudaMemcpyAsync(x, dX, bytes, cudaMemcpyDeviceToHost, st), "copy x");
    ck(cudaStreamSynchronize(st), "refine");
    if (int rc = solve_status(f)) return rc;
    stt.rel_residual = worst;
    stt.steps = steps;
    if (stats) *stats = stt;
    return (int)AMP_OK;
  });
}

int amp_factor_set_row_groups(amp_factor *f, int32_t ngroups, const int64_t *offsets) {
  return guarded([&] {
    if (!f) return fail(AMP_INVALID, "null handle");
    if (f->kind == AMP_LDLT_COMPLEX) return fail(AMP_INVALID, "a complex-symmetric factor: use the amp_c* entry points");
    const int n = f->plan->P.n;
    if (ngroups < 0 || (ngroups > 0 && !offsets)) return fail(AMP_INVALID, "row groups: bad arguments");
    if (ngroups == 0) {
      f->ngroups = 0;
      return (int)AMP_OK;
    }
    if (offsets[0] != 0 || offsets[ngroups] != n) return fail(AMP_INVALID, "row groups: offsets must run from 0 to n");
    std::vector<int> gid(n);
    for (int g = 0; g < ngroups; g++) {
      if (offsets[g + 1] < offsets[g]) return fail(AMP_INVALID, "row groups: offsets must not decrease");
      for (int64_t i = offsets[g]; i < offsets[g + 1]; i++) gid[i] = g;
    }
    ck(cudaSetDevice(f->plan->device), "cudaSetDevice");
    f->groupMem.release();
    f->dRowGroup = f->groupMem.upload(gid);
    f->dGroupNorms = f->groupMem.alloc<double>((size_t)2 * ngroups * amp::multi_max_vectors());
    f->ngroups = ngroups;
    return (int)AMP_OK;
  });
}

int amp_solve_gmres(amp_factor *f, const double *b, double *x, int on_device, const amp_gmres_opts *opts,
                    amp_gmres_stats *stats) {
  return guarded([&] {
    if (!f) return fail(AMP_INVALID, "null handle");
    if (f->kind == AMP_LDLT_COMPLEX) return fail(AMP_INVALID, "a complex-symmetric factor: use the amp_c* entry points");
    if (!f->ok) return fail(AMP_NO_FACTOR, "solveNumeric: no successful numeric factorization");
    amp_gmres_opts o{1e-10, 40, 400};
    if (opts) o = *opts;
    if (o.restart < 1 || o.max_iter < 0) return fail(AMP_INVALID, "gmres: restart >= 1 and maxIter >= 0 required");
    const amp::Plan &P = f->plan->P;
    const int64_t n = P.n;
    amp_gmres_stats res{0.0, 0, 1};
    if (n == 0) {
      if (stats) *stats = res;
      return (int)AMP_OK;
    }
    ck(cudaSetDevice(f->plan->device), "cudaSetDevice");
    ensure_solve_ws(f, 1);
    cudaStream_t st = f->stream;
    const int m = o.restart;
    // workspace (kept by the factor): V (m + 1 vectors), Z (m), r, w, x, b, dot partials and results
    if (m > f->gmresCap) {
      f->gmem.release();
      f->gV = f->gmem.alloc<double>((size_t)(m + 1) * n);
      f->gZ = f->gmem.alloc<double>((size_t)m * n);
      f->gR = f->gmem.alloc<double>((size_t)n);
      f->gW = f->gmem.alloc<double>((size_t)n);
      f->gX = f->gmem.alloc<double>((size_t)n);
      f->gB = f->gmem.alloc<double>((size_t)n);
      f->gPart = f->gmem.alloc<double>((size_t)(m + 1) * amp::dot_partials());
      f->gH = f->gmem.alloc<double>(3 * ((size_t)m + 1));  // both Gram-Schmidt passes and the norm
      f->gmresCap = m;
    }
    double *V = f->gV, *Z = f->gZ, *r = f->gR, *w = f->gW, *xb = f->gX, *bb = f->gB, *part = f->gPart, *dh = f->gH;
    ck(cudaMemcpyAsync(bb, b, sizeof(double) * n, on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st),
       "copy b");
    ck(cudaMemsetAsync(xb, 0, sizeof(double) * n, st), "zero x");
    std::vector<double> h(m + 1), H((size_t)(m + 1) * m), cs(m), sn(m), g(m + 1), y(m);
    auto dots = [&](const double *Vs, int nv, const double *v) {  // h[0..nv) = Vs[j] . v (synchronises)
      timed(f, K_KRYLOV, 2.0 * n * nv, 8.0 * n * (nv + 1),
            [&] { return amp::launch_dots(Vs, nv, n, v, part, dh, st); });
      ck(cudaMemcpyAsync(h.data(), dh, sizeof(double) * nv, cudaMemcpyDeviceToHost, st), "dots");
      ck(cudaStreamSynchronize(st), "dots");
    };
    auto residual = [&]() {  // r = b - A x, returns ||r||
      timed(f, K_RESIDUAL, 2.0 * P.patNnz, 12.0 * P.patNnz + 16.0 * n, [&] {
        amp::launch_matvec((int)n, f->plan->dRowptr, f->plan->dColidx, f->dValues, xb, w, 1, st);
      });
      timed(f, K_KRYLOV, (double)n, 24.0 * n, [&] { amp::launch_sub_from(r, bb, w, n, st); });
      dots(r, 1, r);
      return std::sqrt(h[0]);
    };
    auto precond = [&](const double *v, double *z) {  // z = M^-1 v (the factor's solve)
      device_solve(f, v, z);
      ck(cudaGetLastError(), "kernel launch");
    };
    dots(bb, 1, bb);
    double bnorm = std::sqrt(h[0]);
    if (bnorm == 0) bnorm = 1;
    ck(cudaMemcpyAsync(r, bb, sizeof(double) * n, cudaMemcpyDeviceToDevice, st), "r = b");
    double beta = bnorm == 1 && h[0] == 0 ? 0.0 : std::sqrt(h[0]);
    double relres = beta / bnorm;
    int iters = 0;
    while (relres > o.tol && iters < o.max_iter) {
      timed(f, K_KRYLOV, (double)n, 16.0 * n, [&] { amp::launch_scale_to(V, r, 1.0 / beta, n, st); });
      std::fill(g.begin(), g.end(), 0.0);
      g[0] = beta;
      int k = 0;
      for (; k < m && iters < o.max_iter; k++) {
        iters++;
        precond(V + (int64_t)k * n, Z + (int64_t)k * n);
        timed(f, K_RESIDUAL, 2.0 * P.patNnz, 12.0 * P.patNnz + 16.0 * n, [&] {
          amp::launch_matvec((int)n, f->plan->dRowptr, f->plan->dColidx, f->dValues, Z + (int64_t)k * n, w, 1, st);
        });
        // classical Gram-Schmidt twice (as stable as modified Gram-Schmidt, two reductions per iteration); the
        // coefficients of each pass stay on the device for its update, the next vector is scaled there too, and the
        // host reads all of them with one synchronisation per iteration
        double *dh1 = dh, *dh2 = dh + (m + 1), *dnn = dh + 2 * (m + 1);
        for (int pass = 0; pass < 2; pass++) {
          double *dp = pass ? dh2 : dh1;
          timed(f, K_KRYLOV, 2.0 * n * (k + 1), 8.0 * n * (k + 2),
                [&] { return amp::launch_dots(V, k + 1, n, w, part, dp, st); });
          timed(f, K_KRYLOV, 2.0 * n * (k + 1), 8.0 * n * (k + 3),
                [&] { amp::launch_gs_update(w, V, dp, k + 1, n, st); });
        }
        timed(f, K_KRYLOV, 2.0 * n, 8.0 * n, [&] { return amp::launch_dots(w, 1, n, w, part, dnn, st); });
        timed(f, K_KRYLOV, (double)n, 16.0 * n,
              [&] { amp::launch_scale_by_norm(V + (int64_t)(k + 1) * n, w, dnn, n, st); });
        std::vector<double> hb(3 * ((size_t)m + 1));
        ck(cudaMemcpyAsync(hb.data(), dh, sizeof(double) * 3 * (m + 1), cudaMemcpyDeviceToHost, st), "dots");
        ck(cudaStreamSynchronize(st), "dots");
        for (int j = 0; j <= k; j++) H[(size_t)j * m + k] = (0.0 + hb[j]) + hb[(m + 1) + j];
        const double hn = std::sqrt(hb[2 * (m + 1)]);
        H[(size_t)(k + 1) * m + k] = hn;
        for (int j = 0; j < k; j++) {  // apply the previous Givens rotations
          const double a = H[(size_t)j * m + k], c = H[(size_t)(j + 1) * m + k];
          H[(size_t)j * m + k] = cs[j] * a + sn[j] * c;
          H[(size_t)(j + 1) * m + k] = -sn[j] * a + cs[j] * c;
        }
        const double a = H[(size_t)k * m + k], c = H[(size_t)(k + 1) * m + k];
        double d = std::hypot(a, c);
        if (d == 0) d = 1e-300;
        cs[k] = a / d;
        sn[k] = c / d;
        H[(size_t)k * m + k] = d;
        H[(size_t)(k + 1) * m + k] = 0.0;
        g[k + 1] = -sn[k] * g[k];
        g[k] = cs[k] * g[k];
        relres = std::fabs(g[k + 1]) / bnorm;
        if (relres <= o.tol || hn == 0) {
          k++;
          break;
        }
      }
      for (int i = k - 1; i >= 0; i--) {  // back substitution, then x += Z y
        double s = g[i];
        for (int j = i + 1; j < k; j++) s -= H[(size_t)i * m + j] * y[j];
        y[i] = s / H[(size_t)i * m + i];
      }
      ck(cudaMemcpyAsync(dh, y.data(), sizeof(double) * k, cudaMemcpyHostToDevice, st), "y");
      timed(f, K_KRYLOV, 2.0 * n * k, 8.0 * n * (k + 2), [&] { amp::launch_combine_add(xb, Z, dh, k, n, st); });
      if (relres <= o.tol || iters >= o.max_iter) break;
      beta = residual();
      relres = beta / bnorm;
    }
    res.rel_residual = residual() / bnorm;
    res.iterations = iters;
    res.converged = res.rel_residual <= std::max(o.tol * 10, 1e-14);
    ck(cudaMemcpyAsync(x, xb, sizeof(double) * n, on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, st),
       "copy x");
    ck(cudaStreamSynchronize(st), "gmres");
    if (int rc = solve_status(f)) return rc;
    if (stats) *stats = res;
    return (int)AMP_OK;
  });
}

int amp_factor_download(const amp_factor *f, double *Lx, double *D) {
  return guarded([&] {
    if (!f) return fail(AMP_INVALID, "null handle");
    if (f->kind == AMP_LDLT_COMPLEX) return fail(AMP_INVALID, "a complex-symmetric factor: use the amp_c* entry points");
    const amp::Plan &P = f->plan->P;
    ck(cudaSetDevice(f->plan->device), "cudaSetDevice");
    if (Lx && P.nnzLStored && f->dLx)
      ck(cudaMemcpy(Lx, f->dLx, sizeof(double) * P.nnzLStored, cudaMemcpyDeviceToHost), "copy Lx");
    if (Lx && P.nnzLStored && f->dL32) {
      std::vector<float> tmp(P.nnzLStored);
      ck(cudaMemcpy(tmp.data(), f->dL32, sizeof(float) * P.nnzLStored, cudaMemcpyDeviceToHost), "copy Lx");
      for (int64_t i = 0; i < P.nnzLStored; i++) Lx[i] = tmp[i];
    }
    if (D && P.n) ck(cudaMemcpy(D, f->dD, sizeof(double) * P.n, cudaMemcpyDeviceToHost), "copy D");
    return (int)AMP_OK;
  });
}

int amp_factor_download_pivots(const amp_factor *f, double *Doff, int32_t *piv) {
  return guarded([&] {
    if (!f) return fail(AMP_INVALID, "null handle");
    if (!f->bk) return fail(AMP_INVALID, "download_pivots: not a Bunch-Kaufman factor");
    const amp::Plan &P = f->plan->P;
    ck(cudaSetDevice(f->plan->device), "cudaSetDevice");
    if (Doff && P.n) ck(cudaMemcpy(Doff, f->dDoff, sizeof(double) * P.n, cudaMemcpyDeviceToHost), "copy Doff");
    if (piv && P.n) ck(cudaMemcpy(piv, f->dPiv, sizeof(int32_t) * P.n, cudaMemcpyDeviceToHost), "copy piv");
    return (int)AMP_OK;
  });
}

void amp_factor_destroy(amp_factor *f) { delete f; }

int amp_factor_set_wait_limit(amp_factor *f, int64_t polls) {
  return guarded([&] {
    if (!f || polls < 0) return fail(AMP_INVALID, "set_wait_limit: null handle or negative bound");
    if (polls != f->waitSpins && f->factorGraph) {  // the captured factorization holds the old bound
      ck(cudaSetDevice(f->plan->device), "cudaSetDevice");
      ck(cudaStreamSynchronize(f->stream), "sync");
      ck(cudaGraphExecDestroy(f->factorGraph), "graph destroy");
      f->factorGraph = nullptr;
    }
    f->waitSpins = polls;
    return (int)AMP_OK;
  });
}

int amp_profile_enable(amp_factor *f, int enable) {
  if (!f) return fail(AMP_INVALID, "null handle");
  f->profiling = enable != 0;
  f->recs.clear();
  f->evUsed = 0;
  return AMP_OK;
}

int amp_profile_launches(amp_factor *f, int32_t *kinds, double *ms, double *flops, int32_t cap, int32_t *count) {
  return guarded([&] {
    if (!f) return fail(AMP_INVALID, "null handle");
    ck(cudaStreamSynchronize(f->stream), "sync");
    int c = 0;
    for (auto &r : f->recs) {
      if (c >= cap) break;
      float t = 0;
      ck(cudaEventElapsedTime(&t, r.a, r.b), "elapsed");
      kinds[c] = r.kind;
      ms[c] = t;
      flops[c] = r.flops;
      c++;
    }
    if (count) *count = c;
    return (int)AMP_OK;
  });
}

int amp_profile_read(amp_factor *f, amp_kernel_stat *stats, int32_t cap, int32_t *count) {
  return guarded([&] {
    if (!f) return fail(AMP_INVALID, "null handle");
    ck(cudaStreamSynchronize(f->stream), "sync");
    std::vector<amp_kernel_stat> acc(K_NKINDS);
    for (int k = 0; k < K_NKINDS; k++) {
      std::memset(&acc[k], 0, sizeof(amp_kernel_stat));
      std::snprintf(acc[k].name, sizeof acc[k].name, "%s", kKindNames[k]);
    }
    for (auto &r : f->recs) {
      float ms = 0;
      ck(cudaEventElapsedTime(&ms, r.a, r.b), "elapsed");
      acc[r.kind].launches += r.kernels;
      acc[r.kind].ms += ms;
      acc[r.kind].flops += r.flops;
      acc[r.kind].bytes += r.bytes;
    }
    int c = 0;
    for (int k = 0; k < K_NKINDS && c < cap; k++)
      if (acc[k].launches) stats[c++] = acc[k];
    if (count) *count = c;
    f->recs.clear();
    f->evUsed = 0;
    return (int)AMP_OK;
  });
}


int amp_cfactor_create(amp_plan *pl, amp_factor **out) {
  return guarded([&] {
    if (!pl || !out) return fail(AMP_INVALID, "null handle");
    *out = nullptr;
    ck(cudaSetDevice(pl->device), "cudaSetDevice");
    if (!pl->uploaded) {
      upload_plan(pl);
      pl->dRowptr = pl->mem.upload(pl->rowptr);
      pl->dColidx = pl->mem.upload(pl->colidx);
      pl->uploaded = true;
    }
    upload_cx(pl);
    auto *f = new amp_factor_s();
    f->plan = pl;
    f->kind = AMP_LDLT_COMPLEX;
    f->precision = AMP_FP64;
    try {
      ck(cudaStreamCreateWithFlags(&f->stream, cudaStreamNonBlocking), "cudaStreamCreate");
      ck(cudaEventCreate(&f->ev0), "cudaEventCreate");
      ck(cudaEventCreate(&f->ev1), "cudaEventCreate");
      const amp::Plan &P = pl->P;
      const size_t n = (size_t)std::max(1, P.n);
      f->dLc = f->mem.alloc<amp::cplx>((size_t)P.nnzLStored);
      f->dUc = f->mem.alloc<amp::cplx>((size_t)P.arenaDoubles);
      f->dWc = f->mem.alloc<amp::cplx>((size_t)P.nnzLStored);
      f->dDc = f->mem.alloc<amp::cplx>(n);
      f->dValC = f->mem.alloc<amp::cplx>((size_t)P.patNnz);
      for (amp::cplx **v : {&f->dYc, &f->dBc, &f->dXc, &f->dRc, &f->dDXc}) *v = f->mem.alloc<amp::cplx>(n);
      for (double **v : {&f->dBr, &f->dBi, &f->dXr, &f->dXi}) *v = f->mem.alloc<double>(n);
      f->dNormsC = f->mem.alloc<double>(2);
      f->dScal = f->mem.alloc<double>(2);
      f->dCounts = f->mem.alloc<int>(2);
      f->dStatus = f->mem.alloc<unsigned long long>(1);
      f->dCxFlags = f->mem.alloc<int>((size_t)std::max(1, pl->cx.nGroupFlags + pl->cx.nGroupTickets));
      init_device_once(pl->device);
    } catch (...) {
      delete f;
      throw;
    }
    *out = f;
    return (int)AMP_OK;
  });
}

int amp_cfactor_numeric(amp_factor *f, const double *re, const double *im, int64_t nvalues, int values_on_device,
                        double pivot_tol, amp_factor_result *res) {
  return guarded([&] {
    if (int rc = require_complex(f)) return rc;
    const amp::Plan &P = f->plan->P;
    if (nvalues != P.patNnz)
      return fail(AMP_BAD_LENGTH, "factorNumeric: " + std::to_string(nvalues) + " values for a pattern with " +
                                      std::to_string(P.patNnz) + " entries");
    if (nvalues > 0 && (!re || !im)) return fail(AMP_INVALID, "factor: null values");
    ck(cudaSetDevice(f->plan->device), "cudaSetDevice");
    f->ok = false;
    amp_factor_result r{};
    r.fail_column = -1;
    if (P.n == 0) {
      f->ok = true;
      r.ok = 1;
      if (res) *res = r;
      return (int)AMP_OK;
    }
    cudaStream_t st = f->stream;
    const double *dre = re, *dim = im;
    DevMem tmp;
    if (!values_on_device) {
      double *a = tmp.alloc<double>((size_t)nvalues), *b = tmp.alloc<double>((size_t)nvalues);
      ck(cudaMemcpyAsync(a, re, sizeof(double) * nvalues, cudaMemcpyHostToDevice, st), "copy re");
      ck(cudaMemcpyAsync(b, im, sizeof(double) * nvalues, cudaMemcpyHostToDevice, st), "copy im");
      dre = a;
      dim = b;
    }
    amp::launch_cpack(nvalues, dre, dim, f->dValC, st);
    f->hasValues = true;
    ck(cudaMemcpyAsync(f->dScal, &pivot_tol, sizeof(double), cudaMemcpyHostToDevice, st), "copy pivotTol");
    ck(cudaEventRecord(f->ev0, st), "event");
    enqueue_cfactor(f);
    ck(cudaGetLastError(), "kernel launch");
    ck(cudaEventRecord(f->ev1, st), "event");
    unsigned long long status = 0;
    int counts[2] = {0, 0};
    ck(cudaMemcpyAsync(&status, f->dStatus, sizeof status, cudaMemcpyDeviceToHost, st), "copy status");
    ck(cudaMemcpyAsync(counts, f->dCounts, sizeof counts, cudaMemcpyDeviceToHost, st), "copy counts");
    ck(cudaStreamSynchronize(st), "factor");
    float ms = 0;
    cudaEventElapsedTime(&ms, f->ev0, f->ev1);
    r.ms = ms;
    r.n_perturbed = counts[1];
    if (status == amp::kStatusOk) {
      r.ok = 1;
      f->ok = true;
    } else if (((status >> 24) & 0xff) == 3) {
      if (res) *res = r;
      return fail(AMP_DEVICE_TIMEOUT, "factorNumeric: a device wait timed out");
    } else {
      r.ok = 0;
      r.fail_column = (int32_t)(status >> 32);
    }
    if (res) *res = r;
    return (int)AMP_OK;
  });
}

int amp_csolve_refined(amp_factor *f, const double *br, const double *bi, int32_t nrhs, double *xr, double *xi,
                       int on_device, const amp_refine_opts *opts, amp_refine_stats *stats) {
  return guarded([&] {
    if (int rc = require_complex(f)) return rc;
    if (!f->ok) return fail(AMP_NO_FACTOR, "solveNumeric: no successful numeric factorization");
    const amp::Plan &P = f->plan->P;
    const int n = P.n;
    amp_refine_stats stt{0.0, 0};
    if (nrhs <= 0 || n == 0) {
      if (stats) *stats = stt;
      return (int)AMP_OK;
    }
    ck(cudaSetDevice(f->plan->device), "cudaSetDevice");
    cudaStream_t st = f->stream;
    const int *perm = f->plan->dp.perm;
    const size_t vb = sizeof(double) * (size_t)n;
    for (int k = 0; k < nrhs; k++) {
      const double *kr = br + (size_t)k * n, *ki = bi + (size_t)k * n;
      if (!on_device) {
        ck(cudaMemcpyAsync(f->dBr, kr, vb, cudaMemcpyHostToDevice, st), "copy b");
        ck(cudaMemcpyAsync(f->dBi, ki, vb, cudaMemcpyHostToDevice, st), "copy b");
        kr = f->dBr;
        ki = f->dBi;
      }
      amp::launch_cpack(n, kr, ki, f->dBc, st);
      amp::launch_cpermute_vec(n, f->dBc, perm, f->dYc, true, st);
      csolve_permuted(f, f->dYc);
      amp::launch_cpermute_vec(n, f->dYc, perm, f->dXc, false, st);
      int steps = 0;
      double rel = 0.0;
      for (; opts; steps++) {  // complexSolveRefined: residual against the unperturbed values, up to maxSteps
        ck(cudaMemsetAsync(f->dNormsC, 0, 2 * sizeof(double), st), "memset");
        timed(f, K_RESIDUAL, 8.0 * P.patNnz, 32.0 * P.patNnz, [&] {
          amp::launch_cresidual(n, f->plan->dRowptr, f->plan->dColidx, f->dValC, f->dXc, f->dBc, f->dRc, f->dNormsC,
                                st);
        });
        double nr[2];
        ck(cudaMemcpyAsync(nr, f->dNormsC, sizeof nr, cudaMemcpyDeviceToHost, st), "norms");
        ck(cudaStreamSynchronize(st), "residual");
        double bn = std::sqrt(nr[1]);
        if (bn == 0 || std::isnan(bn)) bn = 1;
        rel = std::sqrt(nr[0]) / bn;
        if (rel < opts->tol || steps >= opts->max_steps) break;
        amp::launch_cpermute_vec(n, f->dRc, perm, f->dYc, true, st);
        csolve_permuted(f, f->dYc);
        amp::launch_cpermute_vec(n, f->dYc, perm, f->dDXc, false, st);
        amp::launch_caxpy(n, f->dXc, f->dDXc, st);
      }
      double *ox = xr + (size_t)k * n, *oi = xi + (size_t)k * n;
      amp::launch_cunpack(n, f->dXc, on_device ? ox : f->dXr, on_device ? oi : f->dXi, st);
      if (!on_device) {
        ck(cudaMemcpyAsync(ox, f->dXr, vb, cudaMemcpyDeviceToHost, st), "copy x");
        ck(cudaMemcpyAsync(oi, f->dXi, vb, cudaMemcpyDeviceToHost, st), "copy x");
      }
      ck(cudaGetLastError(), "kernel launch");
      ck(cudaStreamSynchronize(st), "solve");
      stt.rel_residual = std::max(stt.rel_residual, rel);
      stt.steps = std::max(stt.steps, steps);
    }
    if (stats) *stats = stt;
    return (int)AMP_OK;
  });
}

int amp_csolve(amp_factor *f, const double *br, const double *bi, int32_t nrhs, double *xr, double *xi,
               int on_device) {
  return amp_csolve_refined(f, br, bi, nrhs, xr, xi, on_device, nullptr, nullptr);
}

int amp_cfactor_download(const amp_factor *f, double *Lr, double *Li, double *Dr, double *Di) {
  return guarded([&] {
    if (int rc = require_complex(f)) return rc;
    const amp::Plan &P = f->plan->P;
    ck(cudaSetDevice(f->plan->device), "cudaSetDevice");
    auto split = [&](const amp::cplx *src, int64_t len, double *re, double *im) {
      if ((!re && !im) || len == 0) return;
      std::vector<amp::cplx> h((size_t)len);
      ck(cudaMemcpy(h.data(), src, sizeof(amp::cplx) * len, cudaMemcpyDeviceToHost), "copy factor");
      for (int64_t i = 0; i < len; i++) {
        if (re) re[i] = h[i].re;
        if (im) im[i] = h[i].im;
      }
    };
    split(f->dLc, P.nnzLStored, Lr, Li);
    split(f->dDc, P.n, Dr, Di);
    return (int)AMP_OK;
  });
}

int amp_assembly_create(int kind, int32_t n, const int32_t *rowptr, const int32_t *colidx, int32_t nnodes,
                        const double *coords, int64_t nelem, const int32_t *conn, const int32_t *dofs, int device,
                        amp_assembly **out) {
  return guarded([&] {
    if (!out || n < 0 || nnodes < 0 || nelem < 0 || !rowptr || (nelem > 0 && (!conn || !coords || !dofs)))
      return fail(AMP_INVALID, "assembly: invalid arguments");
    if (kind != AMP_ELEM_P1_TRI_SCALAR && kind != AMP_ELEM_P1_TET_ELASTIC)
      return fail(AMP_INVALID, "assembly: unknown element kind");
    *out = nullptr;
    const int k = kind == AMP_ELEM_P1_TRI_SCALAR ? 3 : 4, bs = kind == AMP_ELEM_P1_TRI_SCALAR ? 1 : 3;
    const int dim = kind == AMP_ELEM_P1_TRI_SCALAR ? 2 : 3, nd = k * bs;
    const int64_t nnz = n ? rowptr[n] : 0;
    if ((uint64_t)nelem * nd * nd >= (1ull << 32)) return fail(AMP_INVALID, "assembly: mesh too large");
    // element slots (elementSlots / blockElementSlots): slot of local entry (r, c) of element e, or -1
    std::vector<int64_t> cnt(nnz + 1, 0);
    std::vector<int> slot((size_t)nelem * nd * nd);
    for (int64_t e = 0; e < nelem; e++)
      for (int r = 0; r < nd; r++) {
        const int vr = conn[k * e + r / bs];
        if (vr < 0 || vr >= nnodes) return fail(AMP_INVALID, "assembly: connectivity out of range");
        const int row = dofs[(int64_t)vr * bs + r % bs];
        for (int c = 0; c < nd; c++) {
          const int vc = conn[k * e + c / bs];
          if (vc < 0 || vc >= nnodes) return fail(AMP_INVALID, "assembly: connectivity out of range");
          const int col = dofs[(int64_t)vc * bs + c % bs];
          int s = -1;
          if (row >= 0 && col >= 0) {
            if (row >= n || col >= n) return fail(AMP_INVALID, "assembly: DOF map out of range");
            const int32_t *b0 = colidx + rowptr[row], *b1 = colidx + rowptr[row + 1];
            const int32_t *it = std::lower_bound(b0, b1, col);
            if (it == b1 || *it != col)
              return fail(AMP_PATTERN_MISMATCH, "assembly: element " + std::to_string(e) + " couples rows " +
                                                    std::to_string(row) + " and " + std::to_string(col) +
                                                    " outside the pattern");
            s = rowptr[row] + (int)(it - b0);
            cnt[s + 1]++;
          }
          slot[((size_t)e * nd + r) * nd + c] = s;
        }
      }
    for (int64_t s = 0; s < nnz; s++) cnt[s + 1] += cnt[s];
    std::vector<uint32_t> gidx(cnt[nnz]);
    {  // contributions of every slot in increasing element order
      std::vector<int64_t> fill(cnt.begin(), cnt.end() - 1);
      for (int64_t e = 0; e < nelem; e++)
        for (int q = 0; q < nd * nd; q++) {
          const int s = slot[(size_t)e * nd * nd + q];
          if (s >= 0) gidx[fill[s]++] = (uint32_t)(e * nd * nd + q);
        }
    }
    auto *a = new amp_assembly_s();
    try {
      a->kind = kind;
      a->device = device;
      a->nd = nd;
      a->ncoef = kind == AMP_ELEM_P1_TRI_SCALAR ? 1 : 2;
      a->nelem = nelem;
      a->nnz = nnz;
      ck(cudaSetDevice(device), "cudaSetDevice");
      a->dConn = a->mem.upload(std::vector<int>(conn, conn + (size_t)nelem * k));
      a->dCoords = a->mem.upload(std::vector<double>(coords, coords + (size_t)nnodes * dim));
      a->dGptr = a->mem.upload(cnt);
      a->dGidx = a->mem.upload(gidx);
      a->dKe = a->mem.alloc<double>((size_t)nelem * nd * nd);
      a->dCoef = a->mem.alloc<double>((size_t)nelem * a->ncoef);
      a->dValues = a->mem.alloc<double>((size_t)nnz);
    } catch (...) {
      delete a;
      throw;
    }
    *out = a;
    return (int)AMP_OK;
  });
}

int amp_assemble(amp_assembly *a, const double *coef, int coef_on_device, double *values, int values_on_device,
                 void *stream) {
  return guarded([&] {
    if (!a || (a->nelem > 0 && !coef) || (a->nnz > 0 && !values)) return fail(AMP_INVALID, "assemble: null argument");
    ck(cudaSetDevice(a->device), "cudaSetDevice");
    cudaStream_t st = (cudaStream_t)stream;
    const double *dCoef = coef;
    if (!coef_on_device && a->nelem > 0) {
      ck(cudaMemcpyAsync(a->dCoef, coef, sizeof(double) * a->nelem * a->ncoef, cudaMemcpyHostToDevice, st),
         "copy coefficients");
      dCoef = a->dCoef;
    }
    double *dV = values_on_device ? values : a->dValues;
    amp::launch_assemble_values(a->kind, a->nelem, a->dConn, a->dCoords, dCoef, a->dKe, a->nnz, a->dGptr, a->dGidx,
                                dV, st);
    ck(cudaGetLastError(), "kernel launch");
    if (!values_on_device && a->nnz > 0)
      ck(cudaMemcpyAsync(values, dV, sizeof(double) * a->nnz, cudaMemcpyDeviceToHost, st), "copy values");
    ck(cudaStreamSynchronize(st), "assemble");
    return (int)AMP_OK;
  });
}

void amp_assembly_destroy(amp_assembly *a) { delete a; }

int amp_factor_set_mass(amp_factor *f, const double *mvalues, int64_t nvalues, int on_device) {
  return guarded([&] {
    if (!f || (nvalues > 0 && !mvalues)) return fail(AMP_INVALID, "set_mass: null handle or values");
    if (f->kind == AMP_LDLT_COMPLEX) return fail(AMP_INVALID, "a complex-symmetric factor: use the amp_c* entry points");
    const amp::Plan &P = f->plan->P;
    if (nvalues != P.patNnz)
      return fail(AMP_BAD_LENGTH, "setMass: " + std::to_string(nvalues) + " values for a pattern with " +
                                      std::to_string(P.patNnz) + " entries");
    ck(cudaSetDevice(f->plan->device), "cudaSetDevice");
    if (!f->dMass) f->dMass = f->massMem.alloc<double>((size_t)P.patNnz);
    if (nvalues)
      ck(cudaMemcpy(f->dMass, mvalues, sizeof(double) * nvalues,
                    on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice), "copy mass");
    return (int)AMP_OK;
  });
}

int amp_shift_invert_apply(amp_factor *f, const double *X, int32_t m, double *Y, int on_device) {
  return guarded([&] {
    if (!f) return fail(AMP_INVALID, "null handle");
    if (f->kind == AMP_LDLT_COMPLEX) return fail(AMP_INVALID, "a complex-symmetric factor: use the amp_c* entry points");
    if (!f->ok) return fail(AMP_NO_FACTOR, "solveNumeric: no successful numeric factorization");
    if (!f->dMass) return fail(AMP_INVALID, "shift-invert: no mass values (amp_factor_set_mass)");
    const amp::Plan &P = f->plan->P;
    if (m <= 0 || P.n == 0) return (int)AMP_OK;
    ck(cudaSetDevice(f->plan->device), "cudaSetDevice");
    const size_t len = (size_t)P.n * m;
    DevMem tmp;
    double *dT = tmp.alloc<double>(len);
    const double *dX = X;
    double *dY = Y;
    if (!on_device) {
      double *a = tmp.alloc<double>(len), *b = tmp.alloc<double>(len);
      ck(cudaMemcpy(a, X, sizeof(double) * len, cudaMemcpyHostToDevice), "copy X");
      dX = a;
      dY = b;
    }
    if (int rc = device_shift_invert(f, dX, m, dY, dT)) return rc;
    if (!on_device) ck(cudaMemcpy(Y, dY, sizeof(double) * len, cudaMemcpyDeviceToHost), "copy Y");
    return (int)AMP_OK;
  });
}

int amp_eigen_block_arnoldi(amp_factor *f, const amp_eigen_opts *opts, double *mu, double *vecs, int on_device,
                            amp_eigen_stats *stats) {
  return guarded([&] {
    if (!f || !opts || !mu) return fail(AMP_INVALID, "eigen: null argument");
    if (f->kind == AMP_LDLT_COMPLEX) return fail(AMP_INVALID, "a complex-symmetric factor: use the amp_c* entry points");
    if (!f->ok) return fail(AMP_NO_FACTOR, "solveNumeric: no successful numeric factorization");
    if (!f->dMass) return fail(AMP_INVALID, "eigen: no mass values (amp_factor_set_mass)");
    const amp::Plan &P = f->plan->P;
    const int64_t n = P.n;
    const amp_eigen_opts o = *opts;
    const int b = std::max(1, o.block_size), nw = o.n_want;
    if (nw < 1 || n < 2) return fail(AMP_INVALID, "eigen: need n_want >= 1 and n >= 2");
    // basis per cycle p (a multiple of b) as the reference sizes it (arnoldi.mjs:37-41), capped by n
    int p = std::max(o.max_basis > 0 ? o.max_basis : std::max(30, 2 * nw + 12), nw + 3 * b);
    p = (p + b - 1) / b * b;
    if (p + b > n) p = (int)((n - b) / b * b);
    if (p < nw + b) return fail(AMP_INVALID, "eigen: the system is too small for n_want Ritz pairs");
    const int nKeep = std::max(nw, std::min(nw + std::max(2, nw), p - 2 * b));
    const double tol = o.tol > 0 ? o.tol : 1e-10;
    const int maxRestarts = o.max_restarts > 0 ? o.max_restarts : 60;
    ck(cudaSetDevice(f->plan->device), "cudaSetDevice");
    cudaStream_t st = f->stream;
    const auto t0 = std::chrono::steady_clock::now();
    // workspace: V, MV ((p + b) n each), W, MW, T (b n each), U (nKeep n), dot partials
    const int64_t need = (int64_t)(2 * (p + b) + 3 * b + nKeep) * n + (int64_t)(p + b) * (amp::dot_partials() + 1);
    if (need > f->eigCap) {
      f->eigMem.release();
      f->eigMem.alloc<double>((size_t)need);
      f->eigCap = need;
    }
    double *base = (double *)f->eigMem.ptrs[0];
    double *V = base, *MV = V + (p + b) * n, *W = MV + (p + b) * n, *MW = W + b * n, *T = MW + b * n,
           *U = T + b * n, *part = U + (int64_t)nKeep * n, *dh = part + (int64_t)(p + b) * amp::dot_partials();
    EigenWork ew{f, n, part, dh, {}};
    // start block: the reference's LCG (arnoldi.mjs seededRandom), vector after vector
    {
      uint32_t s = o.seed ? o.seed : 20261014u;
      std::vector<double> x0((size_t)b * n);
      for (auto &v : x0) {
        s = s * 1664525u + 1013904223u;
        v = (double)s / 4294967296.0 - 0.5;
      }
      ck(cudaMemcpy(V, x0.data(), sizeof(double) * x0.size(), cudaMemcpyHostToDevice), "start block");
    }
    int opVectors = 0;
    // M-orthonormalise the b vectors at X (M X at MX): X <- X R^-1 with R^T R = X^T M X; R to Rout (b x b,
    // row-major) when given. false when the block is (numerically) dependent.
    auto orthonormalise = [&](double *X, double *MX, std::vector<double> *Rout) -> bool {
      amp::launch_matvec((int)n, f->plan->dRowptr, f->plan->dColidx, f->dMass, X, MX, b, st);
      std::vector<double> G((size_t)b * b), R((size_t)b * b, 0.0);
      for (int j = 0; j < b; j++) {
        const auto &h = ew.dots(X, b, MX + (int64_t)j * n);
        for (int i = 0; i < b; i++) G[(size_t)i * b + j] = h[i];
      }
      for (int j = 0; j < b; j++) {  // Cholesky G = R^T R (R upper)
        double d = G[(size_t)j * b + j];
        for (int k = 0; k < j; k++) d -= R[(size_t)k * b + j] * R[(size_t)k * b + j];
        if (!(d > 1e-28 * std::max(1.0, G[0]))) return false;
        R[(size_t)j * b + j] = std::sqrt(d);
        for (int i = j + 1; i < b; i++) {
          double s2 = G[(size_t)j * b + i];
          for (int k = 0; k < j; k++) s2 -= R[(size_t)k * b + j] * R[(size_t)k * b + i];
          R[(size_t)j * b + i] = s2 / R[(size_t)j * b + j];
        }
      }
      std::vector<double> Ri((size_t)b * b, 0.0);  // R^-1 (upper)
      for (int c = 0; c < b; c++) {
        Ri[(size_t)c * b + c] = 1.0 / R[(size_t)c * b + c];
        for (int i = c - 1; i >= 0; i--) {
          double s2 = 0.0;
          for (int k = i + 1; k <= c; k++) s2 += R[(size_t)i * b + k] * Ri[(size_t)k * b + c];
          Ri[(size_t)i * b + c] = -s2 / R[(size_t)i * b + i];
        }
      }
      for (double *Z : {X, MX}) {
        for (int c = 0; c < b; c++) {
          std::vector<double> coef(b);
          for (int j = 0; j < b; j++) coef[j] = Ri[(size_t)j * b + c];
          ew.combine(T + (int64_t)c * n, Z, coef, b);
        }
        ck(cudaMemcpyAsync(Z, T, sizeof(double) * b * n, cudaMemcpyDeviceToDevice, st), "copy block");
      }
      if (Rout) *Rout = R;
      return true;
    };
    if (!orthonormalise(V, MV, nullptr)) return fail(AMP_INVALID, "eigen: degenerate start block");
    // H: projected matrix, (p + b) x p row-major; ncur basis vectors, the last block the one to expand
    std::vector<double> H((size_t)(p + b) * p, 0.0);
    int ncur = b, restarts = 0;
    bool converged = false, exhausted = false;
    std::vector<double> w, Q, res;
    std::vector<int> order;
    int pc = 0;  // projected size of the last Rayleigh-Ritz
    for (;;) {
      // expand the last block until the basis holds p + b vectors (or the Krylov space is exhausted)
      while (ncur < p + b) {
        const int c0 = ncur - b;
        if (int rc = device_shift_invert(f, V + (int64_t)c0 * n, b, W, T)) return rc;
        opVectors += b;
        for (int c = 0; c < b; c++) {  // two passes of block Gram-Schmidt in the M inner product (DGKS)
          double *wc = W + (int64_t)c * n;
          for (int pass = 0; pass < 2; pass++) {
            const auto &h = ew.dots(MV, ncur, wc);
            std::vector<double> hv(h.begin(), h.begin() + ncur);
            ck(cudaMemcpyAsync(dh, hv.data(), sizeof(double) * ncur, cudaMemcpyHostToDevice, st), "h");
            amp::launch_gs_update(wc, V, dh, ncur, n, st);
            ck(cudaStreamSynchronize(st), "gs");
            for (int i = 0; i < ncur; i++) H[(size_t)i * p + c0 + c] += hv[i];
          }
        }
        std::vector<double> R;
        if (!orthonormalise(W, MW, &R)) {  // an invariant subspace: the Ritz values of the basis are exact
          exhausted = true;
          break;
        }
        for (int i = 0; i < b; i++)
          for (int c = 0; c < b; c++) H[(size_t)(ncur + i) * p + c0 + c] = R[(size_t)i * b + c];
        ck(cudaMemcpyAsync(V + (int64_t)ncur * n, W, sizeof(double) * b * n, cudaMemcpyDeviceToDevice, st), "append");
        ck(cudaMemcpyAsync(MV + (int64_t)ncur * n, MW, sizeof(double) * b * n, cudaMemcpyDeviceToDevice, st),
           "append");
        ncur += b;
      }
      // Rayleigh-Ritz on the symmetrised projected matrix of the expanded columns
      pc = exhausted ? ncur : ncur - b;
      std::vector<double> S((size_t)pc * pc);
      for (int i = 0; i < pc; i++)
        for (int j = 0; j < pc; j++) S[(size_t)i * pc + j] = 0.5 * (H[(size_t)i * p + j] + H[(size_t)j * p + i]);
      jacobi_eigen(pc, S, w, Q);
      order.resize(pc);
      for (int i = 0; i < pc; i++) order[i] = i;
      std::stable_sort(order.begin(), order.end(), [&](int a, int c) { return std::fabs(w[a]) > std::fabs(w[c]); });
      // residual of Ritz pair i: || R_last y_i(last block) ||_M (the appended block is M-orthonormal)
      res.assign(pc, 0.0);
      if (!exhausted)
        for (int i = 0; i < pc; i++) {
          double s2 = 0.0;
          for (int r = 0; r < b; r++) {
            double t = 0.0;
            for (int c = 0; c < b; c++) t += H[(size_t)(pc + r) * p + pc - b + c] * Q[(size_t)(pc - b + c) * pc + i];
            s2 += t * t;
          }
          res[i] = std::sqrt(s2);
        }
      converged = true;
      for (int k = 0; k < std::min(nw, pc); k++)
        if (!(res[order[k]] <= tol * std::fabs(w[order[k]]))) converged = false;
      if (converged || exhausted || restarts >= maxRestarts || pc < nw) break;
      // thick restart: keep the nKeep Ritz vectors of largest |mu| and the residual block
      const int k = nKeep;
      for (double *Z : {V, MV}) {
        for (int c = 0; c < k; c++) {
          std::vector<double> coef(pc);
          for (int j = 0; j < pc; j++) coef[j] = Q[(size_t)j * pc + order[c]];
          ew.combine(U + (int64_t)c * n, Z, coef, pc);
        }
        ck(cudaMemcpyAsync(Z + (int64_t)k * n, Z + (int64_t)pc * n, sizeof(double) * b * n, cudaMemcpyDeviceToDevice,
                           st), "residual block");
        ck(cudaMemcpyAsync(Z, U, sizeof(double) * k * n, cudaMemcpyDeviceToDevice, st), "kept vectors");
      }
      std::vector<double> Hn((size_t)(p + b) * p, 0.0);
      for (int c = 0; c < k; c++) {
        Hn[(size_t)c * p + c] = w[order[c]];
        for (int r = 0; r < b; r++) {  // coupling of the residual block: R_last y_c(last block)
          double t = 0.0;
          for (int cc = 0; cc < b; cc++) t += H[(size_t)(pc + r) * p + pc - b + cc] * Q[(size_t)(pc - b + cc) * pc + order[c]];
          Hn[(size_t)(k + r) * p + c] = t;
        }
      }
      H.swap(Hn);
      ncur = k + b;
      restarts++;
    }
    const int nout = std::min(nw, pc);
    double worst = 0.0;
    for (int k = 0; k < nout; k++) {
      mu[k] = w[order[k]];
      worst = std::max(worst, res[order[k]] / std::max(std::fabs(w[order[k]]), 1e-300));
    }
    if (vecs) {  // Ritz vectors V y (M-orthonormal)
      for (int k = 0; k < nout; k++) {
        std::vector<double> coef(pc);
        for (int j = 0; j < pc; j++) coef[j] = Q[(size_t)j * pc + order[k]];
        ew.combine(U, V, coef, pc);
        ck(cudaMemcpy(vecs + (int64_t)k * n, U, sizeof(double) * n,
                      on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost), "copy Ritz vector");
      }
    }
    if (stats) {
      stats->converged = converged || exhausted;
      stats->restarts = restarts;
      stats->op_vectors = opVectors;
      stats->basis = p;
      stats->max_residual = worst;
      stats->ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
    return (int)AMP_OK;
  });
}

int amp_matvec_csr(int32_t n, const int32_t *rowptr, const int32_t *colidx, const double *values, const double *x,
                   int32_t nrhs, double *y, int device) {
  return guarded([&] {
    if (n < 0 || nrhs < 0 || (n > 0 && (!rowptr || !colidx || !values || !x || !y)))
      return fail(AMP_INVALID, "matVec: invalid arguments");
    if (n == 0 || nrhs == 0) return (int)AMP_OK;
    ck(cudaSetDevice(device), "cudaSetDevice");
    const int64_t nnz = rowptr[n];
    DevMem m;
    int *dRp = m.alloc<int>((size_t)n + 1), *dCi = m.alloc<int>((size_t)nnz);
    double *dV = m.alloc<double>((size_t)nnz), *dX = m.alloc<double>((size_t)n * nrhs),
           *dY = m.alloc<double>((size_t)n * nrhs);
    ck(cudaMemcpy(dRp, rowptr, sizeof(int) * ((size_t)n + 1), cudaMemcpyHostToDevice), "copy rowptr");
    ck(cudaMemcpy(dCi, colidx, sizeof(int) * (size_t)nnz, cudaMemcpyHostToDevice), "copy colidx");
    ck(cudaMemcpy(dV, values, sizeof(double) * (size_t)nnz, cudaMemcpyHostToDevice), "copy values");
    ck(cudaMemcpy(dX, x, sizeof(double) * (size_t)n * nrhs, cudaMemcpyHostToDevice), "copy x");
    amp::launch_matvec(n, dRp, dCi, dV, dX, dY, nrhs, nullptr);
    ck(cudaGetLastError(), "kernel launch");
    ck(cudaMemcpy(y, dY, sizeof(double) * (size_t)n * nrhs, cudaMemcpyDeviceToHost), "copy y");
    return (int)AMP_OK;
  });
}

int amp_matvec(amp_factor *f, const double *x, int32_t nrhs, double *y) {
  return guarded([&] {
    if (!f) return fail(AMP_INVALID, "null handle");
    if (f->kind == AMP_LDLT_COMPLEX) return fail(AMP_INVALID, "a complex-symmetric factor: use the amp_c* entry points");
    if (!f->hasValues) return fail(AMP_NO_FACTOR, "matVec: no values on the device (call amp_factor_numeric first)");
    const amp::Plan &P = f->plan->P;
    if (nrhs <= 0 || P.n == 0) return (int)AMP_OK;
    ck(cudaSetDevice(f->plan->device), "cudaSetDevice");
    ensure_solve_ws(f, nrhs);
    size_t bytes = sizeof(double) * (size_t)P.n * nrhs;
    ck(cudaMemcpyAsync(f->dB, x, bytes, cudaMemcpyHostToDevice, f->stream), "copy x");
    amp::launch_matvec(P.n, f->plan->dRowptr, f->plan->dColidx, f->dValues, f->dB, f->dX, nrhs, f->stream);
    ck(cudaMemcpyAsync(y, f->dX, bytes, cudaMemcpyDeviceToHost, f->stream), "copy y");
    ck(cudaStreamSynchronize(f->stream), "matvec");
    return (int)AMP_OK;
  });
}

}  // extern "C"
