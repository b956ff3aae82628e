// Host-callable launchers of the device kernels.
#pragma once
#include <cuda_bf16.h>
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "../host/plan.hpp"
#include "devplan.cuh"

namespace amp {

cudaError_t init_kernel_attributes();  // once per device (with that device current), before its first launch

// ranges: the schedule's per-task child column ranges (AsmTask::ch0 indexes them)
template <class T>
void launch_assemble(const AsmTask *tasks, const ChildRange *ranges, int64_t ntasks, const DevPlan &P,
                     const value_of<T> *values, T *Lx, T *U, const unsigned long long *status, cudaStream_t st);
// one group of pivot blocks per item: nstrips strip tasks, ticket and flags zeroed before the factorization
template <class T>
void launch_group_panel(const GroupItem *items, const StripTask *strips, int nstrips, int *ticket, int *flags,
                        const DevPlan &P, T *Lx, unsigned long long *status, __nv_bfloat16 *Shi, __nv_bfloat16 *Slo,
                        const LdltArgs<T> &ld, cudaStream_t st);
void launch_ldlt_tau(const double *values, const DevPlan &P, double *scal, cudaStream_t st);
// complex-symmetric update tiles (FP64 complex, CUDA cores), one CTA per tile
void launch_update_c(const TileTask *tasks, int64_t ntasks, cplx *Lx, cplx *U, const cplx *W,
                     const unsigned long long *status, cudaStream_t st);
// whole small fronts of one level: tiny (m <= 32, warp per front; sorted by m, the first ntinyMid with m <= 16) and
// small (m <= 128, CTA per front; maxM = their largest m); returns the kernels launched
template <class T>
int launch_fronts_small(const int *tiny, int ntiny, int ntinyMid, const int *small, int nsmall, int maxM,
                        const DevPlan &P, const double *values, T *Lx, T *U, unsigned long long *status,
                        const LdltArgs<T> &la, cudaStream_t st);
// width: the tiles' columns, 256, or 128 / 64 (tasks whose columns are one 128- / 64-column group)
// spin: bound of each role's wait in polls (0 = the default, about 0.5 s)
void launch_update_mx(const MixTask *tasks, int64_t ntasks, const CUtensorMap *maps, float *L32, float *U32,
                      unsigned long long *status, int num_sms, cudaStream_t st, int width = 256, long long spin = 0);
int num_sms();
void launch_update(const TileTask *tasks, int64_t ntasks, const DevPlan &P, double *Lx, double *U, const double *W,
                   const unsigned long long *status, cudaStream_t st);
void launch_permute_in(const double *b, double *y, const int *perm, int n, int q, cudaStream_t st);
void launch_permute_out(const double *y, double *x, const int *perm, int n, int q, cudaStream_t st);
// inverses of the diagonal blocks (with each block's pivot order folded in when P.lpiv is set)
template <class TL>
void launch_diag_inv(const int *blocks, int nblocks, const DevPlan &P, const TL *Lx, TL *Inv, cudaStream_t st);
// D solve of a Bunch-Kaufman factor (1 x 1 and 2 x 2 pivots), q interleaved vectors, between the sweeps
void launch_dsolve_bk(int n, int q, const double *D, const double *Doff, double *y, cudaStream_t st);
template <class TL>
void launch_fwd_blocks(const int4 *tasks, int ntasks, int *ticket, const DevPlan &P, const TL *Lx, const TL *Inv,
                       const TL *Mch, double *y, double *T, int *flags, unsigned long long *hand, int epoch, int *done,
                       unsigned long long *status, cudaStream_t st);
template <class TL>
void launch_bwd_blocks(const int4 *tasks, int ntasks, int *ticket, const DevPlan &P, const TL *Lx, const TL *Inv,
                       const TL *Gch, const double *Dpiv, double *y, int *flags, unsigned long long *hand, int epoch,
                       unsigned long long *status, cudaStream_t st);
// M_b = X_b L[b, b-1] and G_b = L[b+1, b] X_b of consecutive diagonal blocks (tasks {s, b}), after launch_diag_inv
template <class TL>
void launch_chain_mats(const int2 *tasks, int ntasks, const DevPlan &P, const TL *Lx, const TL *Inv, TL *Mch, TL *Gch,
                       cudaStream_t st);

// several right-hand sides (q <= multi_max_vectors(), interleaved: entry i of vector k at [i q + k])
// Vectors move in slices of 16, each with its own ready flags (flags[slice * nflags + block], nflags >= the plan's
// flag count) and done counters (done[slice * nsuper + s]): the flag and done arrays hold multi_max_vectors() / 16
// sets. tasks: the plan's list with block tasks expanded into multi_slices(q) consecutive entries (.w = the slice), or
// left single with .w = -1 (the task moves every vector at once).
int multi_max_vectors();
int multi_slices(int q);
// wide: the list holds .w = -1 tasks (the kernels with the all-vector path)
// Mch / Gch: the chain matrices of a Cholesky factor (launch_chain_mats), or null (LDL^T: substitution order)
template <class TL>
void launch_fwd_multi(const int4 *tasks, int ntasks, bool wide, int *ticket, const DevPlan &P, const TL *Lx,
                      const TL *Inv, const TL *Mch, double *y, double *T, int *flags, int nflags, int epoch, int *done,
                      int q, unsigned long long *status, cudaStream_t st);
template <class TL>
void launch_bwd_multi(const int4 *tasks, int ntasks, bool wide, int *ticket, const DevPlan &P, const TL *Lx,
                      const TL *Inv, const TL *Gch, const double *Dpiv, double *y, int *flags, int nflags, int epoch,
                      int q, unsigned long long *status, cudaStream_t st);
void launch_to_interleaved(const double *B, double *Yil, int n, int q, cudaStream_t st);
void launch_from_interleaved(const double *Xil, double *X, int n, int q, cudaStream_t st);
void launch_rows_permute(const double *src, double *dst, const int *perm, int n, int q, bool scatter, cudaStream_t st);
void launch_residual_multi(int n, const int *rowptr, const int *colidx, const double *val, const double *x,
                           const double *b, double *r, double *norms, int q, const int *rowGroup, cudaStream_t st);

// complex-symmetric LDL^T: packing, permutation, the level sweeps, the residual (csolve.cu)
void launch_cpack(int64_t nnz, const double *re, const double *im, cplx *out, cudaStream_t st);
void launch_cunpack(int n, const cplx *x, double *xr, double *xi, cudaStream_t st);
void launch_ctau(const cplx *values, const DevPlan &P, double *scal, cudaStream_t st);
void launch_cpermute_in(int n, const double *br, const double *bi, const int *perm, cplx *y, cudaStream_t st);
void launch_cpermute_out(int n, const cplx *y, const int *perm, double *xr, double *xi, cudaStream_t st);
void launch_cpermute_vec(int n, const cplx *src, const int *perm, cplx *dst, bool gather, cudaStream_t st);
void launch_caxpy(int n, cplx *x, const cplx *dx, cudaStream_t st);
int launch_csolve_permuted(const DevPlan &P, const int *lvlPtr, int nlevels, const cplx *L, const cplx *D, cplx *y,
                           cudaStream_t st);
void launch_cresidual(int n, const int *rowptr, const int *colidx, const cplx *val, const cplx *x, const cplx *b,
                      cplx *r, double *norms, cudaStream_t st);

}  // namespace amp
