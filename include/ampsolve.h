/*
 * ampsolve.h -- C ABI of the B200-native supernodal sparse direct solver (libampsolve.so).
 *
 * Drop-in boundary for the analyze / factor / solve path of jwt625/applied-multiphysics packages/core
 * (src/la/sparse.mjs, src/la/ldlt.mjs, src/la/order3d.mjs; typed surface src/la/sparse.d.mts and src/la/types.d.mts).
 * Plain pointers and sizes only. All host pointers are borrowed for the duration of the call.
 *
 * Patterns are CSR in full symmetric storage (both triangles, diagonal present, rows sorted ascending), as the
 * reference's CsrPattern (types.d.mts:6). Values are FP64 aligned with the CSR slots. Permutations are new -> old.
 * Right-hand sides and solutions: q vectors stored one after another (b[k * n + i]), original ordering.
 *
 * Errors: every function returns an amp_status. Misuse that the reference throws on returns a nonzero status whose
 * amp_last_error() message is the reference's message; numerical failure of a factorization is not an error: it
 * returns AMP_OK with result.ok = 0 (the reference's ok = false).
 */
#ifndef AMPSOLVE_H
#define AMPSOLVE_H

#include <stdint.h>

#if defined(__GNUC__)
#define AMP_API __attribute__((visibility("default")))
#else
#define AMP_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  AMP_OK = 0,
  AMP_NOT_SPD = 1,          /* Cholesky pivot not > 0 (reported through result.ok = 0 by amp_factor_numeric) */
  AMP_NONFINITE_PIVOT = 2,  /* LDL^T pivot not finite (reported through result.ok = 0) */
  AMP_PATTERN_MISMATCH = 3, /* 'symbolic analysis is for a different sparsity pattern' (sparse.mjs:929) */
  AMP_BAD_LENGTH = 4,       /* 'factorNumeric: N values for a pattern with M entries' (sparse.mjs:945), perm length */
  AMP_NO_FACTOR = 5,        /* 'solveNumeric: no successful numeric factorization' (sparse.mjs:1262) */
  AMP_NEED_COORDS = 6,      /* 'analyze: ordering nd needs node coordinates x and y of length n' (sparse.mjs:678) */
  AMP_DEVICE_TIMEOUT = 7,   /* a bounded device wait gave up */
  AMP_CUDA_ERROR = 8,
  AMP_OOM = 9,
  AMP_INVALID = 10          /* invalid argument (null handle, bad option) */
} amp_status;

typedef enum { AMP_ORDER_AMD = 0, AMP_ORDER_ND = 1, AMP_ORDER_ND3 = 2, AMP_ORDER_GIVEN = 3 } amp_ordering;
/* AMP_LDLT_BK: the real LDL^T with Bunch-Kaufman 1 x 1 / 2 x 2 pivots inside each 64-column pivot block (FP64); the
   reference has static perturbation only (ldlt.mjs:513-522), which AMP_LDLT reproduces. */
typedef enum { AMP_CHOLESKY = 0, AMP_LDLT = 1, AMP_LDLT_COMPLEX = 2, AMP_LDLT_BK = 3 } amp_factor_kind;
typedef enum { AMP_FP64 = 0, AMP_MIXED = 1 } amp_precision;

typedef struct amp_plan_s amp_plan;     /* symbolic analysis + device schedule of one pattern (reference: sym) */
typedef struct amp_factor_s amp_factor; /* numeric factor on the device (reference: NumericFactor / SupernodalLDLT) */

/* Options of amp_analyze; replaces analyze(pat, {perm, ordering, x, y, relax}) (sparse.mjs:666, sparse.d.mts:28) and
 * nd3Order(pat, x, y, z, {leaf}) followed by analyze(pat, {perm}) (order3d.mjs:27). Zero-initialise, then set. */
typedef struct {
  int ordering;          /* amp_ordering; AMP_ORDER_AMD by default */
  int relax;             /* relaxed supernode amalgamation; set 1 for the reference default (relax ?? true) */
  const int32_t *perm;   /* new -> old, length n, for AMP_ORDER_GIVEN */
  const double *x, *y, *z;
  int leaf;              /* ND leaf size; 0 = the reference default (48 for 2D, 2000 for 3D) */
  int device;            /* CUDA device ordinal */
  int group_blocks;      /* schedule: 64-column pivot blocks per group panel (1..16; 0 = the default, 4) */
  int small_front;       /* schedule: largest front factored whole by one CTA (32..128; 0 = the default, 128) */
  int defer_updates;     /* schedule: the update beyond the next group every this many group steps (K = the groups
                            since the last; 1..8, 0 = the default, 1) */
} amp_analyze_opts;

/* Scalars of a symbolic analysis (SymbolicAnalysis fields, types.d.mts:13-20). */
typedef struct {
  int32_t n, nsuper, max_front, nlevels;
  int64_t nnz_l, nnz_a, nnz_l_stored, pattern_nnz;
  double fill, flops, ordering_ms, symbolic_ms;
  int64_t device_bytes; /* device memory of one factor of this plan (L, update arena, schedule) */
} amp_plan_info;

/* Array fields of a symbolic analysis for amp_plan_array (int32 unless noted). The fields after AMP_F_LXP expose
   the device schedule built with the analysis (read-only introspection; no reference counterpart):
   - AMP_F_LEVEL_PTR / AMP_F_LEVEL_SUPERNODES: the supernodes of etree level L (leaves first) are
     LEVEL_SUPERNODES[LEVEL_PTR[L] .. LEVEL_PTR[L + 1]);
   - AMP_F_FWD_TASKS: the one-vector forward sweep's tasks, records {x, y, kind, 0} in launch order: kind 0 diagonal
     block y of supernode x, kind 1 the 64-row chunk y of supernode x's rows below, kind 2 the supernodes
     SOLVE_SMALL[x .. x + y) (one warp each), kind 3 the whole supernode x;
   - AMP_F_FWD_TASKS_MULTI: the multi-vector forward sweep's tasks (kinds 0-2);
   - AMP_F_BWD_TASKS: the backward sweep's tasks in launch order (kinds 0 and 2), a supernode's after its parent's;
   - AMP_F_SOLVE_SMALL: supernodes solved whole by one warp (m <= 32), grouped by level;
   - AMP_F_TINY_FRONTS, AMP_F_TINY_PTR (int64), AMP_F_TINY_MID (int64): fronts factored whole by one warp (m <= 32):
     level L's are TINY_FRONTS[TINY_PTR[L] .. TINY_PTR[L + 1]), sorted by m, those from TINY_MID[L] on with m > 16. */
typedef enum {
  AMP_F_PERM = 0, AMP_F_PINV, AMP_F_PARENT, AMP_F_COLCOUNT, AMP_F_LOWERP, AMP_F_LOWERI, AMP_F_LOWERSRC,
  AMP_F_SUPERSTART, AMP_F_COLSUPER, AMP_F_SUPERPARENT, AMP_F_CHILDHEAD, AMP_F_CHILDNEXT, AMP_F_SP, AMP_F_SI,
  AMP_F_LXP /* int64 */,
  AMP_F_LEVEL_PTR, AMP_F_LEVEL_SUPERNODES, AMP_F_FWD_TASKS, AMP_F_FWD_TASKS_MULTI, AMP_F_BWD_TASKS,
  AMP_F_SOLVE_SMALL, AMP_F_TINY_FRONTS, AMP_F_TINY_PTR /* int64 */, AMP_F_TINY_MID /* int64 */
} amp_field;

typedef struct {
  int kind;         /* amp_factor_kind; either kind in either precision (mixed LDL^T: FP32 fronts, BF16x3 updates) */
  int precision;    /* amp_precision */
} amp_factor_opts;

/* Result of a numeric factorization (sparse.mjs factorNumeric ok; ldlt.mjs LdltFactorResult, types.d.mts:26). */
typedef struct {
  int32_t ok;
  int32_t n_neg, n_perturbed;
  int32_t fail_column;  /* first failing column (permuted order) or -1 */
  double ms;            /* device time of the factorization */
} amp_factor_result;

typedef struct {
  int max_steps;        /* refinement steps (reference default 3) */
  double tol;           /* stop when ||b - A x|| / ||b|| < tol (reference default 1e-14) */
} amp_refine_opts;

typedef struct {
  double rel_residual;  /* max over the right-hand sides */
  int32_t steps;        /* max over the right-hand sides */
} amp_refine_stats;

typedef struct {
  double tol;           /* stop when the residual estimate / ||b|| <= tol (reference default 1e-10) */
  int32_t restart;      /* Krylov vectors per cycle (reference default 40) */
  int32_t max_iter;     /* total iterations (reference default 400) */
} amp_gmres_opts;

typedef struct {
  double rel_residual;  /* true ||b - A x|| / ||b|| of the returned x */
  int32_t iterations;
  int32_t converged;    /* rel_residual <= max(10 tol, 1e-14), as the reference reports */
} amp_gmres_stats;

/* ---- orderings (host) ---- */
/* amdOrder(pat, {denseFactor}) (sparse.mjs:297-592). perm: n entries, new -> old. */
AMP_API int amp_amd_order(int32_t n, const int32_t *rowptr, const int32_t *colidx, double dense_factor, int32_t *perm);
/* ndOrder(pat, x, y, leaf) (sparse.mjs:231-283). */
AMP_API int amp_nd_order(int32_t n, const int32_t *rowptr, const int32_t *colidx, const double *x, const double *y,
                 int32_t leaf, int32_t *perm);
/* nd3Order(pat, x, y, z, {leaf}) (order3d.mjs:27-77). */
AMP_API int amp_nd3_order(int32_t n, const int32_t *rowptr, const int32_t *colidx, const double *x, const double *y,
                  const double *z, int32_t leaf, int32_t *perm);
/* patternFingerprint(pat) (sparse.mjs:908-925): writes "n:nnz:hash" (NUL-terminated) into buf. */
AMP_API int amp_pattern_fingerprint(int32_t n, const int32_t *rowptr, const int32_t *colidx, char *buf, int32_t buflen);

/* ---- symbolic analysis ---- */
/* analyze(pat, opts) (sparse.mjs:666-902): host symbolic phase, then the device schedule is uploaded. */
AMP_API int amp_analyze(int32_t n, const int32_t *rowptr, const int32_t *colidx, const amp_analyze_opts *opts,
                amp_plan **out);
AMP_API int amp_plan_get_info(const amp_plan *plan, amp_plan_info *info);
/* Copies one SymbolicAnalysis array (amp_field) into dst (capacity len elements); *out_len = its length. */
AMP_API int amp_plan_array(const amp_plan *plan, int field, void *dst, int64_t len, int64_t *out_len);
/* Autotuner of the device schedule (no reference counterpart: the reference's fixed crossovers, e.g. WASM_MIN_FRONT
 * and QCAP in la/wasm/*.mjs, are constants). Times the numeric factorization of `values` (kind, precision as in
 * amp_factor_opts) on this plan's device for each candidate schedule -- pivot blocks per group panel {1, 2, 4, 8} x
 * largest whole-front CTA front {64, 128}, then with the fastest of those the update beyond the next group deferred
 * over {2, 4, 8} group steps -- and keeps the fastest; ties go to the earlier candidate. The choice is
 * cached per (pattern fingerprint, kind, precision) for the process, so another plan of the same pattern takes it
 * without timing (cached = 1). Call before the plan's first amp_factor_create (AMP_INVALID otherwise). */
typedef struct {
  int32_t group_blocks, small_front;  /* the chosen schedule */
  int32_t cached;                     /* 1 when taken from the cache, without timing */
  int32_t candidates;                 /* schedules timed */
  double ms_best, ms_default;         /* factorization time of the choice and of the default schedule */
  int32_t defer_updates;              /* the chosen schedule's deferral of the update beyond the next group */
} amp_tune_result;
AMP_API int amp_plan_autotune(amp_plan *plan, const double *values, int64_t nvalues, int values_on_device, int kind,
                              int precision, amp_tune_result *result);
/* sym.patternKey */
AMP_API int amp_plan_fingerprint(const amp_plan *plan, char *buf, int32_t buflen);
/* checkSymbolic(sym, pat) (sparse.mjs:928-930): AMP_PATTERN_MISMATCH when pat is not the analysed pattern. */
AMP_API int amp_plan_check_pattern(const amp_plan *plan, int32_t n, const int32_t *rowptr, const int32_t *colidx);
AMP_API void amp_plan_destroy(amp_plan *plan);

/* ---- numeric factorization ---- */
/* Allocates the device factor of a plan: new SparseCholesky(pat, null, {sym}) storage (sparse.mjs:1318) or
 * new SupernodalLDLT(sym) (ldlt.mjs:432-448). */
AMP_API int amp_factor_create(amp_plan *plan, const amp_factor_opts *opts, amp_factor **out);
/* factorNumeric(sym, values) (sparse.mjs:941) / SupernodalLDLT.factor(values, {pivotTol}) (ldlt.mjs:450).
 * values: nvalues FP64 in CSR slot order, host memory (values_on_device = 0) or device memory (1).
 * LDL^T: pivots with |d| < pivot_tol * max |A(i, i)| become +-that bound (counted in n_perturbed); n_neg counts the
 * negative pivots (the inertia); a non-finite small pivot gives ok = 0. pivot_tol is ignored for Cholesky. */
AMP_API int amp_factor_numeric(amp_factor *f, const double *values, int64_t nvalues, int values_on_device, double pivot_tol,
                       amp_factor_result *result);
/* solveNumeric / solveNumericMulti (sparse.mjs:1261-1310), SupernodalLDLT.solve / solveMany (ldlt.mjs:565-643).
 * b, x: nrhs vectors of length n one after another; host (on_device = 0) or device (1) memory. */
AMP_API int amp_solve(amp_factor *f, const double *b, int32_t nrhs, double *x, int on_device);
/* solveRefined(pat, values, b, {maxSteps, tol}) (ldlt.mjs:253-275): FP64 iterative refinement against the values
 * of the last amp_factor_numeric call (the unperturbed matrix). */
AMP_API int amp_solve_refined(amp_factor *f, const double *b, int32_t nrhs, double *x, int on_device,
                      const amp_refine_opts *opts, amp_refine_stats *stats);
/* Row groups for amp_solve_refined: the factored matrix is block diagonal with ngroups independent systems, rows
 * [offsets[g], offsets[g + 1]) (offsets[0] = 0, offsets[ngroups] = n, non-decreasing). Refinement then measures
 * ||b - A x|| / ||b|| per system and right-hand side, as a separate solveRefined call per system would
 * (ldlt.mjs:257-269), and stops when every one is below tol; stats report the largest. ngroups = 0 clears. */
AMP_API int amp_factor_set_row_groups(amp_factor *f, int32_t ngroups, const int64_t *offsets);
/* gmres(matvec, precond, b, {tol, restart, maxIter}) (gmres-real.mjs:31-105) with matvec = the factored matrix (FP64
 * CSR on the device) and precond = this factor's solve: restarted, right-preconditioned GMRES from x0 = 0, so with a
 * mixed-precision factor it is GMRES-based iterative refinement. One right-hand side; b, x host or device memory. */
AMP_API int amp_solve_gmres(amp_factor *f, const double *b, double *x, int on_device, const amp_gmres_opts *opts,
                    amp_gmres_stats *stats);
/* num.Lx (the m x nc column-major blocks at Lxp) and D (LDL^T) copied to host; either pointer may be null. */
AMP_API int amp_factor_download(const amp_factor *f, double *Lx, double *D);
/* The pivots of an AMP_LDLT_BK factor (n entries each, permuted order; either pointer may be null): Doff[j] = D(j+1, j)
 * when (j, j + 1) is a 2 x 2 pivot, else 0 (amp_factor_download's D holds every pivot's diagonal); piv[f + c0 + i] =
 * the column of the 64-column pivot block at c0 of the supernode starting at f that became its i-th pivot. The block's
 * L columns are in that order and its rows in earlier columns of the supernode stay in the original order, so
 * P_b (A's Schur complement block) P_b^T = L_bb D_b L_bb^T block by block. No counterpart in the reference (its LDL^T
 * has static perturbation only, ldlt.mjs:513-522). */
AMP_API int amp_factor_download_pivots(const amp_factor *f, double *Doff, int32_t *piv);
AMP_API void amp_factor_destroy(amp_factor *f);
/* Bound of this factor's device waits, in polls (0 = the defaults: about a second for the solve sweeps' inter-CTA
 * waits, half a second for the tensor-core update's pipeline waits). A wait that runs out ends its kernel early and
 * the call returns AMP_DEVICE_TIMEOUT; the device stays usable. No counterpart in the reference (its solver runs on
 * one CPU thread and never waits); for callers that want a stuck device reported sooner, and for tests of that path.
 * Changing the bound discards the factor's captured factorization graph (it is captured again on the next call). */
AMP_API int amp_factor_set_wait_limit(amp_factor *f, int64_t polls);

/* Per-kernel-class device time of the calls made while profiling is on (CUDA events around every launch on the
 * factor's stream; graphs are not used meanwhile). Algorithmic flops / bytes are the counts the work requires.
 * Replaces the reference's opt-in timing records (sparse.mjs:20-29 timingSink, SparseCholesky.timing). */
typedef struct {
  char name[24];
  int32_t launches; /* kernel launches */
  double ms, flops, bytes;
} amp_kernel_stat;
AMP_API int amp_profile_enable(amp_factor *f, int enable);
AMP_API int amp_profile_read(amp_factor *f, amp_kernel_stat *stats, int32_t cap, int32_t *count);
/* The individual timed regions behind amp_profile_read (call before it; it clears the records; a region is one
 * kernel, or the few of one class launched together: a level's small-front classes, a dot product's two passes):
 * kernel class index (order of amp_profile_read's names: assemble, group_panel, update_syrk, solve_forward,
 * solve_backward, permute, residual_spmv, potrf (unused: POTRF runs inside group_panel), diag_inverse, krylov,
 * small_fronts, chain_mats), device ms, flops. */
AMP_API int amp_profile_launches(amp_factor *f, int32_t *kinds, double *ms, double *flops, int32_t cap,
                                 int32_t *count);

/* matVec(pat, val, x) (sparse.mjs:219-228) on the device: y = A x for nrhs vectors (host pointers). */
AMP_API int amp_matvec(amp_factor *f, const double *x, int32_t nrhs, double *y);
/* matVec(pat, val, x) (sparse.mjs:219-228) without a factor: y = A x for nrhs vectors on device `device` (host
 * pointers; the call allocates its device buffers and waits for the result). */
AMP_API int amp_matvec_csr(int32_t n, const int32_t *rowptr, const int32_t *colidx, const double *values,
                           const double *x, int32_t nrhs, double *y, int device);

/* ---- complex-symmetric LDL^T (ldlt.mjs:648-900 ComplexSupernodalLDLT, complexSolveRefined) ----
 * A = A^T complex (no conjugation) on the plan's pattern, values as two FP64 arrays (re, im) aligned with the CSR
 * slots, as the reference takes them. FP64 complex factor on the device: every front through the group-panel
 * kernels (1 x 1 pivots with the reference's static perturbation: a pivot of magnitude below tau = pivotTol *
 * max_i |A(i, i)| is scaled to magnitude tau; a non-finite one fails), complex update tiles on the CUDA cores and
 * level-scheduled complex solves. The factor is destroyed with amp_factor_destroy; the real-valued entry points
 * reject it, and these reject real factors. */
/* new ComplexSupernodalLDLT(sym) (ldlt.mjs:649-666) */
AMP_API int amp_cfactor_create(amp_plan *plan, amp_factor **out);
/* factor(re, im, {pivotTol}) (ldlt.mjs:667-800): result.ok, n_perturbed, fail_column (n_neg is 0: no inertia). */
AMP_API int amp_cfactor_numeric(amp_factor *f, const double *re, const double *im, int64_t nvalues,
                                int values_on_device, double pivot_tol, amp_factor_result *result);
/* solve(br, bi) (ldlt.mjs:802-862) for nrhs right-hand sides one after another; host (0) or device (1) pointers. */
AMP_API int amp_csolve(amp_factor *f, const double *br, const double *bi, int32_t nrhs, double *xr, double *xi,
                       int on_device);
/* solveRefined(pat, re, im, br, bi, {maxSteps, tol}) (complexSolveRefined, ldlt.mjs:870-900) against the values of
 * the last amp_cfactor_numeric (unperturbed): stats report the worst relative residual and the most steps. */
AMP_API int amp_csolve_refined(amp_factor *f, const double *br, const double *bi, int32_t nrhs, double *xr,
                               double *xi, int on_device, const amp_refine_opts *opts, amp_refine_stats *stats);
/* Lr, Li (the m x nc column-major blocks at Lxp) and Dr, Di copied to host; any pointer may be null. */
AMP_API int amp_cfactor_download(const amp_factor *f, double *Lr, double *Li, double *Dr, double *Di);

/* ---- on-device assembly of the values (physics/src/common/scalar.ts:96-146 assembleCells; la/sparse.mjs:113-185
 * elementSlots / blockElementSlots; fem/tri.mjs:192-225 restrictMatrix) ---- */
typedef struct amp_assembly_s amp_assembly;
typedef enum {
  AMP_ELEM_P1_TRI_SCALAR = 0,  /* P1 triangles, 2D, one coefficient per element (conductivity), fem/tri.mjs:45-80 */
  AMP_ELEM_P1_TET_ELASTIC = 1  /* P1 tets, 3D, 3 DOFs per node, (E, nu) per element, physics/src/elastic/index.ts */
} amp_element_kind;
/* The element slots of a mesh in the system's CSR pattern (n rows, full symmetric storage), computed on the host and
 * kept on the device with the mesh: coords (dim per node: 2 for triangles, 3 for tets), conn (nelem x nodes per
 * element), dofs (nnodes x DOFs per node: the system row of node v's component c at dofs[v bs + c], or -1 for a DOF
 * removed by the Dirichlet restriction, whose element rows and columns are dropped). AMP_PATTERN_MISMATCH when an
 * element couples two rows the pattern does not connect. */
AMP_API int amp_assembly_create(int kind, int32_t n, const int32_t *rowptr, const int32_t *colidx, int32_t nnodes,
                                const double *coords, int64_t nelem, const int32_t *conn, const int32_t *dofs,
                                int device, amp_assembly **out);
/* values = the assembled system (the pattern's nnz CSR values) for per-element coefficients coef (kind 0: one per
 * element; kind 1: E and nu per element), summed per CSR slot in element order as the reference's element loop adds
 * them. coef host (coef_on_device 0) or device (1); values host (0) or device (1); stream: a cudaStream_t (null =
 * default); the call waits for its work. */
AMP_API int amp_assemble(amp_assembly *a, const double *coef, int coef_on_device, double *values,
                         int values_on_device, void *stream);
AMP_API void amp_assembly_destroy(amp_assembly *a);

/* ---- shift-invert eigen operator (physics/src/common/eigen.ts:116-175 shiftInvertEigen; la/arnoldi.mjs) ---- */
/* The factor holds A = K - sigma M (Cholesky or LDL^T). amp_factor_set_mass gives M's values on the same pattern
 * (nvalues CSR slots, host or device memory; copied to the device once). */
AMP_API int amp_factor_set_mass(amp_factor *f, const double *mvalues, int64_t nvalues, int on_device);
/* op(X) = A^-1 (M X) for m vectors of length n one after another (eigen.ts:150-160): M X by the device SpMV, then one
 * multi-vector solve; host (on_device 0) or device (1) pointers. */
AMP_API int amp_shift_invert_apply(amp_factor *f, const double *X, int32_t m, double *Y, int on_device);

typedef struct {
  int32_t n_want;       /* Ritz values wanted: those of largest modulus (eigenvalues nearest the shift) */
  int32_t block_size;   /* vectors per block (reference default 1) */
  int32_t max_basis;    /* basis size per cycle (reference default max(30, 2 nWant + 12)) */
  int32_t max_restarts; /* thick restarts (reference default 60) */
  double tol;           /* converged when the Ritz residual <= tol |mu| (reference default 1e-10) */
  uint32_t seed;        /* start block: the reference's LCG (arnoldi.mjs seededRandom) */
} amp_eigen_opts;

typedef struct {
  int32_t converged;    /* all n_want Ritz pairs below the tolerance */
  int32_t restarts;
  int32_t op_vectors;   /* operator applications (vectors) */
  int32_t basis;        /* basis size used per cycle */
  double max_residual;  /* largest Ritz residual / |mu| of the returned pairs */
  double ms;            /* wall time of the Krylov iteration */
} amp_eigen_stats;

/* blockArnoldi(n, op, {nWant, blockSize, maxBasis, tol, maxRestarts, seed}) (la/arnoldi.mjs:36-200) with op =
 * amp_shift_invert_apply, run on the device: the Krylov basis, its M-products and the orthogonalisation live in device
 * memory and only the small projected matrix is on the host (one round trip per block, none per vector). The basis
 * is M-orthonormal (op is self-adjoint in the M inner product for symmetric K and M, M positive definite), so the
 * projected matrix is symmetric; block Lanczos with full reorthogonalisation and thick restart. mu: the n_want Ritz
 * values of largest modulus, by decreasing |mu| (eigenvalue lambda = sigma + 1 / mu); vecs: the matching M-orthonormal
 * Ritz vectors, n each one after another, host (on_device 0) or device (1). */
AMP_API int amp_eigen_block_arnoldi(amp_factor *f, const amp_eigen_opts *opts, double *mu, double *vecs, int on_device,
                                    amp_eigen_stats *stats);

/* Partial Cholesky of ONE dense front in place, allocating nothing. No counterpart in the reference's API.
 * For callers that cannot call cudaMalloc: applications that give all device memory to their own pool at start-up,
 * or that must not let an allocation stall their other streams. F: device pointer to an m x m column-major front
 * (ld = m, lower part read and written); nc pivot columns are factored (L11, L21 in place) and the trailing
 * (m - nc) block receives the Schur update. Limit: m <= 16384; larger fronts are rejected with AMP_INVALID.
 * Scratch: a static device array of 2 KB per GPU that loads the library, kept until exit and shared by every call
 * (each call resets it); calls that overlap on the GPU race on it. The first call on a device looks up the array's
 * address with that device current (devices 0..63); the look-up is serialised across host threads. stream: a
 * cudaStream_t (null = default stream); the call waits for its work.
 * *fail_column: -1, or the first pivot column that was not positive. After a failure F holds a partial result: the
 * pivot blocks before the failing one are factored and their updates applied; the rest is as those updates left it. */
AMP_API int amp_front_factor_noalloc(double *F, int32_t m, int32_t nc, void *stream, int32_t *fail_column);

/* Message of the last failing call on this thread ("" when none). */
AMP_API const char *amp_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* AMPSOLVE_H */
