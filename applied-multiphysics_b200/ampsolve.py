"""Python host mirror of the reference's sparse direct solver API over the C ABI of libampsolve.so.

Names, argument meaning and error behaviour follow jwt625/applied-multiphysics packages/core/src/la/sparse.mjs
(analyze, factorNumeric, solveNumeric, solveNumericMulti, SparseCholesky, amdOrder, ndOrder, patternFingerprint,
checkSymbolic, matVec), ldlt.mjs (SupernodalLDLT) and order3d.mjs (nd3Order): misuse raises AmpError with the
reference's message, a numerical failure returns ok = False. The symbolic phase runs on the host inside the library;
the numeric factorization and the solves run on the GPU. There is no CPU fallback: without libampsolve.so (or without
a GPU for the numeric calls) every call raises.
"""
from __future__ import annotations

import ctypes as C
from decimal import ROUND_HALF_UP, Decimal
import os
import time
from typing import Sequence

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libampsolve.so")
_lib = None

AMP_OK, AMP_NOT_SPD, AMP_NONFINITE_PIVOT, AMP_PATTERN_MISMATCH, AMP_BAD_LENGTH, AMP_NO_FACTOR, AMP_NEED_COORDS, \
    AMP_DEVICE_TIMEOUT, AMP_CUDA_ERROR, AMP_OOM, AMP_INVALID = range(11)
ORDER_AMD, ORDER_ND, ORDER_ND3, ORDER_GIVEN = range(4)
CHOLESKY, LDLT, LDLT_COMPLEX, LDLT_BK = 0, 1, 2, 3  # LDLT_BK: Bunch-Kaufman pivots in each pivot block
AMP_ELEM_P1_TRI_SCALAR, AMP_ELEM_P1_TET_ELASTIC = 0, 1
FP64, MIXED = 0, 1

FIELDS = ["perm", "pinv", "parent", "colCount", "lowerP", "lowerI", "lowerSrc", "superStart", "colSuper",
          "superParent", "childHead", "childNext", "Sp", "Si", "Lxp",
          # the device schedule (amp_field after AMP_F_LXP): read-only introspection
          "levelPtr", "levelSupernodes", "fwdTasks", "fwdTasksMulti", "bwdTasks", "solveSmall", "tinyFronts",
          "tinyPtr", "tinyMid"]
_INT64_FIELDS = ("Lxp", "tinyPtr", "tinyMid")


class AmpError(Exception):
    """Raised where the reference throws an Error; ``code`` is the amp_status."""

    def __init__(self, code: int, msg: str):
        super().__init__(msg)
        self.code = code


class _AnalyzeOpts(C.Structure):
    _fields_ = [("ordering", C.c_int), ("relax", C.c_int), ("perm", C.c_void_p), ("x", C.c_void_p),
                ("y", C.c_void_p), ("z", C.c_void_p), ("leaf", C.c_int), ("device", C.c_int),
                ("group_blocks", C.c_int), ("small_front", C.c_int), ("defer_updates", C.c_int)]


class _PlanInfo(C.Structure):
    _fields_ = [("n", C.c_int32), ("nsuper", C.c_int32), ("max_front", C.c_int32), ("nlevels", C.c_int32),
                ("nnz_l", C.c_int64), ("nnz_a", C.c_int64), ("nnz_l_stored", C.c_int64), ("pattern_nnz", C.c_int64),
                ("fill", C.c_double), ("flops", C.c_double), ("ordering_ms", C.c_double),
                ("symbolic_ms", C.c_double), ("device_bytes", C.c_int64)]


class _FactorOpts(C.Structure):
    _fields_ = [("kind", C.c_int), ("precision", C.c_int)]


class _FactorResult(C.Structure):
    _fields_ = [("ok", C.c_int32), ("n_neg", C.c_int32), ("n_perturbed", C.c_int32), ("fail_column", C.c_int32),
                ("ms", C.c_double)]


class _GmresOpts(C.Structure):
    _fields_ = [("tol", C.c_double), ("restart", C.c_int32), ("max_iter", C.c_int32)]


class _GmresStats(C.Structure):
    _fields_ = [("rel_residual", C.c_double), ("iterations", C.c_int32), ("converged", C.c_int32)]


class _KernelStat(C.Structure):
    _fields_ = [("name", C.c_char * 24), ("launches", C.c_int32), ("ms", C.c_double), ("flops", C.c_double),
                ("bytes", C.c_double)]


class _RefineOpts(C.Structure):
    _fields_ = [("max_steps", C.c_int), ("tol", C.c_double)]


class _RefineStats(C.Structure):
    _fields_ = [("rel_residual", C.c_double), ("steps", C.c_int32)]


class _TuneResult(C.Structure):
    _fields_ = [("group_blocks", C.c_int32), ("small_front", C.c_int32), ("cached", C.c_int32),
                ("candidates", C.c_int32), ("ms_best", C.c_double), ("ms_default", C.c_double),
                ("defer_updates", C.c_int32)]


class _EigenOpts(C.Structure):
    _fields_ = [("n_want", C.c_int32), ("block_size", C.c_int32), ("max_basis", C.c_int32),
                ("max_restarts", C.c_int32), ("tol", C.c_double), ("seed", C.c_uint32)]


class _EigenStats(C.Structure):
    _fields_ = [("converged", C.c_int32), ("restarts", C.c_int32), ("op_vectors", C.c_int32), ("basis", C.c_int32),
                ("max_residual", C.c_double), ("ms", C.c_double)]


_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")

# every entry point of include/ampsolve.h with its argument types
SIGNATURES = {
    "amp_amd_order": (C.c_int, [C.c_int32, _i32p, _i32p, C.c_double, _i32p]),
    "amp_nd_order": (C.c_int, [C.c_int32, _i32p, _i32p, C.c_void_p, C.c_void_p, C.c_int32, _i32p]),
    "amp_nd3_order": (C.c_int, [C.c_int32, _i32p, _i32p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, _i32p]),
    "amp_pattern_fingerprint": (C.c_int, [C.c_int32, _i32p, _i32p, C.c_char_p, C.c_int32]),
    "amp_analyze": (C.c_int, [C.c_int32, _i32p, _i32p, C.POINTER(_AnalyzeOpts), C.POINTER(C.c_void_p)]),
    "amp_plan_get_info": (C.c_int, [C.c_void_p, C.POINTER(_PlanInfo)]),
    "amp_plan_array": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_int64, C.POINTER(C.c_int64)]),
    "amp_plan_fingerprint": (C.c_int, [C.c_void_p, C.c_char_p, C.c_int32]),
    "amp_plan_check_pattern": (C.c_int, [C.c_void_p, C.c_int32, _i32p, _i32p]),
    "amp_plan_destroy": (None, [C.c_void_p]),
    "amp_plan_autotune": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int64, C.c_int, C.c_int, C.c_int,
                                    C.POINTER(_TuneResult)]),
    "amp_factor_create": (C.c_int, [C.c_void_p, C.POINTER(_FactorOpts), C.POINTER(C.c_void_p)]),
    "amp_factor_numeric": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int64, C.c_int, C.c_double,
                                     C.POINTER(_FactorResult)]),
    "amp_solve": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_int]),
    "amp_solve_refined": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_int, C.POINTER(_RefineOpts),
                                    C.POINTER(_RefineStats)]),
    "amp_factor_set_row_groups": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p]),
    "amp_solve_gmres": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.POINTER(_GmresOpts),
                                  C.POINTER(_GmresStats)]),
    "amp_factor_download": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "amp_factor_download_pivots": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "amp_factor_destroy": (None, [C.c_void_p]),
    "amp_matvec": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p]),
    "amp_factor_set_wait_limit": (C.c_int, [C.c_void_p, C.c_int64]),
    "amp_matvec_csr": (C.c_int, [C.c_int32, _i32p, _i32p, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_int]),
    "amp_factor_set_mass": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int64, C.c_int]),
    "amp_cfactor_create": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    "amp_cfactor_numeric": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_int, C.c_double,
                                      C.POINTER(_FactorResult)]),
    "amp_csolve": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_int]),
    "amp_csolve_refined": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_int,
                                     C.POINTER(_RefineOpts), C.POINTER(_RefineStats)]),
    "amp_cfactor_download": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "amp_assembly_create": (C.c_int, [C.c_int, C.c_int32, _i32p, _i32p, C.c_int32, C.c_void_p, C.c_int64, C.c_void_p,
                                      C.c_void_p, C.c_int, C.POINTER(C.c_void_p)]),
    "amp_assemble": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p]),
    "amp_assembly_destroy": (None, [C.c_void_p]),
    "amp_shift_invert_apply": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_int]),
    "amp_eigen_block_arnoldi": (C.c_int, [C.c_void_p, C.POINTER(_EigenOpts), C.c_void_p, C.c_void_p, C.c_int,
                                          C.POINTER(_EigenStats)]),
    "amp_profile_enable": (C.c_int, [C.c_void_p, C.c_int]),
    "amp_profile_read": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32, C.POINTER(C.c_int32)]),
    "amp_profile_launches": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32,
                                       C.POINTER(C.c_int32)]),
    "amp_last_error": (C.c_char_p, []),
}


def lib():
    """The loaded libampsolve.so (raises when it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            raise RuntimeError(f"{_LIB_PATH} is missing: build it with __graft_entry__.build() (no CPU fallback)")
        L = C.CDLL(_LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _check(code: int):
    if code != AMP_OK:
        raise AmpError(code, lib().amp_last_error().decode())


def _pat(pat):
    n = int(pat.n)
    rp = np.ascontiguousarray(pat.rowptr, dtype=np.int32)
    ci = np.ascontiguousarray(pat.colidx, dtype=np.int32)
    if ci.size == 0:
        ci = np.zeros(1, np.int32)
    return n, rp, ci


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _ptr(a):
    return None if a is None else a.ctypes.data


# ---- orderings (sparse.mjs amdOrder / ndOrder, order3d.mjs nd3Order) ----------------------------------------------
def amdOrder(pat, denseFactor: float = 10.0) -> np.ndarray:
    n, rp, ci = _pat(pat)
    out = np.zeros(max(n, 1), np.int32)
    _check(lib().amp_amd_order(n, rp, ci, denseFactor, out))
    return out[:n]


def ndOrder(pat, x, y, leaf: int = 48) -> np.ndarray:
    n, rp, ci = _pat(pat)
    out = np.zeros(max(n, 1), np.int32)
    xa, ya = _f64(x), _f64(y)
    _check(lib().amp_nd_order(n, rp, ci, _ptr(xa), _ptr(ya), leaf, out))
    return out[:n]


def nd3Order(pat, x, y, z, leaf: int = 2000) -> np.ndarray:
    n, rp, ci = _pat(pat)
    out = np.zeros(max(n, 1), np.int32)
    xa, ya, za = _f64(x), _f64(y), _f64(z)
    _check(lib().amp_nd3_order(n, rp, ci, _ptr(xa), _ptr(ya), _ptr(za), leaf, out))
    return out[:n]


def patternFingerprint(pat) -> str:
    n, rp, ci = _pat(pat)
    buf = C.create_string_buffer(64)
    _check(lib().amp_pattern_fingerprint(n, rp, ci, buf, 64))
    return buf.value.decode()


# ---- symbolic analysis --------------------------------------------------------------------------------------------
class SymbolicAnalysis:
    """Result of analyze (SymbolicAnalysis, types.d.mts:13-20): scalars eagerly, arrays on first access."""

    def __init__(self, handle: int):
        self._h = handle
        info = _PlanInfo()
        _check(lib().amp_plan_get_info(handle, C.byref(info)))
        self.n = info.n
        self.nsuper = info.nsuper
        self.maxFront = info.max_front
        self.nlevels = info.nlevels
        self.nnzL = info.nnz_l
        self.nnzA = info.nnz_a
        self.nnzLStored = info.nnz_l_stored
        self.fill = info.fill
        self.flops = info.flops
        self.deviceBytes = info.device_bytes
        self.timing = {"ordering_ms": info.ordering_ms, "symbolic_ms": info.symbolic_ms}
        buf = C.create_string_buffer(64)
        _check(lib().amp_plan_fingerprint(handle, buf, 64))
        self.patternKey = buf.value.decode()
        self._arrays = {}

    def __getattr__(self, name):
        if name in FIELDS:
            if name not in self._arrays:
                k = FIELDS.index(name)
                ln = C.c_int64(0)
                _check(lib().amp_plan_array(self._h, k, None, 0, C.byref(ln)))
                arr = np.zeros(max(ln.value, 1), np.int64 if name in _INT64_FIELDS else np.int32)
                _check(lib().amp_plan_array(self._h, k, arr.ctypes.data, ln.value, C.byref(ln)))
                self._arrays[name] = arr[: ln.value]
            return self._arrays[name]
        raise AttributeError(name)

    @property
    def handle(self) -> int:
        return self._h

    def __del__(self):
        h = self.__dict__.get("_h")
        if h and _lib is not None:
            _lib.amp_plan_destroy(h)
            self._h = None


def analyze(pat, opts: dict | None = None, **kw) -> SymbolicAnalysis:
    """analyze(pat, {perm, ordering: 'amd' | 'nd' | 'nd3', x, y, z, relax, leaf}) (sparse.mjs:666)."""
    o = dict(opts or {})
    o.update(kw)
    n, rp, ci = _pat(pat)
    ao = _AnalyzeOpts()
    ao.relax = 1 if o.get("relax", True) else 0
    ao.leaf = int(o.get("leaf", 0) or 0)
    ao.device = int(o.get("device", 0))
    ao.group_blocks = int(o.get("groupBlocks", 0) or 0)
    ao.small_front = int(o.get("smallFront", 0) or 0)
    ao.defer_updates = int(o.get("deferUpdates", 0) or 0)
    keep = []
    perm = o.get("perm")
    if perm is not None:
        pa = np.ascontiguousarray(perm, dtype=np.int32)
        if pa.shape[0] != n:
            raise AmpError(AMP_BAD_LENGTH, f"analyze: perm has length {pa.shape[0]}, pattern has {n} rows")
        keep.append(pa)
        ao.ordering, ao.perm = ORDER_GIVEN, pa.ctypes.data
    else:
        ordering = o.get("ordering", "amd")
        if ordering == "nd":
            x, y = o.get("x"), o.get("y")
            if x is None or y is None or len(x) != n or len(y) != n:
                raise AmpError(AMP_NEED_COORDS, "analyze: ordering nd needs node coordinates x and y of length n")
            xa, ya = _f64(x), _f64(y)
            keep += [xa, ya]
            ao.ordering, ao.x, ao.y = ORDER_ND, xa.ctypes.data, ya.ctypes.data
        elif ordering == "nd3":
            x, y, z = o.get("x"), o.get("y"), o.get("z")
            if any(c is None or len(c) != n for c in (x, y, z)):
                raise AmpError(AMP_NEED_COORDS, "nd3Order: needs DOF coordinates x, y and z of length n")
            xa, ya, za = _f64(x), _f64(y), _f64(z)
            keep += [xa, ya, za]
            ao.ordering, ao.x, ao.y, ao.z = ORDER_ND3, xa.ctypes.data, ya.ctypes.data, za.ctypes.data
        elif ordering == "amd":
            ao.ordering = ORDER_AMD
        else:
            raise AmpError(AMP_INVALID, f"analyze: unknown ordering {ordering}")
    h = C.c_void_p()
    _check(lib().amp_analyze(n, rp, ci, C.byref(ao), C.byref(h)))
    return SymbolicAnalysis(h.value)


def autotune(sym: SymbolicAnalysis, values, kind: int = CHOLESKY, precision: int = FP64) -> dict:
    """Pick the device schedule (pivot blocks per group panel, whole-front cut-off) of `sym` by timing the
    factorization of `values` for each candidate (amp_plan_autotune); call before the first factor of `sym`."""
    v = _f64(values)
    r = _TuneResult()
    _check(lib().amp_plan_autotune(sym.handle, v.ctypes.data if v.size else None, v.size, 0, kind, precision,
                                   C.byref(r)))
    return {"groupBlocks": r.group_blocks, "smallFront": r.small_front, "deferUpdates": r.defer_updates,
            "cached": bool(r.cached),
            "candidates": r.candidates, "msBest": r.ms_best, "msDefault": r.ms_default}


def checkSymbolic(sym: SymbolicAnalysis, pat) -> None:
    """Throw unless `sym` was analysed from `pat` (sparse.mjs:928-930)."""
    n, rp, ci = _pat(pat)
    if sym is None:
        raise AmpError(AMP_PATTERN_MISMATCH, "symbolic analysis is for a different sparsity pattern")
    _check(lib().amp_plan_check_pattern(sym.handle, n, rp, ci))


# ---- numeric factor ------------------------------------------------------------------------------------------------
class NumericFactor:
    """Device factor of one symbolic analysis (NumericFactor, types.d.mts:23; SupernodalLDLT storage)."""

    def __init__(self, sym: SymbolicAnalysis, kind: int = CHOLESKY, precision: int = FP64):
        self.sym = sym
        self.kind = kind
        self.precision = precision
        self.kernel = "cuda-sm100a"
        self.ok = False
        self.nNeg = 0
        self.nPerturbed = 0
        self.ms = 0.0
        self.failColumn = -1
        fo = _FactorOpts(kind, precision)
        h = C.c_void_p()
        _check(lib().amp_factor_create(sym.handle, C.byref(fo), C.byref(h)))
        self._h = h.value

    @property
    def handle(self) -> int:
        return self._h

    def factor(self, values, pivotTol: float = 1e-13, on_device: bool = False) -> bool:
        res = _FactorResult()
        if on_device:  # values is a device pointer (int) with the pattern's nnz entries
            ptr, nv = values
            _check(lib().amp_factor_numeric(self._h, C.c_void_p(ptr), int(nv), 1, pivotTol, C.byref(res)))
        else:
            v = _f64(values)
            _check(lib().amp_factor_numeric(self._h, v.ctypes.data if v.size else None, v.size, 0, pivotTol,
                                            C.byref(res)))
        self.ok = bool(res.ok)
        self.nNeg, self.nPerturbed, self.ms, self.failColumn = res.n_neg, res.n_perturbed, res.ms, res.fail_column
        return self.ok

    def solve_block(self, B: np.ndarray) -> np.ndarray:
        """B: (q, n) FP64 host array; returns X (q, n)."""
        B = _f64(B)
        q = B.shape[0] if B.ndim == 2 else 1
        X = np.empty_like(B)
        if B.size:
            _check(lib().amp_solve(self._h, B.ctypes.data, q, X.ctypes.data, 0))
        elif not self.ok:
            _check(lib().amp_solve(self._h, None, q, None, 0))
        return X

    def solve_refined_block(self, B: np.ndarray, maxSteps: int = 3, tol: float = 1e-14):
        B = _f64(B)
        q = B.shape[0] if B.ndim == 2 else 1
        X = np.empty_like(B)
        st = _RefineStats()
        ro = _RefineOpts(maxSteps, tol)
        _check(lib().amp_solve_refined(self._h, B.ctypes.data if B.size else None, q,
                                       X.ctypes.data if X.size else None, 0, C.byref(ro), C.byref(st)))
        return X, st.rel_residual, st.steps

    def set_row_groups(self, offsets) -> None:
        """The factored matrix is block diagonal: rows [offsets[g], offsets[g + 1]) form independent systems.
        Refinement then stops when ||b - A x|| / ||b|| of every system and right-hand side is below tol, as separate
        solveRefined calls (ldlt.mjs:257-269) would. offsets=None clears."""
        if offsets is None:
            _check(lib().amp_factor_set_row_groups(self._h, 0, None))
            return
        o = np.ascontiguousarray(offsets, dtype=np.int64)
        _check(lib().amp_factor_set_row_groups(self._h, len(o) - 1, o.ctypes.data))

    def solve_gmres(self, b, tol: float = 1e-10, restart: int = 40, maxIter: int = 400) -> dict:
        """gmres(A, precond = this factor's solve, b, {tol, restart, maxIter}) (gmres-real.mjs:31-105) on the device,
        from x0 = 0: GMRES-based refinement with a mixed-precision factor. Returns {x, iterations, relres,
        converged} as the reference does."""
        bb = _f64(b)
        x = np.empty_like(bb)
        st = _GmresStats()
        _check(lib().amp_solve_gmres(self._h, bb.ctypes.data if bb.size else None, x.ctypes.data if x.size else None,
                                     0, C.byref(_GmresOpts(tol, restart, maxIter)), C.byref(st)))
        return {"x": x, "iterations": st.iterations, "relres": st.rel_residual, "converged": bool(st.converged)}

    def solve_gmres_ptr(self, b_ptr: int, x_ptr: int, on_device: bool, tol: float = 1e-10, restart: int = 40,
                        maxIter: int = 400):
        """solve_gmres for raw buffers (device, or host pinned): returns (relres, iterations, converged)."""
        st = _GmresStats()
        _check(lib().amp_solve_gmres(self._h, C.c_void_p(b_ptr), C.c_void_p(x_ptr), 1 if on_device else 0,
                                     C.byref(_GmresOpts(tol, restart, maxIter)), C.byref(st)))
        return st.rel_residual, st.iterations, bool(st.converged)

    @property
    def Lx(self) -> np.ndarray:
        out = np.zeros(max(self.sym.nnzLStored, 1))
        _check(lib().amp_factor_download(self._h, out.ctypes.data, None))
        return out[: self.sym.nnzLStored]

    @property
    def D(self) -> np.ndarray:
        out = np.zeros(max(self.sym.n, 1))
        _check(lib().amp_factor_download(self._h, None, out.ctypes.data))
        return out[: self.sym.n]

    def pivots(self):
        """(Doff, piv) of a Bunch-Kaufman factor: Doff[j] = D(j + 1, j) of a 2 x 2 pivot (j, j + 1), else 0; piv[f + c0
        + i] = the column of the pivot block at c0 of the supernode at f that became its i-th pivot."""
        n = max(self.sym.n, 1)
        doff, piv = np.zeros(n), np.zeros(n, np.int32)
        _check(lib().amp_factor_download_pivots(self._h, doff.ctypes.data, piv.ctypes.data))
        return doff[: self.sym.n], piv[: self.sym.n]

    def profile(self, enable: bool = True) -> None:
        """Time every kernel launch of the following calls with CUDA events (see profile_read)."""
        _check(lib().amp_profile_enable(self._h, 1 if enable else 0))

    def profile_launches(self, cap: int = 100000):
        """(kinds, ms, flops) arrays of the individual launches since profile(True); call before profile_read."""
        kinds = np.zeros(cap, np.int32)
        ms = np.zeros(cap)
        fl = np.zeros(cap)
        cnt = C.c_int32(0)
        _check(lib().amp_profile_launches(self._h, kinds.ctypes.data, ms.ctypes.data, fl.ctypes.data, cap,
                                          C.byref(cnt)))
        return kinds[: cnt.value], ms[: cnt.value], fl[: cnt.value]

    def profile_read(self) -> list:
        """Per kernel class: {name, launches, ms, flops, bytes} of the launches since profile(True)."""
        arr = (_KernelStat * 16)()
        cnt = C.c_int32(0)
        _check(lib().amp_profile_read(self._h, arr, 16, C.byref(cnt)))
        return [{"name": a.name.decode(), "launches": a.launches, "ms": a.ms, "flops": a.flops, "bytes": a.bytes}
                for a in arr[: cnt.value]]

    def solve_device(self, b_ptr: int, x_ptr: int, q: int = 1) -> None:
        """x = A^-1 b for device pointers (q vectors of length n one after another)."""
        _check(lib().amp_solve(self._h, C.c_void_p(b_ptr), q, C.c_void_p(x_ptr), 1))

    def solve_refined_device(self, b_ptr: int, x_ptr: int, q: int = 1, maxSteps: int = 3, tol: float = 1e-14):
        st = _RefineStats()
        ro = _RefineOpts(maxSteps, tol)
        _check(lib().amp_solve_refined(self._h, C.c_void_p(b_ptr), q, C.c_void_p(x_ptr), 1, C.byref(ro), C.byref(st)))
        return st.rel_residual, st.steps

    def solve_refined_host_pinned(self, b_ptr: int, x_ptr: int, q: int = 1, maxSteps: int = 3, tol: float = 1e-14):
        """solveRefined with host (pinned) buffers: the library copies b in and x out."""
        st = _RefineStats()
        ro = _RefineOpts(maxSteps, tol)
        _check(lib().amp_solve_refined(self._h, C.c_void_p(b_ptr), q, C.c_void_p(x_ptr), 0, C.byref(ro), C.byref(st)))
        return st.rel_residual, st.steps

    def set_mass(self, mvalues) -> None:
        """M's values on the factored pattern (the shift-invert operator op(X) = A^-1 M X, eigen.ts:150-160)."""
        m = _f64(mvalues)
        _check(lib().amp_factor_set_mass(self._h, m.ctypes.data if m.size else None, m.size, 0))

    def shift_invert_apply(self, X: np.ndarray) -> np.ndarray:
        """A^-1 (M X) for X (m, n) or (n,) on the device."""
        Xa = _f64(X)
        m = Xa.shape[0] if Xa.ndim == 2 else 1
        Y = np.empty_like(Xa)
        _check(lib().amp_shift_invert_apply(self._h, Xa.ctypes.data, m, Y.ctypes.data, 0))
        return Y

    def block_arnoldi(self, nWant: int, blockSize: int = 1, maxBasis: int = 0, tol: float = 1e-10,
                      maxRestarts: int = 60, seed: int = 20261014):
        """blockArnoldi with op = shift_invert_apply on the device (la/arnoldi.mjs:36-200): (mu (nWant,), Ritz
        vectors (nWant, n), stats dict); mu by decreasing modulus."""
        n = self.sym.n
        mu = np.zeros(max(nWant, 1))
        vecs = np.zeros((max(nWant, 1), n))
        st = _EigenStats()
        o = _EigenOpts(nWant, blockSize, maxBasis, maxRestarts, tol, seed & 0xFFFFFFFF)
        _check(lib().amp_eigen_block_arnoldi(self._h, C.byref(o), mu.ctypes.data, vecs.ctypes.data, 0, C.byref(st)))
        stats = {"converged": bool(st.converged), "restarts": st.restarts, "opVectors": st.op_vectors,
                 "basis": st.basis, "maxResidual": st.max_residual, "ms": st.ms}
        return mu[:nWant], vecs[:nWant], stats

    def set_wait_limit(self, polls: int) -> None:
        """Bound of this factor's device waits in polls (0 = the defaults, about a second). A wait that runs out
        makes the call raise AmpError with code AMP_DEVICE_TIMEOUT; the device stays usable."""
        _check(lib().amp_factor_set_wait_limit(self._h, int(polls)))

    def matVec(self, x) -> np.ndarray:
        xa = _f64(x)
        y = np.empty_like(xa)
        q = xa.shape[0] if xa.ndim == 2 else 1
        _check(lib().amp_matvec(self._h, xa.ctypes.data, q, y.ctypes.data))
        return y

    def __del__(self):
        h = self.__dict__.get("_h")
        if h and _lib is not None:
            _lib.amp_factor_destroy(h)
            self._h = None


class Assembly:
    """On-device assembly of a system's CSR values from its mesh (assembleCells, physics/src/common/scalar.ts:96-146,
    with the element slots of la/sparse.mjs:113-185 computed once): kind AMP_ELEM_P1_TRI_SCALAR (coefficient per
    triangle) or AMP_ELEM_P1_TET_ELASTIC ((E, nu) per tet)."""

    def __init__(self, kind: int, pat, coords, conn, dofs, device: int = 0):
        n, rp, ci = _pat(pat)
        self.kind, self.nnz = kind, int(rp[-1]) if n else 0
        self._keep = [np.ascontiguousarray(coords, np.float64), np.ascontiguousarray(conn, np.int32),
                      np.ascontiguousarray(dofs, np.int32)]
        xy, cn, dm = self._keep
        h = C.c_void_p()
        _check(lib().amp_assembly_create(kind, n, rp, ci, xy.shape[0], xy.ctypes.data, cn.shape[0], cn.ctypes.data,
                                         dm.ctypes.data, device, C.byref(h)))
        self._h = h.value

    def assemble(self, coef) -> np.ndarray:
        """The assembled values (host copy) for per-element coefficients."""
        c = _f64(coef)
        v = np.empty(self.nnz)
        _check(lib().amp_assemble(self._h, c.ctypes.data, 0, v.ctypes.data, 0, None))
        return v

    def assemble_device(self, coef_ptr: int, coef_on_device: bool, values_ptr: int, stream: int = 0) -> None:
        """Assemble into a device buffer of nnz doubles (coefficients from host or device memory)."""
        _check(lib().amp_assemble(self._h, C.c_void_p(coef_ptr), 1 if coef_on_device else 0, C.c_void_p(values_ptr),
                                  1, C.c_void_p(stream) if stream else None))

    def __del__(self):
        h = self.__dict__.get("_h")
        if h and _lib is not None:
            _lib.amp_assembly_destroy(h)
            self._h = None


def _nnz_of(sym: SymbolicAnalysis) -> int:
    return int(sym.patternKey.split(":")[1])


def factorNumeric(sym: SymbolicAnalysis, values, num: NumericFactor | None = None, pat=None,
                  opts: dict | None = None) -> NumericFactor:
    """factorNumeric(sym, values, num?, pat?, {factor?}) (sparse.mjs:941): ok = False when not positive definite."""
    if pat is not None:
        checkSymbolic(sym, pat)
    nv = len(values)
    if nv != _nnz_of(sym):
        raise AmpError(AMP_BAD_LENGTH, f"factorNumeric: {nv} values for a pattern with {_nnz_of(sym)} entries")
    if num is None or num.sym is not sym:
        num = NumericFactor(sym, CHOLESKY, FP64)
    num.factor(values)
    return num


def solveNumeric(num: NumericFactor, b, out=None) -> np.ndarray:
    """solveNumeric(num, b, out?) (sparse.mjs:1261)."""
    if num is None or not num.ok:
        raise AmpError(AMP_NO_FACTOR, "solveNumeric: no successful numeric factorization")
    x = num.solve_block(_f64(b).reshape(1, -1)).reshape(-1)
    if out is not None:
        out[:] = x
        return out
    return x


def solveNumericMulti(num: NumericFactor, bs: Sequence, outs=None) -> list:
    """solveNumericMulti(num, bs[], outs?) (sparse.mjs:1308): one pass over the factor for all vectors."""
    if num is None or not num.ok:
        raise AmpError(AMP_NO_FACTOR, "solveNumericMulti: no successful numeric factorization")
    if len(bs) == 0:
        return []
    X = num.solve_block(np.stack([_f64(b) for b in bs]))
    res = []
    for k in range(len(bs)):
        if outs is not None and outs[k] is not None:
            outs[k][:] = X[k]
            res.append(outs[k])
        else:
            res.append(X[k].copy())
    return res


def matVec(pat, val, x, out=None, device: int = 0) -> np.ndarray:
    """y = A x on full CSR storage (sparse.mjs:219-228), computed on the GPU (amp_matvec_csr)."""
    n, rp, ci = _pat(pat)
    v = _f64(val)
    xa = _f64(x)
    y = np.empty_like(xa)
    q = xa.shape[0] if xa.ndim == 2 else 1
    if len(v) != int(rp[-1] if n else 0):
        raise ValueError(f"matVec: {len(v)} values for a pattern with {int(rp[-1]) if n else 0} entries")
    _check(lib().amp_matvec_csr(n, rp, ci, v.ctypes.data if v.size else None, xa.ctypes.data if xa.size else None, q,
                                y.ctypes.data if y.size else None, device))
    if out is not None:
        out[:] = y
        return out
    return y


class SparseCholesky:
    """new SparseCholesky(pat, perm?, {sym, ordering, x, y, factor}) (sparse.mjs:1318-1372)."""

    def __init__(self, pat, perm=None, sym: SymbolicAnalysis | None = None, ordering: str = "amd", x=None, y=None,
                 z=None, factor=None, precision: int = FP64):
        t0 = time.perf_counter()
        self.factorKind = factor
        if sym is not None:
            checkSymbolic(sym, pat)
            self.sym = sym
        else:
            self.sym = analyze(pat, {"perm": perm} if perm is not None else {"ordering": ordering, "x": x, "y": y,
                                                                             "z": z})
        self.n = int(pat.n)
        self.perm = self.sym.perm
        self.nnzL = self.sym.nnzL
        self.num = None
        self.ok = False
        self.precision = precision
        reused = sym is not None
        self.timing = {"n": self.n, "nnzA": self.sym.nnzA, "nnzL": self.nnzL, "fill": self.sym.fill,
                       "flops": self.sym.flops, "nsuper": self.sym.nsuper, "symbolicReused": reused,
                       "ordering_ms": 0.0 if reused else self.sym.timing["ordering_ms"],
                       "symbolic_ms": 0.0 if reused else (time.perf_counter() - t0) * 1e3 -
                       self.sym.timing["ordering_ms"], "factor_ms": 0.0, "nFactor": 0, "solve_ms": 0.0, "nSolve": 0,
                       "kernel": "cuda-sm100a"}

    def factor(self, values) -> bool:
        t0 = time.perf_counter()
        nv = len(values)
        if nv != _nnz_of(self.sym):
            raise AmpError(AMP_BAD_LENGTH, f"factorNumeric: {nv} values for a pattern with {_nnz_of(self.sym)} entries")
        if self.num is None:
            self.num = NumericFactor(self.sym, CHOLESKY, self.precision)
        self.ok = self.num.factor(values)
        self.timing["factor_ms"] += (time.perf_counter() - t0) * 1e3
        self.timing["nFactor"] += 1
        return self.ok

    def solve(self, b, out=None) -> np.ndarray:
        t0 = time.perf_counter()
        if not self.ok:
            raise AmpError(AMP_NO_FACTOR, "SparseCholesky: solve without a successful factorization")
        r = solveNumeric(self.num, b, out)
        self.timing["solve_ms"] += (time.perf_counter() - t0) * 1e3
        self.timing["nSolve"] += 1
        return r

    def solveMany(self, bs, outs=None) -> list:
        t0 = time.perf_counter()
        if not self.ok:
            raise AmpError(AMP_NO_FACTOR, "SparseCholesky: solve without a successful factorization")
        r = solveNumericMulti(self.num, bs, outs)
        self.timing["solve_ms"] += (time.perf_counter() - t0) * 1e3
        self.timing["nSolve"] += len(bs)
        return r


class SupernodalLDLT:
    """Real symmetric LDL^T over a supernodal analysis: 1x1 pivots with static perturbation (|d| < tau -> +-tau,
    tau = pivotTol * max |A(i, i)|), inertia and refinement (ldlt.mjs:431-645). Factor and solves run on the GPU.

    pivoting="bunch-kaufman" (no reference counterpart; FP64) chooses 1 x 1 and 2 x 2 pivots by the Bunch-Kaufman rule
    inside each 64-column pivot block of every supernode (the symbolic structure is unchanged); a column with no entry
    at or above tau still takes the static perturbation. nNeg counts the negative eigenvalues of D's blocks."""

    def __init__(self, sym: SymbolicAnalysis, factor=None, precision: int = FP64, pivoting: str = "static"):
        if pivoting not in ("static", "bunch-kaufman"):
            raise AmpError(AMP_INVALID, f"SupernodalLDLT: unknown pivoting {pivoting!r}")
        self.sym = sym
        self.factorKind = factor
        self.pivoting = pivoting
        self.kernel = "cuda-sm100a"
        self.num = NumericFactor(sym, LDLT_BK if pivoting == "bunch-kaufman" else LDLT, precision)
        self.nnzL = sym.nnzL
        self.nNeg = 0
        self.nPerturbed = 0
        self.ok = False

    def factor(self, values, pivotTol: float = 1e-13) -> dict:
        nv = len(values)
        if nv != _nnz_of(self.sym):
            raise AmpError(AMP_BAD_LENGTH, f"factorNumeric: {nv} values for a pattern with {_nnz_of(self.sym)} entries")
        self.ok = self.num.factor(values, pivotTol=pivotTol)
        self.nNeg, self.nPerturbed = self.num.nNeg, self.num.nPerturbed
        return {"ok": self.ok, "nNeg": self.nNeg, "nPerturbed": self.nPerturbed, "ms": self.num.ms}

    @property
    def Lx(self) -> np.ndarray:
        return self.num.Lx

    @property
    def D(self) -> np.ndarray:
        return self.num.D

    def _need(self):
        if not self.ok:
            raise AmpError(AMP_NO_FACTOR, "solveNumeric: no successful numeric factorization")

    def solve(self, b, out=None) -> np.ndarray:
        self._need()
        x = self.num.solve_block(_f64(b)[None, :])[0]
        if out is not None:
            out[:] = x
            return out
        return x

    def solveMany(self, b, q: int, out=None) -> np.ndarray:
        """q right-hand sides stored one after another in b (b[k n + i]); one device pass per sweep for all q."""
        self._need()
        n = self.sym.n
        x = self.num.solve_block(_f64(b).reshape(q, n)).reshape(q * n)
        if out is not None:
            out[:] = x
            return out
        return x

    def solveRefined(self, pat, values, b, maxSteps: int = 3, tol: float = 1e-14) -> dict:
        """Refinement against the factored (unperturbed) matrix: r = b - A x, x += solve(r) (ldlt.mjs:253-275).
        `pat` / `values` must be the pattern and values that were factored; the residual runs on the device copy."""
        self._need()
        checkSymbolic(self.sym, pat)
        if len(values) != _nnz_of(self.sym):
            raise AmpError(AMP_BAD_LENGTH, f"solveRefined: {len(values)} values for a pattern with "
                                           f"{_nnz_of(self.sym)} entries")
        X, rel, steps = self.num.solve_refined_block(_f64(b)[None, :], maxSteps=maxSteps, tol=tol)
        return {"x": X[0], "relResidual": rel, "steps": steps}

    def solveGmres(self, b, tol: float = 1e-10, restart: int = 40, maxIter: int = 400) -> dict:
        """FP64 GMRES on the factored matrix preconditioned by this factor (GMRES-IR for a mixed-precision factor of
        an indefinite matrix, gmres-real.mjs:31-105)."""
        self._need()
        return self.num.solve_gmres(b, tol=tol, restart=restart, maxIter=maxIter)


class ComplexSupernodalLDLT:
    """Complex-symmetric multifrontal LDL^T (A = A^T, no conjugation) over a supernodal analysis, on the GPU: the
    reference's ComplexSupernodalLDLT (ldlt.mjs:648-864) with its solveRefined (:870-900). Values and right-hand sides
    are (re, im) pairs of FP64 arrays on the CSR slots / rows, as the reference takes them."""

    def __init__(self, sym: SymbolicAnalysis):
        self.sym = sym
        self.kernel = "cuda-sm100a"
        self.ok = False
        self.nPerturbed = 0
        h = C.c_void_p()
        _check(lib().amp_cfactor_create(sym.handle, C.byref(h)))
        self._h = h.value

    def factor(self, re, im, pivotTol: float = 1e-13) -> dict:
        r, i = _f64(re), _f64(im)
        if len(r) != _nnz_of(self.sym) or len(i) != len(r):
            raise AmpError(AMP_BAD_LENGTH, f"factorNumeric: {len(r)} values for a pattern with "
                                           f"{_nnz_of(self.sym)} entries")
        res = _FactorResult()
        _check(lib().amp_cfactor_numeric(self._h, r.ctypes.data if r.size else None,
                                         i.ctypes.data if i.size else None, r.size, 0, pivotTol, C.byref(res)))
        self.ok, self.nPerturbed = bool(res.ok), res.n_perturbed
        return {"ok": self.ok, "nPerturbed": self.nPerturbed, "ms": res.ms}

    def _need(self):
        if not self.ok:
            raise AmpError(AMP_NO_FACTOR, "solveNumeric: no successful numeric factorization")

    def solve(self, br, bi) -> dict:
        self._need()
        r, i = _f64(br), _f64(bi)
        xr, xi = np.empty_like(r), np.empty_like(i)
        _check(lib().amp_csolve(self._h, r.ctypes.data, i.ctypes.data, 1, xr.ctypes.data, xi.ctypes.data, 0))
        return {"re": xr, "im": xi}

    def solveRefined(self, pat, re, im, br, bi, maxSteps: int = 3, tol: float = 1e-14) -> dict:
        """Refinement against the factored (unperturbed) values; `pat`, `re`, `im` must be what was factored."""
        self._need()
        checkSymbolic(self.sym, pat)
        if len(re) != _nnz_of(self.sym):
            raise AmpError(AMP_BAD_LENGTH, f"solveRefined: {len(re)} values for a pattern with "
                                           f"{_nnz_of(self.sym)} entries")
        r, i = _f64(br), _f64(bi)
        xr, xi = np.empty_like(r), np.empty_like(i)
        st = _RefineStats()
        _check(lib().amp_csolve_refined(self._h, r.ctypes.data, i.ctypes.data, 1, xr.ctypes.data, xi.ctypes.data, 0,
                                        C.byref(_RefineOpts(maxSteps, tol)), C.byref(st)))
        return {"re": xr, "im": xi, "relResidual": st.rel_residual, "steps": st.steps}

    def factors(self):
        """(Lr, Li, Dr, Di) host copies."""
        nl, n = max(self.sym.nnzLStored, 1), max(self.sym.n, 1)
        Lr, Li, Dr, Di = np.zeros(nl), np.zeros(nl), np.zeros(n), np.zeros(n)
        _check(lib().amp_cfactor_download(self._h, Lr.ctypes.data, Li.ctypes.data, Dr.ctypes.data, Di.ctypes.data))
        return Lr[: self.sym.nnzLStored], Li[: self.sym.nnzLStored], Dr[: self.sym.n], Di[: self.sym.n]

    def __del__(self):
        h = self.__dict__.get("_h")
        if h and _lib is not None:
            _lib.amp_factor_destroy(h)
            self._h = None


# ---- 'auto' choice between the direct solver and the iterative one ----------------------------------------------------
# The reference's study setting 'auto' (physics/src/common/scalar.ts:264-283) picks AMG-PCG over the direct factor when
# the factor's symbolic flops per DOF reach a break-even measured for its single-threaded CPU factor (3e5 flop/DOF: a
# 15.6k-node tet10 heat pattern at 2.7e5 had both within 10%), or when 8 nnzL bytes exceed a 1 GiB memory budget.
AUTO_FLOPS_PER_DOF_CPU = 3e5
AUTO_MAX_FACTOR_BYTES_CPU = 2 ** 30
# The same rule for this GPU factor. AMG-PCG (on the host, as in the reference) costs about 3e5 flop/DOF at the CPU
# factor's 23 GFlop/s, i.e. about 13 us per DOF. The GPU factor + solve runs at 13 TFLOP/s end to end on the 3D
# elasticity system in FP64 (0.79 TFLOP in 60 ms, its slowest measured rate; 26 in mixed precision, 63 on the 3D P2
# heat system), so the break-even is 13e-6 s x 13e12 flop/s = 1.7e8 flop/DOF; the memory bound is the factor's
# device memory (L, update arena and schedule) against a budget of 128 GiB of the B200's 180 GB.
AUTO_FLOPS_PER_DOF_GPU = 1.7e8
AUTO_MAX_FACTOR_BYTES_GPU = 128 * 2 ** 30


def autoSolverChoice(n: int, flops: float, nnzL: int, factorBytes: int | None = None,
                     flopsPerDof: float = AUTO_FLOPS_PER_DOF_GPU, maxFactorBytes: int = AUTO_MAX_FACTOR_BYTES_GPU) -> dict:
    """{'kind': 'cholesky' | 'amg-pcg', 'reason': str} for a pattern with n rows and an analysis giving flops and nnzL
    (autoSolverChoice, scalar.ts:271-276: the memory test first, then flop/DOF against the break-even). factorBytes:
    the factor's memory (the plan's deviceBytes); 8 nnzL when None, as the reference counts it. With
    flopsPerDof=AUTO_FLOPS_PER_DOF_CPU and maxFactorBytes=AUTO_MAX_FACTOR_BYTES_CPU the choice and the message are the
    reference's."""
    fpd = flops / max(n, 1)
    nbytes = 8 * nnzL if factorBytes is None else factorBytes
    if nbytes > maxFactorBytes:
        return {"kind": "amg-pcg",
                "reason": f"direct factor {_js_fixed0(nbytes / 2 ** 20)} MiB > {_js_num(maxFactorBytes / 2 ** 20)} MiB"}
    if fpd >= flopsPerDof:
        return {"kind": "amg-pcg", "reason": f"direct factor {_js_exp(fpd, 2)} flop/DOF >= {_js_exp(flopsPerDof, 0)}"}
    return {"kind": "cholesky", "reason": f"direct factor {_js_exp(fpd, 2)} flop/DOF < {_js_exp(flopsPerDof, 0)}"}


def _js_exp(x: float, digits: int) -> str:
    """Number.prototype.toExponential(digits) of x >= 0: the exact value rounded half up, '2.70e+5'."""
    if x == 0:
        return f"{0:.{digits}f}e+0"
    d = Decimal(x)
    e = d.adjusted()
    q = Decimal(1).scaleb(-digits)
    m = d.scaleb(-e).quantize(q, rounding=ROUND_HALF_UP)
    if m >= 10:
        e += 1
        m = d.scaleb(-e).quantize(q, rounding=ROUND_HALF_UP)
    return f"{m}e{'+' if e >= 0 else '-'}{abs(e)}"


def _js_fixed0(x: float) -> str:
    """Number.prototype.toFixed(0) of x >= 0 (half up)."""
    return str(Decimal(x).quantize(Decimal(1), rounding=ROUND_HALF_UP))


def _js_num(x: float) -> str:
    """String(x) for the whole numbers used here."""
    return str(int(x)) if x == int(x) else repr(x)


def autoSolverChoiceFor(sym: SymbolicAnalysis, **kw) -> dict:
    """autoSolverChoice from an analysis, with the factor's device memory as its size."""
    return autoSolverChoice(sym.n, sym.flops, sym.nnzL, factorBytes=kw.pop("factorBytes", sym.deviceBytes), **kw)
