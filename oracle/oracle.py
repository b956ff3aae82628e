"""ctypes binding of the CPU oracle (oracle/amp_oracle.c). TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` / ``--impl reference`` legs of bench.py import this
module, and only as the checker or the timed CPU baseline; the product library never links or calls it.

Every function restates the reference (jwt625/applied-multiphysics, packages/core/src/la/) line by line; the C file
cites the reference file:line per function. Patterns are any object with ``n``, ``rowptr`` (int32) and ``colidx``
(int32) attributes (full symmetric CSR storage, sorted rows, diagonal present).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libamporacle.so")
_lib = None

_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")


def build() -> str:
    """Compile the oracle (make in oracle/); returns the library path."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        L.orc_fingerprint_hash.restype = C.c_uint32
        L.orc_fingerprint_hash.argtypes = [C.c_int, _i32p, _i32p]
        L.orc_amd_order.restype = C.c_int
        L.orc_amd_order.argtypes = [C.c_int, _i32p, _i32p, C.c_double, _i32p]
        L.orc_nd_order.restype = C.c_int
        L.orc_nd_order.argtypes = [C.c_int, _i32p, _i32p, _f64p, _f64p, C.c_int, _i32p]
        L.orc_nd3_order.restype = C.c_int
        L.orc_nd3_order.argtypes = [C.c_int, _i32p, _i32p, _f64p, _f64p, _f64p, C.c_int, _i32p]
        L.orc_analyze.restype = C.c_void_p
        L.orc_analyze.argtypes = [C.c_int, _i32p, _i32p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_int,
                                  C.POINTER(C.c_int)]
        L.orc_sym_free.argtypes = [C.c_void_p]
        L.orc_sym_info.argtypes = [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int64), C.POINTER(C.c_double)]
        L.orc_sym_arrays.argtypes = [C.c_void_p, C.POINTER(C.c_void_p)]
        L.orc_factor.restype = C.c_int
        L.orc_factor.argtypes = [C.c_void_p, _f64p, C.c_int, C.c_int, C.c_double, _f64p, _f64p, _i32p]
        L.orc_factor_range.restype = C.c_int
        L.orc_factor_range.argtypes = [C.c_void_p, _f64p, C.c_int, C.c_int, C.c_double, _f64p, _f64p, _i32p, C.c_int,
                                       C.c_int]
        L.orc_solve_chol.argtypes = [C.c_void_p, _f64p, _f64p, _f64p, C.c_int]
        L.orc_solve_ldlt.argtypes = [C.c_void_p, _f64p, _f64p, _f64p, C.c_int, _f64p, C.c_int]
        L.orc_matvec.argtypes = [C.c_int, _i32p, _i32p, _f64p, _f64p, _f64p]
        L.orc_solve_refined.restype = C.c_int
        L.orc_solve_refined.argtypes = [C.c_void_p, _i32p, _i32p, _f64p, _f64p, _f64p, C.c_int, _f64p, C.c_int,
                                        C.c_double, _f64p, C.POINTER(C.c_double)]
        L.orc_cfactor.restype = C.c_int
        L.orc_cfactor.argtypes = [C.c_void_p, _f64p, _f64p, C.c_double, _f64p, _f64p, _f64p, _f64p, _i32p]
        L.orc_csolve.argtypes = [C.c_void_p, _f64p, _f64p, _f64p, _f64p, _f64p, _f64p, _f64p, _f64p]
        L.orc_up_create.restype = C.c_void_p
        L.orc_up_create.argtypes = [C.c_int, _i32p, _i32p, _i32p]
        L.orc_up_Lp.restype = C.POINTER(C.c_int)
        L.orc_up_Lp.argtypes = [C.c_void_p]
        L.orc_up_nnzL.restype = C.c_int64
        L.orc_up_nnzL.argtypes = [C.c_void_p]
        L.orc_up_factor.restype = C.c_int
        L.orc_up_factor.argtypes = [C.c_void_p, _f64p]
        L.orc_up_solve.argtypes = [C.c_void_p, _f64p, _f64p]
        L.orc_up_free.argtypes = [C.c_void_p]
        L.orc_ldlt_up.restype = C.c_int
        L.orc_ldlt_up.argtypes = [C.c_int, _i32p, _i32p, _i32p, _f64p, C.c_double, C.c_void_p, C.c_void_p, _i32p]
        _lib = L
    return _lib


def _pat(pat):
    return (int(pat.n), np.ascontiguousarray(pat.rowptr, dtype=np.int32),
            np.ascontiguousarray(pat.colidx, dtype=np.int32))


def fingerprint(pat) -> str:
    """patternFingerprint (sparse.mjs:908-925): "n:nnz:hash"."""
    n, rp, ci = _pat(pat)
    h = lib().orc_fingerprint_hash(n, rp, ci)
    return f"{n}:{int(rp[n])}:{h:x}"


def amd_order(pat, dense_factor: float = 10.0) -> np.ndarray:
    n, rp, ci = _pat(pat)
    out = np.zeros(max(n, 1), np.int32)
    if lib().orc_amd_order(n, rp, ci, dense_factor, out) != 0:
        raise RuntimeError("amdOrder: internal error")
    return out[:n]


def nd_order(pat, x, y, leaf: int = 48) -> np.ndarray:
    n, rp, ci = _pat(pat)
    out = np.zeros(max(n, 1), np.int32)
    lib().orc_nd_order(n, rp, ci, np.ascontiguousarray(x, np.float64), np.ascontiguousarray(y, np.float64), leaf, out)
    return out[:n]


def nd3_order(pat, x, y, z, leaf: int = 2000) -> np.ndarray:
    n, rp, ci = _pat(pat)
    out = np.zeros(max(n, 1), np.int32)
    lib().orc_nd3_order(n, rp, ci, np.ascontiguousarray(x, np.float64), np.ascontiguousarray(y, np.float64),
                        np.ascontiguousarray(z, np.float64), leaf, out)
    return out[:n]


_FIELDS = ["perm", "pinv", "parent", "colCount", "lowerP", "lowerI", "lowerSrc", "superStart", "colSuper",
           "superParent", "childHead", "childNext", "Sp", "Si", "Lxp"]


class Symbolic:
    """Result of the oracle's analyze (sparse.mjs:666-902); arrays are numpy copies, ``handle`` the C object."""

    def __init__(self, handle):
        self.handle = handle
        L = lib()
        ints = (C.c_int * 5)()
        longs = (C.c_int64 * 3)()
        dbls = (C.c_double * 2)()
        L.orc_sym_info(handle, ints, longs, dbls)
        self.n, self.nsuper, self.maxFront, self.patNnz = ints[0], ints[1], ints[2], ints[3]
        self.hash = ints[4] & 0xFFFFFFFF
        self.nnzL, self.nnzA, self.nnzLStored = longs[0], longs[1], longs[2]
        self.fill, self.flops = dbls[0], dbls[1]
        ptrs = (C.c_void_p * 15)()
        L.orc_sym_arrays(handle, ptrs)
        n, ns = self.n, self.nsuper
        lens = {"perm": n, "pinv": n, "parent": n, "colCount": n, "lowerP": n + 1, "lowerI": self.nnzA,
                "lowerSrc": self.nnzA, "superStart": ns + 1, "colSuper": n, "superParent": ns, "childHead": ns,
                "childNext": ns, "Sp": ns + 1, "Si": None, "Lxp": ns + 1}
        for i, name in enumerate(_FIELDS):
            ln = lens[name]
            if name == "Si":
                ln = int(self.Sp[ns]) if ns > 0 else 0
            if name == "Lxp":
                arr = np.ctypeslib.as_array(C.cast(ptrs[i], C.POINTER(C.c_int64)), shape=(ln,)).copy() if ln else \
                    np.zeros(0, np.int64)
            elif ln == 0 or not ptrs[i]:
                arr = np.zeros(ln, np.int32) if not ptrs[i] else \
                    np.ctypeslib.as_array(C.cast(ptrs[i], C.POINTER(C.c_int32)), shape=(max(ln, 1),))[:ln].copy()
            else:
                arr = np.ctypeslib.as_array(C.cast(ptrs[i], C.POINTER(C.c_int32)), shape=(ln,)).copy()
            setattr(self, name, arr)
        self.patternKey = f"{self.n}:{self.patNnz}:{self.hash:x}"

    def __del__(self):
        if getattr(self, "handle", None) and _lib is not None:
            _lib.orc_sym_free(self.handle)
            self.handle = None


def analyze(pat, perm=None, ordering: str = "amd", x=None, y=None, relax: bool = True) -> Symbolic:
    n, rp, ci = _pat(pat)
    err = C.c_int(0)
    keep = []
    pp = None
    if perm is not None:
        pa = np.ascontiguousarray(perm, np.int32)
        if pa.shape[0] != n:
            raise ValueError(f"analyze: perm has length {pa.shape[0]}, pattern has {n} rows")
        keep.append(pa)
        pp = pa.ctypes.data
    xp = yp = None
    if ordering == "nd" and perm is None:
        if x is None or y is None or len(x) != n or len(y) != n:
            raise ValueError("analyze: ordering nd needs node coordinates x and y of length n")
        xa, ya = np.ascontiguousarray(x, np.float64), np.ascontiguousarray(y, np.float64)
        keep += [xa, ya]
        xp, yp = xa.ctypes.data, ya.ctypes.data
    h = lib().orc_analyze(n, rp, ci, pp, 1 if ordering == "nd" else 0, xp, yp, 1 if relax else 0, C.byref(err))
    if not h:
        raise RuntimeError(f"oracle analyze failed (code {err.value})")
    return Symbolic(h)


def factor(sym: Symbolic, values, kind: str = "chol", simd: bool = False, pivot_tol: float = 1e-13):
    """Multifrontal factor (sparse.mjs factorNumeric / ldlt.mjs SupernodalLDLT.factor).

    simd=False: the JS "blocked" loops; simd=True: the SSE2 restatement of the WASM front kernel for m >= 32.
    Returns (ok, Lx, D, nNeg, nPerturbed); D is None for Cholesky.
    """
    v = np.ascontiguousarray(values, np.float64)
    Lx = np.zeros(max(int(sym.nnzLStored), 1), np.float64)
    D = np.zeros(max(sym.n, 1), np.float64)
    st = np.zeros(2, np.int32)
    ok = lib().orc_factor(sym.handle, v if v.size else np.zeros(1), 0 if kind == "chol" else 1, 1 if simd else 0,
                          pivot_tol, Lx, D, st)
    return bool(ok), Lx[: sym.nnzLStored], (None if kind == "chol" else D[: sym.n]), int(st[0]), int(st[1])


def subtree_first(sym: Symbolic, root: int) -> int:
    """First supernode (in postorder) of the subtree rooted at supernode `root`."""
    first = root
    stack = [root]
    ch = [[] for _ in range(sym.nsuper)]
    for s in range(sym.nsuper):
        if sym.superParent[s] >= 0:
            ch[sym.superParent[s]].append(s)
    while stack:
        s = stack.pop()
        first = min(first, s)
        stack.extend(ch[s])
    return first


def factor_subtree(sym: Symbolic, values, root: int, kind: str = "chol", simd: bool = True, pivot_tol: float = 1e-13):
    """Factor only the subtree rooted at supernode `root` (a bounded CPU sample); returns (ok, flops of the sample)."""
    s0 = subtree_first(sym, root)
    v = np.ascontiguousarray(values, np.float64)
    Lx = np.zeros(max(int(sym.nnzLStored), 1), np.float64)
    D = np.zeros(max(sym.n, 1), np.float64)
    st = np.zeros(2, np.int32)
    ok = lib().orc_factor_range(sym.handle, v, 0 if kind == "chol" else 1, 1 if simd else 0, pivot_tol, Lx, D, st,
                                s0, root)
    c0, c1 = int(sym.superStart[s0]), int(sym.superStart[root + 1])
    flops = float(np.sum(sym.colCount[c0:c1].astype(np.float64) ** 2))
    return bool(ok), flops


def solve_chol(sym: Symbolic, Lx, b, simd: bool = False) -> np.ndarray:
    x = np.zeros(max(sym.n, 1))
    lib().orc_solve_chol(sym.handle, np.ascontiguousarray(Lx if len(Lx) else np.zeros(1), np.float64),
                         np.ascontiguousarray(b if len(b) else np.zeros(1), np.float64), x, 1 if simd else 0)
    return x[: sym.n]


def solve_ldlt(sym: Symbolic, Lx, D, b, q: int = 1, simd: bool = False) -> np.ndarray:
    x = np.zeros(max(sym.n * q, 1))
    lib().orc_solve_ldlt(sym.handle, np.ascontiguousarray(Lx, np.float64), np.ascontiguousarray(D, np.float64),
                         np.ascontiguousarray(b, np.float64), q, x, 1 if simd else 0)
    return x[: sym.n * q]


def matvec(pat, values, x) -> np.ndarray:
    n, rp, ci = _pat(pat)
    y = np.zeros(max(n, 1))
    lib().orc_matvec(n, rp, ci, np.ascontiguousarray(values, np.float64), np.ascontiguousarray(x, np.float64), y)
    return y[:n]


def solve_refined(sym: Symbolic, pat, values, Lx, D, b, kind: str = "ldlt", max_steps: int = 3, tol: float = 1e-14):
    n, rp, ci = _pat(pat)
    x = np.zeros(max(n, 1))
    rel = C.c_double(0)
    Dv = np.ascontiguousarray(D if D is not None else np.zeros(1), np.float64)
    steps = lib().orc_solve_refined(sym.handle, rp, ci, np.ascontiguousarray(values, np.float64),
                                    np.ascontiguousarray(Lx, np.float64), Dv, 0 if kind == "chol" else 1,
                                    np.ascontiguousarray(b, np.float64), max_steps, tol, x, C.byref(rel))
    return x[:n], rel.value, steps


def cfactor(sym: Symbolic, re, im, pivot_tol: float = 1e-13):
    """ComplexSupernodalLDLT.factor(re, im, {pivotTol}) (ldlt.mjs:667-800): (ok, Lr, Li, Dr, Di, nPerturbed)."""
    n, nl = max(sym.n, 1), max(int(sym.nnzLStored), 1)
    Lr, Li, Dr, Di = np.zeros(nl), np.zeros(nl), np.zeros(n), np.zeros(n)
    st = np.zeros(2, np.int32)
    ok = lib().orc_cfactor(sym.handle, np.ascontiguousarray(re, np.float64), np.ascontiguousarray(im, np.float64),
                           pivot_tol, Lr, Li, Dr, Di, st)
    k = int(sym.nnzLStored)
    return bool(ok), Lr[:k], Li[:k], Dr[: sym.n], Di[: sym.n], int(st[0])


def csolve(sym: Symbolic, Lr, Li, Dr, Di, br, bi):
    """ComplexSupernodalLDLT.solve(br, bi) (ldlt.mjs:802-862): (xr, xi)."""
    n = max(sym.n, 1)
    xr, xi = np.zeros(n), np.zeros(n)
    f = lambda a: np.ascontiguousarray(a if len(a) else np.zeros(1), np.float64)  # noqa: E731
    lib().orc_csolve(sym.handle, f(Lr), f(Li), f(Dr), f(Di), f(br), f(bi), xr, xi)
    return xr[: sym.n], xi[: sym.n]


def cmatvec(pat, re, im, xr, xi):
    """y = A x for complex A = re + i im on the pattern and complex x (the residual of complexSolveRefined)."""
    yr = matvec(pat, re, xr) - matvec(pat, im, xi)
    yi = matvec(pat, re, xi) + matvec(pat, im, xr)
    return yr, yi


class UpLookingCholesky:
    """The reference's own test oracle (sparse.mjs:1379-1544)."""

    def __init__(self, pat, perm):
        n, rp, ci = _pat(pat)
        self.n = n
        self._h = lib().orc_up_create(n, rp, ci, np.ascontiguousarray(perm, np.int32))
        self.nnzL = int(lib().orc_up_nnzL(self._h))
        self.Lp = np.ctypeslib.as_array(lib().orc_up_Lp(self._h), shape=(n + 1,)).copy()

    def factor(self, values) -> bool:
        return bool(lib().orc_up_factor(self._h, np.ascontiguousarray(values, np.float64)))

    def solve(self, b) -> np.ndarray:
        x = np.zeros(max(self.n, 1))
        lib().orc_up_solve(self._h, np.ascontiguousarray(b, np.float64), x)
        return x[: self.n]

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.orc_up_free(self._h)
            self._h = None


def ldlt_up(pat, perm, values, pivot_tol: float = 1e-13, b=None):
    """Up-looking LDL^T (ldlt.mjs SymbolicLDLT + LDLT): returns (ok, nNeg, nPerturbed, x or None)."""
    n, rp, ci = _pat(pat)
    st = np.zeros(2, np.int32)
    x = np.zeros(max(n, 1)) if b is not None else None
    bb = np.ascontiguousarray(b, np.float64) if b is not None else None
    ok = lib().orc_ldlt_up(n, rp, ci, np.ascontiguousarray(perm, np.int32), np.ascontiguousarray(values, np.float64),
                           pivot_tol, bb.ctypes.data if bb is not None else None,
                           x.ctypes.data if x is not None else None, st)
    return bool(ok), int(st[0]), int(st[1]), (x[:n] if x is not None else None)
