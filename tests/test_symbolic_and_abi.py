"""CPU tests of the product's host side: symbolic phase vs the oracle (bit-exact), the C ABI, the Python mirror.

No GPU is touched: analyze, the orderings and the fingerprint run on the host inside libampsolve.so, and the error
paths below are all raised before any device work (sparse.mjs:666-930 for the reference behaviour).
"""
import ctypes as C
import os
import re

import numpy as np
import pytest

import ampsolve as A
import oracle as O
import workloads as W

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "ampsolve.h")

SYM_FIELDS = ["perm", "pinv", "parent", "colCount", "lowerP", "lowerI", "lowerSrc", "superStart", "colSuper",
              "superParent", "childHead", "childNext", "Sp", "Si", "Lxp"]


def assert_same_symbolic(ps, osym):
    assert (ps.n, ps.nsuper, ps.maxFront) == (osym.n, osym.nsuper, osym.maxFront)
    assert (ps.nnzL, ps.nnzA, ps.nnzLStored) == (osym.nnzL, osym.nnzA, osym.nnzLStored)
    assert ps.flops == osym.flops and ps.fill == osym.fill
    assert ps.patternKey == osym.patternKey
    for f in SYM_FIELDS:
        a, b = np.asarray(getattr(ps, f)), np.asarray(getattr(osym, f))
        assert a.shape == b.shape, f
        assert np.array_equal(a.astype(np.int64), b.astype(np.int64)), f


CASES = [
    ("hex654-amd", lambda: W.hex_q1(6, 5, 4), "amd"),
    ("hex884-nd", lambda: W.hex_q1(8, 8, 4), "nd"),
    ("poisson2d-32-amd", lambda: W.poisson2d(32), "amd"),
    ("poisson2d-40-nd", lambda: W.poisson2d(40), "nd"),
    ("grid27-9-amd", lambda: W.grid27(9, 9, 9, sym=True), "amd"),
    ("chain-200-amd", lambda: W.chain(200), "amd"),
    ("elastic3d-6-nd3", lambda: W.elastic3d(6), "nd3"),
    ("heat3d-p2-3-nd3", lambda: W.heat3d_p2(3, 4, 0.2, 4, 1), "nd3"),
    ("maxwell3d-4-nd3", lambda: W.maxwell3d(4, 2, 12.0, 0.0, 5, 1), "nd3"),
]


@pytest.mark.parametrize("relax", [True, False])
@pytest.mark.parametrize("name,make,ordering", CASES, ids=[c[0] for c in CASES])
def test_product_symbolic_equals_oracle(name, make, ordering, relax):
    w = make()
    if ordering == "nd3":
        leaf = 40
        operm = O.nd3_order(w.pat, w.x, w.y, w.z, leaf)
        assert np.array_equal(A.nd3Order(w.pat, w.x, w.y, w.z, leaf), operm)
        osym = O.analyze(w.pat, perm=operm, relax=relax)
        ps = A.analyze(w.pat, ordering="nd3", x=w.x, y=w.y, z=w.z, leaf=leaf, relax=relax)
    elif ordering == "nd":
        assert np.array_equal(A.ndOrder(w.pat, w.x, w.y), O.nd_order(w.pat, w.x, w.y))
        osym = O.analyze(w.pat, ordering="nd", x=w.x, y=w.y, relax=relax)
        ps = A.analyze(w.pat, ordering="nd", x=w.x, y=w.y, relax=relax)
    else:
        assert np.array_equal(A.amdOrder(w.pat), O.amd_order(w.pat))
        osym = O.analyze(w.pat, relax=relax)
        ps = A.analyze(w.pat, relax=relax)
    assert_same_symbolic(ps, osym)
    assert A.patternFingerprint(w.pat) == O.fingerprint(w.pat)


def test_product_symbolic_given_perm_and_dense_factor():
    w = W.hex_q1(5, 4, 3)
    rng = np.random.default_rng(3)
    perm = rng.permutation(w.n).astype(np.int32)
    assert_same_symbolic(A.analyze(w.pat, perm=perm), O.analyze(w.pat, perm=perm))
    for df in (0.5, 2.0, 10.0):  # dense-row threshold max(16, df sqrt n)
        assert np.array_equal(A.amdOrder(w.pat, df), O.amd_order(w.pat, df))


def fnv1a_fingerprint(pat):
    """Independent restatement of patternFingerprint (sparse.mjs:908-925): FNV-1a over the little-endian bytes of
    rowptr then colidx, as "n:nnz:hex"."""
    h = 0x811C9DC5
    for arr in (pat.rowptr[: pat.n + 1], pat.colidx[: int(pat.rowptr[pat.n])]):
        for byte in np.ascontiguousarray(arr, "<i4").tobytes():
            h = ((h ^ byte) * 0x01000193) & 0xFFFFFFFF
    return f"{pat.n}:{int(pat.rowptr[pat.n])}:{h:x}"


def test_fingerprint_independent_restatement():
    for w in (W.hex_q1(3, 3, 2), W.poisson2d(6), W.chain(17)):
        assert A.patternFingerprint(w.pat) == fnv1a_fingerprint(w.pat) == O.fingerprint(w.pat)


def header_symbols():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"AMP_API\s+[\w\s\*]+?\b(amp_\w+)\s*\(", txt)))


def test_abi_exports_every_header_symbol():
    syms = header_symbols()
    assert len(syms) >= 20
    lib = C.CDLL(A._LIB_PATH)
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing


def test_abi_error_paths_without_gpu():
    w = W.hex_q1(4, 4, 3)
    with pytest.raises(A.AmpError, match="needs node coordinates"):
        A.analyze(w.pat, ordering="nd")
    with pytest.raises(A.AmpError, match="perm has length"):
        A.analyze(w.pat, perm=np.arange(w.n - 1))
    sym = A.analyze(w.pat)
    other = W.CsrPattern(w.pat.n, w.pat.rowptr.copy(), w.pat.colidx.copy())
    last = other.rowptr[1] - 1
    other.colidx[last] = (other.colidx[last] + 1) % other.n
    with pytest.raises(A.AmpError, match="different sparsity pattern"):
        A.checkSymbolic(sym, other)
    with pytest.raises(A.AmpError, match="different sparsity pattern"):
        A.SparseCholesky(other, sym=sym)
    A.checkSymbolic(sym, w.pat)
    # C ABI directly: invalid handles and arguments return codes and set the message
    raw = C.CDLL(A._LIB_PATH)  # untyped view: plain pointers and ints
    raw.amp_last_error.restype = C.c_char_p
    assert raw.amp_plan_get_info(None, None) == A.AMP_INVALID
    assert b"null" in raw.amp_last_error()
    h = C.c_void_p()
    assert raw.amp_analyze(-1, None, None, None, C.byref(h)) == A.AMP_INVALID
    assert raw.amp_plan_check_pattern(C.c_void_p(sym.handle), other.n, C.c_void_p(other.rowptr.ctypes.data),
                                      C.c_void_p(other.colidx.ctypes.data)) == A.AMP_PATTERN_MISMATCH
    assert b"different sparsity pattern" in raw.amp_last_error()


def test_empty_pattern_analyze():
    empty = W.CsrPattern(0, np.zeros(1, np.int32), np.zeros(0, np.int32))
    sym = A.analyze(empty)
    assert sym.n == 0 and sym.nsuper == 0 and sym.nnzL == 0
    assert sym.patternKey == O.fingerprint(empty)
