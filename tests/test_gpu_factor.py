"""GPU parity: the sm_100a FP64 factor and solves against the oracle (CPU restatement of the reference)."""
import numpy as np
import pytest

import ampsolve as amp
import oracle as orc
import workloads as wl

pytestmark = pytest.mark.gpu

# FP64 parity bar: relative error of the solution vs the oracle's FP64 solution
TOL = 1e-12


def rel(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


CASES = [
    ("hex654", lambda: wl.hex_q1(6, 5, 4), {}),
    ("hex884-nd", lambda: wl.hex_q1(8, 8, 4), {"ordering": "nd"}),
    ("poisson2d-64", lambda: wl.poisson2d(64), {}),
    ("grid27-11", lambda: wl.grid27(11, 11, 11, sym=True), {}),
    ("grid27-10-zeros", lambda: wl.grid27(10, 10, 10, zero_every=3, sym=True), {}),
    ("elastic3d-8", lambda: wl.elastic3d(8), {"ordering": "nd3"}),
    ("elastic3d-14", lambda: wl.elastic3d(14), {"ordering": "nd3"}),
    ("elastic3d-16-multichunk", lambda: wl.elastic3d(16), {"ordering": "nd3"}),
    ("chain-300", lambda: wl.chain(300), {}),
]


@pytest.mark.parametrize("name,make,opts", CASES, ids=[c[0] for c in CASES])
def test_factor_solve_matches_oracle(name, make, opts):
    w = make()
    o = dict(opts)
    if o.get("ordering") in ("nd", "nd3"):
        o.update(x=w.x, y=w.y, z=w.z)
    sym = amp.analyze(w.pat, o)
    so = orc.analyze(w.pat, perm=sym.perm)
    num = amp.factorNumeric(sym, w.values)
    assert num.ok
    ok, Lx, _, _, _ = orc.factor(so, w.values)
    assert ok
    rng = np.random.default_rng(5)
    b = rng.uniform(-1, 1, w.n)
    x = amp.solveNumeric(num, b)
    xo = orc.solve_chol(so, Lx, b)
    assert rel(x, xo) <= TOL, rel(x, xo)
    # the factor itself (lower parts of the stored blocks)
    Lg = num.Lx
    ss, Sp, Lxp = so.superStart, so.Sp, so.Lxp
    worst = 0.0
    for s in range(so.nsuper):
        nc, m, lo = ss[s + 1] - ss[s], Sp[s + 1] - Sp[s], Lxp[s]
        A = Lg[lo: lo + m * nc].reshape(nc, m).T
        B = Lx[lo: lo + m * nc].reshape(nc, m).T
        mask = np.tril(np.ones((m, nc), bool))
        d = np.max(np.abs(A[mask] - B[mask])) if mask.any() else 0.0
        worst = max(worst, d / max(np.max(np.abs(B[mask])), 1e-300))
    assert worst <= 1e-11, worst
    # residual
    r = orc.matvec(w.pat, w.values, x) - b
    assert np.linalg.norm(r) / np.linalg.norm(b) < 1e-12


def test_multi_rhs_and_refined():
    w = wl.elastic3d(10, q=5)
    sym = amp.analyze(w.pat, ordering="nd3", x=w.x, y=w.y, z=w.z)
    num = amp.factorNumeric(sym, w.values)
    assert num.ok
    xs = amp.solveNumericMulti(num, list(w.rhs))
    so = orc.analyze(w.pat, perm=sym.perm)
    ok, Lx, _, _, _ = orc.factor(so, w.values)
    for k in range(5):
        xo = orc.solve_chol(so, Lx, w.rhs[k])
        assert rel(xs[k], xo) <= TOL
    X, relres, steps = num.solve_refined_block(w.rhs, maxSteps=3, tol=1e-14)
    assert relres < 1e-13


def test_not_positive_definite_and_errors():
    w = wl.hex_q1(4, 4, 3)
    v = w.values.copy()
    rp, ci = w.pat.rowptr, w.pat.colidx
    for i in range(w.n):
        for p in range(rp[i], rp[i + 1]):
            if ci[p] == i:
                v[p] -= 1e3
    ch = amp.SparseCholesky(w.pat)
    assert ch.factor(v) is False
    with pytest.raises(amp.AmpError, match="without a successful factorization"):
        ch.solve(np.zeros(w.n))
    num = amp.factorNumeric(amp.analyze(w.pat), -w.values)
    assert num.ok is False
    with pytest.raises(amp.AmpError, match="no successful numeric factorization"):
        amp.solveNumeric(num, np.zeros(w.n))
    with pytest.raises(amp.AmpError, match="no successful numeric factorization"):
        amp.solveNumericMulti(num, [np.zeros(w.n), np.zeros(w.n)])


def test_symbolic_reuse_scaled_values():
    w = wl.hex_q1(6, 5, 4)
    b = np.sin(0.7 * np.arange(w.n)) + 0.3
    sn = amp.SparseCholesky(w.pat)
    assert sn.factor(w.values)
    xs = sn.solve(b)
    sn2 = amp.SparseCholesky(w.pat, sym=sn.sym)
    assert sn2.timing["symbolicReused"] is True
    assert sn2.factor(2 * w.values)
    x2 = sn2.solve(b)
    assert np.max(np.abs(2 * x2 - xs)) <= 1e-12 * np.max(np.abs(xs))


def test_empty_pattern():
    pat = wl.CsrPattern(0, np.zeros(1, np.int32), np.zeros(0, np.int32))
    ch = amp.SparseCholesky(pat)
    assert ch.factor(np.zeros(0))
    assert ch.solve(np.zeros(0)).shape == (0,)
