"""GPU LDL^T (FP64, static pivot perturbation) against the oracle's SupernodalLDLT (ldlt.mjs:450-643).

Tolerances. The update order differs from the reference's, and small indefinite pivots amplify rounding in their
columns, so two correct FP64 factorizations of an indefinite matrix agree only as far as its conditioning allows (on
the shifted elasticity case, min |d| = 1.3e-5 and max |L| = 1e4, a 1-ulp symmetric perturbation of A moves the
oracle's own L by 2e-8 and D by 9e-8 in relative Frobenius norm). The bar is therefore relative to that sensitivity:
L, D and the solutions within max(1e-11, 100 x the oracle's change under a 1-ulp perturbation of A), in relative
Frobenius / 2-norm: a different operation order (tiles, K = 256 groups, the pivot block's inverse in the TRSM)
accumulates many roundings, not one (on the shifted 27-point grid a dense numpy LDL^T differs from the oracle by
25 x the 1-ulp change in D). Refined residuals below 1e-12 are the strict check, independent of the order of
operations.
Inertia (nNeg) and the perturbation count are exact.
"""
import math

import numpy as np
import pytest

import ampsolve as A
import oracle as O
import workloads as W

pytestmark = pytest.mark.gpu

FLOOR = 1e-11
SENS = 100  # times the oracle's own change under a 1-ulp perturbation of A


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def ulp_perturbed(pat, values):
    """A (1 + e) with e = +-2^-53 chosen per unordered pair {i, j}, so the perturbed matrix stays symmetric."""
    rows = np.repeat(np.arange(pat.n, dtype=np.int64), np.diff(pat.rowptr))
    cols = pat.colidx.astype(np.int64)
    key = np.minimum(rows, cols) * pat.n + np.maximum(rows, cols)
    sign = np.where(((key * 2654435761) >> 7) & 1, 1.0, -1.0)
    return values * (1.0 + sign * 2.0 ** -53)


def diag_slots(pat):
    return np.array([pat.rowptr[i] + int(np.searchsorted(pat.colidx[pat.rowptr[i]:pat.rowptr[i + 1]], i))
                     for i in range(pat.n)])


def shifted(w, sigma):
    v = w.values.copy()
    v[diag_slots(w.pat)] -= sigma
    return v


def relres(pat, vals, x, b):
    return float(np.linalg.norm(O.matvec(pat, vals, x) - b) / np.linalg.norm(b))


def lower_parts(sym, Lx):
    out = []
    for s in range(sym.nsuper):
        nc = int(sym.superStart[s + 1] - sym.superStart[s])
        m = int(sym.Sp[s + 1] - sym.Sp[s])
        blk = np.asarray(Lx[sym.Lxp[s]:sym.Lxp[s] + m * nc]).reshape(nc, m)
        for c in range(nc):
            out.append(blk[c, c:])
    return np.concatenate(out) if out else np.zeros(0)


def run_case(w, values, sym_kw, nrhs=2):
    psym = A.analyze(w.pat, **sym_kw)
    osym = O.analyze(w.pat, perm=psym.perm)
    ok_o, Lx_o, D_o, nneg_o, npert_o = O.factor(osym, values, kind="ldlt")
    ok_p, Lx_p, D_p, _, _ = O.factor(osym, ulp_perturbed(w.pat, values), kind="ldlt")
    assert ok_o and ok_p
    Lo = lower_parts(osym, Lx_o)
    tol_L = max(FLOOR, SENS * rel(lower_parts(osym, Lx_p), Lo))
    tol_D = max(FLOOR, SENS * rel(D_p, D_o))
    f = A.SupernodalLDLT(psym)
    r = f.factor(values)
    assert r["ok"]
    assert (r["nNeg"], r["nPerturbed"]) == (nneg_o, npert_o)
    assert rel(lower_parts(osym, f.Lx), Lo) <= tol_L
    assert rel(f.D, D_o) <= tol_D
    rng = np.random.default_rng(7)
    B = rng.uniform(-1, 1, (nrhs, w.n))
    Xg = f.solveMany(B.reshape(-1), nrhs).reshape(nrhs, w.n)
    for k in range(nrhs):
        xo = O.solve_ldlt(osym, Lx_o, D_o, B[k])
        tol_x = max(FLOOR, SENS * rel(O.solve_ldlt(osym, Lx_p, D_p, B[k]), xo))
        assert rel(Xg[k], xo) <= tol_x
        assert rel(f.solve(B[k]), xo) <= tol_x  # the one-vector sweep, same bound
    ref = f.solveRefined(w.pat, values, B[0], maxSteps=5, tol=1e-14)
    assert ref["relResidual"] < 1e-12
    return r


CASES = [
    ("grid27-10-shift30", lambda: W.grid27(10, 10, 10, sym=True), 30.0, {}),
    ("grid27-9-zeros-shift30", lambda: W.grid27(9, 9, 9, zero_every=3, sym=True), 30.0, {}),
    ("hex884-nd-shift", lambda: W.hex_q1(8, 8, 4), None, {"ordering": "nd"}),
    ("elastic3d-14-shift", lambda: W.elastic3d(14), None, {"ordering": "nd3"}),
    ("maxwell3d-8-k2", lambda: W.maxwell3d(8, 2, 12.0, 40.0, 5, 1), 0.0, {"ordering": "nd3"}),
]


@pytest.mark.parametrize("name,make,sigma,kw", CASES, ids=[c[0] for c in CASES])
def test_ldlt_matches_oracle(name, make, sigma, kw):
    w = make()
    if sigma is None:  # a third of the median diagonal entry: indefinite
        sigma = 0.3 * float(np.median(w.values[diag_slots(w.pat)]))
    if kw.get("ordering") in ("nd", "nd3"):
        kw = dict(kw, x=w.x, y=w.y, z=w.z)
    r = run_case(w, shifted(w, sigma) if sigma else w.values, kw)
    assert r["nNeg"] > 0


def test_ldlt_inertia_sylvester():
    n = 300

    def lap1d(k):
        return 2 - 2 * math.cos(k * math.pi / (n + 1))

    sigma = 0.5 * (lap1d(10) + lap1d(11))
    w = W.chain(n, 2 - sigma, -1.0)
    f = A.SupernodalLDLT(A.analyze(w.pat))
    r = f.factor(w.values)
    assert r["ok"] and r["nNeg"] == 10


def test_ldlt_perturbation_and_refinement():
    from test_oracle_properties import two_by_two_system

    pat, vals, xr, br = two_by_two_system(40)
    ident = np.arange(pat.n, dtype=np.int32)
    f = A.SupernodalLDLT(A.analyze(pat, perm=ident))
    r = f.factor(vals)
    assert r["ok"] and r["nPerturbed"] > 0
    ok_o, _, _, nneg_o, npert_o = O.factor(O.analyze(pat, perm=ident), vals, kind="ldlt")
    assert ok_o and (r["nNeg"], r["nPerturbed"]) == (nneg_o, npert_o)
    res = f.solveRefined(pat, vals, br, maxSteps=30)
    assert np.max(np.abs(res["x"] - xr)) / np.max(np.abs(xr)) < 1e-10


def test_ldlt_nonfinite_pivot_fails_and_solve_raises():
    w = W.grid27(8, 8, 8, sym=True)
    sym = A.analyze(w.pat)
    last = int(sym.perm[w.n - 1])
    v = shifted(w, 30.0)
    v[diag_slots(w.pat)[last]] = float("nan")
    f = A.SupernodalLDLT(sym)
    assert not f.factor(v)["ok"]
    with pytest.raises(A.AmpError, match="no successful numeric factorization"):
        f.solve(np.ones(w.n))
    assert f.factor(shifted(w, 30.0))["ok"]  # the same object factors again


# ---- mixed precision (FP32 fronts, BF16x3 tensor-core updates) + FP64 GMRES-IR (gmres-real.mjs:31-105) ----------
MIXED_CASES = [
    ("grid27-10-shift30", lambda: W.grid27(10, 10, 10, sym=True), 30.0, {}),
    ("maxwell3d-8-k2", lambda: W.maxwell3d(8, 2, 12.0, 40.0, 5, 1), 0.0, {"ordering": "nd3"}),
    ("elastic3d-12-shift", lambda: W.elastic3d(12), None, {"ordering": "nd3"}),
]


@pytest.mark.parametrize("name,make,sigma,kw", MIXED_CASES, ids=[c[0] for c in MIXED_CASES])
def test_mixed_ldlt_gmres_ir(name, make, sigma, kw):
    w = make()
    if sigma is None:
        sigma = 0.05 * float(np.median(w.values[diag_slots(w.pat)]))
    if kw.get("ordering") == "nd3":
        kw = dict(kw, x=w.x, y=w.y, z=w.z)
    vals = shifted(w, sigma) if sigma else w.values
    sym = A.analyze(w.pat, **kw)
    f64 = A.SupernodalLDLT(sym)
    r64 = f64.factor(vals)
    fmx = A.SupernodalLDLT(sym, precision=A.MIXED)
    rmx = fmx.factor(vals)
    assert r64["ok"] and rmx["ok"] and rmx["nNeg"] > 0
    b = np.random.default_rng(3).uniform(-1, 1, w.n)
    out = fmx.solveGmres(b, tol=1e-13, restart=40, maxIter=200)
    assert out["converged"] and out["relres"] < 1e-12
    x64 = f64.solveRefined(w.pat, vals, b, maxSteps=5, tol=1e-15)["x"]
    assert np.linalg.norm(out["x"] - x64) / np.linalg.norm(x64) < 1e-9
    assert relres(w.pat, vals, out["x"], b) < 1e-12


def test_gmres_with_fp64_cholesky_converges_at_once():
    w = W.elastic3d(8)
    sym = A.analyze(w.pat, ordering="nd3", x=w.x, y=w.y, z=w.z)
    num = A.NumericFactor(sym)
    assert num.factor(w.values)
    out = num.solve_gmres(w.rhs[0], tol=1e-13)
    assert out["converged"] and out["iterations"] <= 2 and out["relres"] < 1e-13
