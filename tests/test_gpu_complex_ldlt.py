"""GPU complex-symmetric LDL^T (ComplexSupernodalLDLT, ldlt.mjs:648-900) against the oracle's restatement of it.

The systems are complex-symmetric (A = A^T, no conjugation): lossy Maxwell pencils K - k^2 (eps' + i eps'') M on
Nedelec edges (the reference's driven Helmholtz and lossy-mode use), indefinite in their real part, and a shifted
27-point grid with a complex diagonal. The perturbation count must be exact; L, D and the solution agree with the
oracle to a bound relative to the oracle's own sensitivity (its change under a 1-ulp perturbation of the values,
times 100, floor 1e-11: the update order differs, as for the real LDL^T), and the refined residual reaches 1e-12.
"""
import numpy as np
import pytest
import scipy.sparse as sp

import ampsolve as A
import oracle as O
import workloads as W

pytestmark = pytest.mark.gpu

FLOOR, SENS = 1e-11, 100


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def lower(so, L):
    out = []
    for s in range(so.nsuper):
        nc, m = int(so.superStart[s + 1] - so.superStart[s]), int(so.Sp[s + 1] - so.Sp[s])
        blk = L[so.Lxp[s]: so.Lxp[s] + m * nc].reshape(nc, m)
        out += [blk[c, c + 1:] for c in range(nc)]
    return np.concatenate(out) if out else np.zeros(0)


def ulp(pat, v, sign_seed):
    rows = np.repeat(np.arange(pat.n, dtype=np.int64), np.diff(pat.rowptr))
    cols = pat.colidx.astype(np.int64)
    key = np.minimum(rows, cols) * pat.n + np.maximum(rows, cols) + sign_seed
    return v * (1.0 + np.where(((key * 2654435761) >> 7) & 1, 1.0, -1.0) * 2.0 ** -53)


def maxwell_lossy(N, k2, loss):
    w0 = W.maxwell3d(N, 2, 12.0, 0.0, 5, 1)
    w1 = W.maxwell3d(N, 2, 12.0, 1.0, 5, 1)
    K, M = w0.values, w0.values - w1.values
    return w0, K - k2 * M, -k2 * loss * M


def grid_complex(N):
    w = W.grid27(N, N, N, sym=True)
    im = np.zeros_like(w.values)
    for i in range(w.n):
        for p in range(w.pat.rowptr[i], w.pat.rowptr[i + 1]):
            if w.pat.colidx[p] == i:
                im[p] = 0.5 + 0.01 * (i % 5)
    diag = np.array([w.pat.colidx[p] == i for i in range(w.n) for p in range(w.pat.rowptr[i], w.pat.rowptr[i + 1])])
    re = w.values - 30.0 * diag
    return w, re, im


CASES = [
    ("maxwell6-lossy", lambda: maxwell_lossy(6, 30.0, 0.05), "nd3"),
    ("maxwell10-lossy", lambda: maxwell_lossy(10, 35.0, 0.02), "nd3"),
    ("grid27-9-complex-diag", lambda: grid_complex(9), "amd"),
]


@pytest.mark.parametrize("name,make,ordering", CASES, ids=[c[0] for c in CASES])
def test_complex_ldlt_matches_oracle(name, make, ordering):
    w, re, im = make()
    sym = A.analyze(w.pat, ordering="nd3", x=w.x, y=w.y, z=w.z) if ordering == "nd3" else A.analyze(w.pat)
    so = O.analyze(w.pat, perm=sym.perm)
    ok, Lr, Li, Dr, Di, npert = O.cfactor(so, re, im)
    okp, Lr2, Li2, Dr2, Di2, _ = O.cfactor(so, ulp(w.pat, re, 0), ulp(w.pat, im, 7))
    assert ok and okp
    f = A.ComplexSupernodalLDLT(sym)
    r = f.factor(re, im)
    assert r["ok"] and r["nPerturbed"] == npert
    gLr, gLi, gDr, gDi = f.factors()
    Lo, Lp, Lg = lower(so, Lr + 1j * Li), lower(so, Lr2 + 1j * Li2), lower(so, gLr + 1j * gLi)
    assert rel(Lg, Lo) <= max(FLOOR, SENS * rel(Lp, Lo))
    Do, Dp, Dg = Dr + 1j * Di, Dr2 + 1j * Di2, gDr + 1j * gDi
    assert rel(Dg, Do) <= max(FLOOR, SENS * rel(Dp, Do))
    rng = np.random.default_rng(9)
    br, bi = rng.uniform(-1, 1, w.n), rng.uniform(-1, 1, w.n)
    xo = np.array(O.csolve(so, Lr, Li, Dr, Di, br, bi))
    xp = np.array(O.csolve(so, Lr2, Li2, Dr2, Di2, br, bi))
    x = f.solve(br, bi)
    xg = np.array([x["re"], x["im"]])
    assert rel(xg, xo) <= max(FLOOR, SENS * rel(xp, xo))
    out = f.solveRefined(w.pat, re, im, br, bi, maxSteps=5, tol=1e-14)
    assert out["relResidual"] <= 1e-12
    Ac = sp.csr_matrix((re + 1j * im, w.pat.colidx, w.pat.rowptr), shape=(w.n, w.n))
    xs = out["re"] + 1j * out["im"]
    assert np.linalg.norm(Ac @ xs - (br + 1j * bi)) / np.linalg.norm(br + 1j * bi) <= 1e-12


def test_complex_ldlt_perturbation_failure_and_kind_checks():
    n = 6
    rp = np.arange(0, n * n + 1, n, dtype=np.int32)
    ci = np.tile(np.arange(n, dtype=np.int32), n)
    pat = W.CsrPattern(n, rp, ci)
    Ar = np.eye(n) * 2.0 + 0.1
    Ai = np.eye(n) * 0.5
    Ar[0, 0], Ai[0, 0] = 0.0, 0.0  # the first pivot is zero: perturbed to tau (the oracle agrees)
    sym = A.analyze(pat, perm=np.arange(n, dtype=np.int32))
    f = A.ComplexSupernodalLDLT(sym)
    r = f.factor(Ar.reshape(-1), Ai.reshape(-1))
    so = O.analyze(pat, perm=np.arange(n, dtype=np.int32))
    ok, *_, npert = O.cfactor(so, Ar.reshape(-1), Ai.reshape(-1))
    assert r["ok"] and ok and r["nPerturbed"] == npert == 1
    Ar[3, 3] = np.nan
    assert not f.factor(Ar.reshape(-1), Ai.reshape(-1))["ok"]
    with pytest.raises(A.AmpError, match="no successful numeric factorization"):
        f.solve(np.ones(n), np.zeros(n))
    # a complex factor is not a real one: the real-valued entry points reject it
    assert A.lib().amp_solve(f._h, None, 1, None, 0) == A.AMP_INVALID
