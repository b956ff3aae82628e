"""GPU LDL^T with Bunch-Kaufman pivots inside each 64-column pivot block (SupernodalLDLT(pivoting="bunch-kaufman")).

The reference has static perturbation only (ldlt.mjs:513-522), so there is no reference output to match pivot for
pivot; the checks are the factorization's defining properties, on matrices small enough for dense numpy:
  - reconstruction: with each block's interchanges applied to the columns left of it (the factor keeps them in the
    original order), Q P A P^T Q^T = L D L^T to round-off (D block diagonal with 1 x 1 and 2 x 2 pivots);
  - inertia: nNeg equals the number of negative eigenvalues of A (numpy's eigvalsh; a KKT matrix's is its constraint
    count), since no pivot is perturbed on these matrices;
  - solves: one and several right-hand sides against numpy's dense solve within a condition-scaled bound, refined
    residuals below 1e-12;
  - KKT systems (zero diagonals): the static rule perturbs every zero pivot, the Bunch-Kaufman factor interchanges
    those that have a usable pivot inside their block and perturbs fewer; GMRES on either reaches 1e-12.
"""
import numpy as np
import pytest

import ampsolve as A
import workloads as W

pytestmark = pytest.mark.gpu


def csr_from_dense(Ad):
    """Full symmetric CSR of a dense symmetric matrix (its nonzeros and the whole diagonal)."""
    n = Ad.shape[0]
    mask = (Ad != 0) | np.eye(n, dtype=bool)
    rp = np.zeros(n + 1, np.int32)
    rp[1:] = np.cumsum(mask.sum(axis=1))
    ci = np.nonzero(mask)[1].astype(np.int32)
    return W.CsrPattern(n, rp, ci), Ad[mask].astype(np.float64)


def dense_of(pat, values):
    Ad = np.zeros((pat.n, pat.n))
    rows = np.repeat(np.arange(pat.n), np.diff(pat.rowptr))
    Ad[rows, pat.colidx] = values
    return Ad


def kkt(nx, ny, ncons, seed, natural_first=False):
    """[[H, B^T], [B, 0]]: H the 5-point Laplacian of an nx x ny grid, B ncons rows coupling 3 random nodes each
    (full row rank with probability one); inertia (nx ny, ncons, 0). natural_first puts the constraints first."""
    rng = np.random.default_rng(seed)
    n1 = nx * ny
    H = np.zeros((n1, n1))
    for i in range(nx):
        for j in range(ny):
            k = i * ny + j
            H[k, k] = 4.0
            for di, dj in ((1, 0), (0, 1)):
                if i + di < nx and j + dj < ny:
                    kk = (i + di) * ny + j + dj
                    H[k, kk] = H[kk, k] = -1.0
    B = np.zeros((ncons, n1))
    for r in range(ncons):
        B[r, rng.choice(n1, 3, replace=False)] = rng.uniform(0.5, 1.5, 3)
    K = np.block([[H, B.T], [B, np.zeros((ncons, ncons))]])
    if natural_first:
        p = np.r_[np.arange(n1, n1 + ncons), np.arange(n1)]
        K = K[np.ix_(p, p)]
    return K


def bk_parts(sym, f):
    """(L, D, Q) in the standard form: Q P A P^T Q^T = L D L^T, Q the blocks' pivot orders (new -> original position)."""
    n = sym.n
    Lx, Dd = f.Lx, f.D
    doff, piv = f.num.pivots()
    ss, Sp, Si, Lxp = (np.asarray(getattr(sym, k)) for k in ("superStart", "Sp", "Si", "Lxp"))
    Q = np.arange(n)
    for s in range(sym.nsuper):
        f0, nc = int(ss[s]), int(ss[s + 1] - ss[s])
        for c0 in range(0, nc, 64):
            w = min(64, nc - c0)
            assert sorted(piv[f0 + c0:f0 + c0 + w]) == list(range(w))  # a permutation of the block's columns
            Q[f0 + c0:f0 + c0 + w] = f0 + c0 + piv[f0 + c0:f0 + c0 + w]
    Qinv = np.empty(n, np.int64)
    Qinv[Q] = np.arange(n)
    L = np.zeros((n, n))
    for s in range(sym.nsuper):
        f0, nc, m = int(ss[s]), int(ss[s + 1] - ss[s]), int(Sp[s + 1] - Sp[s])
        blk = np.asarray(Lx[Lxp[s]:Lxp[s] + m * nc]).reshape(nc, m).T.copy()
        for c0 in range(64, nc, 64):  # apply each block's interchanges to the columns left of it
            w = min(64, nc - c0)
            blk[c0:c0 + w, :c0] = blk[c0 + piv[f0 + c0:f0 + c0 + w], :c0]
        rows = np.asarray(Si[Sp[s]:Sp[s] + m])
        grow = np.concatenate([f0 + np.arange(nc), Qinv[rows[nc:]]])
        for j in range(nc):
            L[grow[j:], f0 + j] = blk[j:, j]
    D = np.diag(Dd) + np.diag(doff[:-1], -1) + np.diag(doff[:-1], 1)
    return L, D, Q, doff


def check_bk(pat, values, sym_kw, nrhs=3, expect_neg=None):
    psym = A.analyze(pat, **sym_kw)
    f = A.SupernodalLDLT(psym, pivoting="bunch-kaufman")
    r = f.factor(values)
    assert r["ok"]
    assert r["nPerturbed"] == 0
    Ad = dense_of(pat, values)
    ev = np.linalg.eigvalsh(Ad)
    assert r["nNeg"] == int((ev < 0).sum())
    if expect_neg is not None:
        assert r["nNeg"] == expect_neg
    L, D, Q, doff = bk_parts(psym, f)
    perm = np.asarray(psym.perm)
    Aq = Ad[np.ix_(perm, perm)][np.ix_(Q, Q)]
    assert np.allclose(np.diag(L), 1.0)
    aL, aD = np.abs(L), np.abs(D)
    err = np.linalg.norm(Aq - L @ D @ L.T) / max(np.linalg.norm(Ad), np.linalg.norm(aL @ aD @ aL.T))
    assert err < 1e-13, err  # the backward error of an LDL^T, u || |L| |D| |L^T| || up to a small factor
    # solves: one vector, several (the multi-vector sweeps), refined
    cond = np.linalg.cond(Ad)
    rng = np.random.default_rng(11)
    B = rng.uniform(-1, 1, (nrhs, pat.n))
    Xd = np.linalg.solve(Ad, B.T).T
    tol = max(1e-12, 1e-15 * cond)
    x1 = f.solve(B[0])
    assert np.linalg.norm(x1 - Xd[0]) / np.linalg.norm(Xd[0]) < tol
    Xm = f.solveMany(B.reshape(-1), nrhs).reshape(nrhs, pat.n)
    assert np.linalg.norm(Xm - Xd) / np.linalg.norm(Xd) < tol
    ref = f.solveRefined(pat, values, B[0], maxSteps=5, tol=1e-14)
    assert ref["relResidual"] < 1e-12
    return r, doff


def kkt_case(natural_first):
    K = kkt(16, 16, 60, seed=1) if not natural_first else kkt(12, 12, 40, seed=2, natural_first=True)
    pat, vals = csr_from_dense(K)
    kw = {"perm": np.arange(pat.n, dtype=np.int32)} if natural_first else {}
    return pat, vals, kw, (60 if not natural_first else 40)


@pytest.mark.parametrize("natural_first", [False, True])
def test_bk_kkt_fewer_perturbed_pivots(natural_first):
    """KKT systems, whose constraint rows have zero diagonals. The reference's static rule perturbs every zero pivot;
    the Bunch-Kaufman factor interchanges a zero pivot with a usable one inside its pivot block and perturbs only those
    whose column has no entry inside the block (their partners lie outside the supernode, and taking them would change
    the symbolic structure). Both solve the system to 1e-12 with FP64 GMRES on the factor."""
    pat, vals, kw, ncons = kkt_case(natural_first)
    sym = A.analyze(pat, **kw)
    st = A.SupernodalLDLT(sym)
    rs = st.factor(vals)
    bk = A.SupernodalLDLT(sym, pivoting="bunch-kaufman")
    rb = bk.factor(vals)
    assert rs["ok"] and rb["ok"]
    assert rs["nPerturbed"] == ncons  # every constraint pivot is an exact zero for the static rule
    if natural_first:  # constraint columns first: a zero pivot has no partner inside its own supernode
        assert rb["nPerturbed"] <= rs["nPerturbed"]
    else:  # AMD order: most zero pivots meet a larger pivot inside their block and are interchanged with it
        assert rb["nPerturbed"] < rs["nPerturbed"] // 2
    b = np.random.default_rng(4).uniform(-1, 1, pat.n)
    xd = np.linalg.solve(dense_of(pat, vals), b)
    for f in (st, bk):
        g = f.solveGmres(b, tol=1e-13, restart=40, maxIter=200)
        assert g["converged"] and g["relres"] < 1e-12
        assert np.linalg.norm(g["x"] - xd) / np.linalg.norm(xd) < 1e-10


def test_bk_dense_multiblock():
    """One dense indefinite supernode of 300 columns (five pivot blocks): interchanges inside each block, the TRSM
    of later blocks' rows in the pivot order, the inverse blocks with the pivot order folded in."""
    rng = np.random.default_rng(5)
    n = 300
    M = rng.standard_normal((n, n))
    Ad = (M + M.T) / 2
    Ad[np.arange(0, n, 7), np.arange(0, n, 7)] = 0.0  # some zero diagonal entries
    Ad[np.abs(Ad) < 0.3] = 0.0
    Ad[np.arange(0, n, 7), np.arange(0, n, 7)] = 0.0
    pat, vals = csr_from_dense(Ad)
    r, doff = check_bk(pat, vals, {"perm": np.arange(n, dtype=np.int32)}, nrhs=20)
    assert np.count_nonzero(doff) > 0


@pytest.mark.parametrize("shift", [30.0, 55.0])
def test_bk_shifted_grid27(shift):
    """A 27-point 10^3 grid shifted into its spectrum (AMD): many supernodes, rows below, a multi-block root."""
    w = W.grid27(10, 10, 10, sym=True)
    v = w.values.copy()
    slots = np.array([w.pat.rowptr[i] + int(np.searchsorted(w.pat.colidx[w.pat.rowptr[i]:w.pat.rowptr[i + 1]], i))
                      for i in range(w.n)])
    v[slots] -= shift
    check_bk(w.pat, v, {}, nrhs=40)


def test_bk_maxwell():
    """Nedelec curl-curl - k^2 eps_r mass on an 8^3 cube at k^2 = 30 (indefinite, 348 negative eigenvalues; nested
    dissection on edge midpoints)."""
    w0 = W.maxwell3d(8, 2, 12.0, 0.0, 5, 1)
    w1 = W.maxwell3d(8, 2, 12.0, 1.0, 5, 1)
    v = w0.values - 30.0 * (w0.values - w1.values)
    r, _ = check_bk(w0.pat, v, {"ordering": "nd3", "x": w0.x, "y": w0.y, "z": w0.z}, nrhs=4, expect_neg=348)


def test_bk_gmres_and_reuse():
    """GMRES with the FP64 Bunch-Kaufman factor as preconditioner converges at once; a second factorization of new
    values on the same object (the captured graph replayed) matches a fresh factor of those values."""
    w = W.grid27(10, 10, 10, sym=True)
    slots = np.array([w.pat.rowptr[i] + int(np.searchsorted(w.pat.colidx[w.pat.rowptr[i]:w.pat.rowptr[i + 1]], i))
                      for i in range(w.n)])
    vals = w.values.copy()
    vals[slots] -= 30.0
    psym = A.analyze(w.pat)
    f = A.SupernodalLDLT(psym, pivoting="bunch-kaufman")
    assert f.factor(vals)["ok"]
    b = np.random.default_rng(4).uniform(-1, 1, w.n)
    g = f.solveGmres(b, tol=1e-13)
    assert g["converged"] and g["iterations"] <= 3
    vals2 = vals.copy()
    vals2[slots] -= 7.0  # another shift on the same pattern
    r2 = f.factor(vals2)
    assert r2["ok"]
    fresh = A.SupernodalLDLT(psym, pivoting="bunch-kaufman")
    rf = fresh.factor(vals2)
    assert rf["ok"] and (rf["nNeg"], rf["nPerturbed"]) == (r2["nNeg"], r2["nPerturbed"])
    x1, x2 = f.solve(b), fresh.solve(b)
    assert np.array_equal(x1, x2)  # the same arithmetic on the same values


def test_bk_rejects_mixed_and_bad_option():
    w = W.chain(10)
    sym = A.analyze(w.pat)
    with pytest.raises(A.AmpError):
        A.SupernodalLDLT(sym, pivoting="rook")
    with pytest.raises(A.AmpError):
        A.SupernodalLDLT(sym, precision=A.MIXED, pivoting="bunch-kaufman")
