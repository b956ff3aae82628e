"""CPU tests of the oracle against the reference's own property tests (no GPU).

The reference pins its solver with properties, not stored vectors; each test below restates one of them for the C
oracle (oracle/amp_oracle.c), on the same fixtures:
  la-sparse.test.mjs:67-161      patterns, orderings, column counts vs up-looking, solve vs up-looking, errors
  sparse-fem.test.mjs:47-57      AMD gives less fill than ND on a 2D triangle mesh
  la-real-front.test.mjs:52-90   WASM (SIMD) factor == JS factor bitwise, Cholesky and LDL^T
  la-real-solve.test.mjs:48-104  WASM solve == JS solve bitwise, special RHS entries, q = 1, 2, 3, 4, 11
  la-ldlt.test.mjs:59-68         static pivot perturbation counted, refinement recovers the solution to 1e-10
  core-solvers.test.mjs:86-100   LDL^T inertia: nNeg = 10 on a shifted 1D Laplacian (Sylvester)
  core-solvers.test.mjs:162-171  nd3Order gives less fill than the natural order
"""
import math

import numpy as np
import pytest

import oracle as O
import workloads as W


def is_perm(p, n):
    p = np.asarray(p)
    return p.shape[0] == n and (n == 0 or (np.array_equal(np.sort(p), np.arange(n))))


def entry(pat, i, j):
    lo, hi = pat.rowptr[i], pat.rowptr[i + 1]
    k = np.searchsorted(pat.colidx[lo:hi], j)
    return lo + k if k < hi - lo and pat.colidx[lo + k] == j else -1


def relres(pat, values, x, b):
    r = O.matvec(pat, values, x) - b
    return float(np.linalg.norm(r) / np.linalg.norm(b))


@pytest.mark.parametrize("make", [lambda: W.hex_q1(3, 3, 2), lambda: W.poisson2d(12), lambda: W.grid27(5, 4, 3, sym=True),
                                  lambda: W.elastic3d(3), lambda: W.heat3d_p2(2, 2, 0.3, 4, 1),
                                  lambda: W.maxwell3d(3, 2, 12.0, 0.0, 5, 1)])
def test_patterns_sorted_symmetric_with_diagonal(make):
    w = make()
    pat = w.pat
    for i in range(pat.n):
        row = pat.colidx[pat.rowptr[i]:pat.rowptr[i + 1]]
        assert np.all(np.diff(row) > 0)
        assert entry(pat, i, i) >= 0
        for p in range(pat.rowptr[i], pat.rowptr[i + 1]):
            q = entry(pat, int(pat.colidx[p]), i)
            assert q >= 0
            assert w.values[q] == w.values[p]  # symmetric values


def test_orderings_are_permutations_and_analyses_consistent():
    w = W.hex_q1(8, 8, 4)
    n = w.n
    perm = O.amd_order(w.pat)
    assert is_perm(perm, n)
    amd = O.analyze(w.pat, perm=perm)
    nd = O.analyze(w.pat, perm=O.nd_order(w.pat, w.x, w.y))
    assert amd.nnzL >= amd.nnzA and nd.nnzL >= nd.nnzA
    assert amd.fill > 1 and math.isfinite(amd.flops)
    assert is_perm(O.nd3_order(w.pat, w.x, w.y, w.z, 16), n)


@pytest.mark.parametrize("relax", [False, True])
@pytest.mark.parametrize("make,ordering", [(lambda: W.hex_q1(5, 4, 3), "amd"), (lambda: W.poisson2d(10), "nd"),
                                           (lambda: W.elastic3d(4), "nd3")])
def test_colcount_equals_uplooking_structure(make, ordering, relax):
    w = make()
    if ordering == "nd3":
        sym = O.analyze(w.pat, perm=O.nd3_order(w.pat, w.x, w.y, w.z, 40), relax=relax)
    else:
        sym = O.analyze(w.pat, ordering=ordering, x=w.x, y=w.y, relax=relax)
    up = O.UpLookingCholesky(w.pat, sym.perm)
    assert sym.nnzL == up.nnzL
    assert np.array_equal(sym.colCount, np.diff(up.Lp))
    assert is_perm(sym.perm, sym.n)
    for s in range(sym.nsuper):
        f, nc = sym.superStart[s], sym.superStart[s + 1] - sym.superStart[s]
        rows = sym.Si[sym.Sp[s]:sym.Sp[s + 1]]
        assert np.array_equal(rows[:nc], np.arange(f, f + nc))
        assert np.all(np.diff(rows) > 0)
    if not relax:
        nc = np.diff(sym.superStart).astype(np.int64)
        assert sym.nnzLStored - int(np.sum(nc * (nc - 1) // 2)) == sym.nnzL
    assert sym.flops == float(np.sum(sym.colCount.astype(np.float64) ** 2))


def test_supernodal_solve_matches_uplooking_and_reuses_symbolic():
    w = W.hex_q1()
    n = w.n
    b = np.sin(0.7 * np.arange(n)) + 0.3
    sym = O.analyze(w.pat)
    ok, Lx, _, _, _ = O.factor(sym, w.values)
    assert ok
    up = O.UpLookingCholesky(w.pat, sym.perm)
    assert up.factor(w.values)
    xs, xu = O.solve_chol(sym, Lx, b), up.solve(b)
    assert np.max(np.abs(xs - xu)) / np.max(np.abs(xu)) < 1e-12
    assert relres(w.pat, w.values, xs, b) < 1e-12
    ok2, Lx2, _, _, _ = O.factor(sym, 2 * w.values)  # same symbolic analysis, new values
    assert ok2
    x2 = O.solve_chol(sym, Lx2, b)
    assert np.all(np.abs(2 * x2 - xs) <= 1e-12 * np.max(np.abs(xu)))


def test_indefinite_matrix_is_reported():
    w = W.hex_q1(4, 4, 3)
    v = w.values.copy()
    for i in range(w.n):
        v[entry(w.pat, i, i)] -= 1e3
    ok, *_ = O.factor(O.analyze(w.pat), v)
    assert not ok
    ok, *_ = O.factor(O.analyze(w.pat), -w.values)
    assert not ok


def test_fingerprint_detects_a_changed_pattern():
    w = W.hex_q1(4, 4, 3)
    other = W.CsrPattern(w.pat.n, w.pat.rowptr.copy(), w.pat.colidx.copy())
    last = other.rowptr[1] - 1
    other.colidx[last] = (other.colidx[last] + 1) % other.n
    assert O.fingerprint(w.pat) != O.fingerprint(other)
    assert O.fingerprint(w.pat) == O.analyze(w.pat).patternKey


def test_empty_pattern_and_nd_without_coordinates():
    empty = W.CsrPattern(0, np.zeros(1, np.int32), np.zeros(0, np.int32))
    sym = O.analyze(empty)
    assert sym.n == 0 and sym.nsuper == 0 and sym.nnzL == 0
    ok, Lx, *_ = O.factor(sym, np.zeros(0))
    assert ok
    assert O.solve_chol(sym, Lx, np.zeros(0)).shape == (0,)
    w = W.hex_q1(4, 4, 3)
    with pytest.raises(ValueError, match="needs node coordinates"):
        O.analyze(w.pat, ordering="nd")


def test_amd_beats_nd_on_fill_in_2d():
    w = W.poisson2d(24)
    amd = O.analyze(w.pat)
    nd = O.analyze(w.pat, ordering="nd", x=w.x, y=w.y)
    assert amd.nnzL <= nd.nnzL


def test_nd3_less_fill_than_natural():
    m = 12
    w = W.grid27(m, m, m)
    q = np.arange(w.n)
    x, y, z = (q % m).astype(float), (q // m % m).astype(float), (q // (m * m)).astype(float)
    perm = O.nd3_order(w.pat, x, y, z, 64)
    assert is_perm(perm, w.n)
    nat = O.analyze(w.pat, perm=np.arange(w.n, dtype=np.int32))
    nd3 = O.analyze(w.pat, perm=perm)
    assert nd3.nnzL < nat.nnzL


def same_lower(sym, La, Lb):
    """Lower parts (rows >= c) of every stored supernode block are equal bit for bit."""
    for s in range(sym.nsuper):
        nc = sym.superStart[s + 1] - sym.superStart[s]
        m = sym.Sp[s + 1] - sym.Sp[s]
        lo = sym.Lxp[s]
        blk_a = La[lo:lo + m * nc].reshape(nc, m)
        blk_b = Lb[lo:lo + m * nc].reshape(nc, m)
        for c in range(nc):
            if blk_a[c, c:].tobytes() != blk_b[c, c:].tobytes():
                return False
    return True


def bitwise(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return a.shape == b.shape and a.tobytes() == b.tobytes()


FRONT_CASES = [("cube 11^3", (11, 11, 11), 0), ("slab 23x9x5", (23, 9, 5), 0), ("cube 10^3 zeros", (10, 10, 10), 3)]


@pytest.mark.parametrize("name,dims,zero_every", FRONT_CASES)
def test_simd_factor_equals_scalar_bitwise_cholesky(name, dims, zero_every):
    w = W.grid27(*dims, zero_every=zero_every)
    sym = O.analyze(w.pat)
    assert sym.maxFront >= 32  # the SIMD front kernel engages (WASM_MIN_FRONT)
    ok_s, L_s, *_ = O.factor(sym, w.values, simd=False)
    ok_v, L_v, *_ = O.factor(sym, w.values, simd=True)
    assert ok_s and ok_v
    assert same_lower(sym, L_s, L_v)
    b = w.rhs[0] if w.rhs.shape[0] else np.ones(w.n)
    assert bitwise(O.solve_chol(sym, L_s, b), O.solve_chol(sym, L_v, b))


@pytest.mark.parametrize("name,dims,zero_every", FRONT_CASES)
def test_simd_factor_equals_scalar_bitwise_ldlt(name, dims, zero_every):
    w = W.grid27(*dims, zero_every=zero_every, shift=30.0)
    sym = O.analyze(w.pat)
    r_s = O.factor(sym, w.values, kind="ldlt", simd=False)
    r_v = O.factor(sym, w.values, kind="ldlt", simd=True)
    assert r_s[0] and r_v[0] and r_s[3] > 0  # indefinite
    assert same_lower(sym, r_s[1], r_v[1])
    assert bitwise(r_s[2], r_v[2])
    assert r_s[3:] == r_v[3:]  # nNeg, nPerturbed


def test_front_failure_on_bad_last_pivot():
    """A -1e6 or NaN on the last-eliminated diagonal fails the factor in both kernels (la-real-front.test.mjs:99-114)."""
    w = W.grid27(10, 10, 10)
    sym = O.analyze(w.pat)
    last = int(sym.perm[w.n - 1])
    for bad in (-1e6, float("nan")):
        v = w.values.copy()
        v[entry(w.pat, last, last)] = bad
        for simd in (False, True):
            assert not O.factor(sym, v, simd=simd)[0]
            assert not O.factor(sym, v, kind="ldlt", simd=simd)[0] or not math.isnan(bad)


class Lcg:
    """The reference tests' uint32 LCG (la-real-solve.test.mjs:33-34): U(-0.5, 0.5)."""

    def __init__(self, seed=12345):
        self.s = seed

    def __call__(self):
        self.s = (self.s * 1664525 + 1013904223) & 0xFFFFFFFF
        return self.s / 4294967296 - 0.5


def special_rhs(rnd, n, zeros=0, special=False):
    b = np.zeros(n)
    for i in range(n):
        if zeros and i % zeros == 0:
            b[i] = -0.0 if i % (2 * zeros) == 0 else 0.0
        else:
            b[i] = rnd()
    if special:
        b[1], b[n - 2], b[n >> 1] = np.nan, np.inf, 5e-324
    return b


SOLVE_CASES = [("cube 12^3", (12, 12, 12), 0), ("slab 29x9x7", (29, 9, 7), 0), ("cube 11^3 zeros", (11, 11, 11), 3)]


@pytest.mark.parametrize("name,dims,zero_every", SOLVE_CASES)
def test_simd_solve_equals_scalar_bitwise(name, dims, zero_every):
    rnd = Lcg()
    w = W.grid27(*dims, zero_every=zero_every, sym=True)  # la-real-solve.test.mjs:15-30: symmetric values
    sym = O.analyze(w.pat)
    ok, Lx, *_ = O.factor(sym, w.values)
    assert ok and sym.nnzL >= 50000  # the SIMD solve engages (SOLVE_MIN_NNZL)
    for o in ({}, {"zeros": 3}, {"special": True}):
        b = special_rhs(rnd, w.n, **o)
        assert bitwise(O.solve_chol(sym, Lx, b, simd=True), O.solve_chol(sym, Lx, b, simd=False))
    b = special_rhs(rnd, w.n)
    assert relres(w.pat, w.values, O.solve_chol(sym, Lx, b), b) < 1e-12
    # LDL^T of the shifted (indefinite) matrix, single and many right-hand sides
    wi = W.grid27(*dims, zero_every=zero_every, shift=30.0, sym=True)
    okl, Ll, D, nneg, _ = O.factor(sym, wi.values, kind="ldlt")
    assert okl and nneg > 0
    for o in ({}, {"zeros": 3}, {"special": True}):
        b = special_rhs(rnd, w.n, **o)
        assert bitwise(O.solve_ldlt(sym, Ll, D, b, 1, simd=True), O.solve_ldlt(sym, Ll, D, b, 1, simd=False))
    for q in (1, 2, 3, 4, 11):
        b = np.concatenate([special_rhs(rnd, w.n, zeros=5 if k % 2 else 0) for k in range(q)])
        xv = O.solve_ldlt(sym, Ll, D, b, q, simd=True)
        xs = O.solve_ldlt(sym, Ll, D, b, q, simd=False)
        assert bitwise(xv, xs)
        if q == 3:  # each of the q vectors agrees with its single-vector solve to round-off
            for k in range(q):
                xk = O.solve_ldlt(sym, Ll, D, b[k * w.n:(k + 1) * w.n], 1)
                assert np.max(np.abs(xs[k * w.n:(k + 1) * w.n] - xk)) <= 1e-10 * np.max(np.abs(xk))  # indefinite: cond ~1e3


def two_by_two_system(nb):
    """Symmetric test matrix with [[0, a], [a, 0]] diagonal blocks (la-ldlt.test.mjs:13-46, real case)."""
    rnd = Lcg(4242)
    n = 2 * nb
    ent = {}

    def add(i, j, v):
        for a, b in ([(i, j)] if i == j else [(i, j), (j, i)]):
            ent[(a, b)] = ent.get((a, b), 0.0) + v

    for k in range(nb):
        add(2 * k, 2 * k + 1, 2 + rnd())
        add(2 * k, 2 * k, 0.0)
        add(2 * k + 1, 2 * k + 1, 0.0)
        if k + 1 < nb:
            add(2 * k + 1, 2 * k + 2, 0.3 * rnd())
    keys = sorted(ent, key=lambda t: t[0] * n + t[1])
    rowptr = np.zeros(n + 1, np.int32)
    for (i, _) in keys:
        rowptr[i + 1] += 1
    rowptr = np.cumsum(rowptr).astype(np.int32)
    colidx = np.array([j for (_, j) in keys], np.int32)
    vals = np.array([ent[k] for k in keys])
    xr = np.array([rnd() for _ in range(n)])
    pat = W.CsrPattern(n, rowptr, colidx)
    return pat, vals, xr, O.matvec(pat, vals, xr)


def test_ldlt_perturbation_counted_and_refinement_recovers_solution():
    pat, vals, xr, br = two_by_two_system(40)
    ident = np.arange(pat.n, dtype=np.int32)
    sym = O.analyze(pat, perm=ident)
    ok, Lx, D, nneg, npert = O.factor(sym, vals, kind="ldlt")
    assert ok and npert > 0
    x, rel, steps = O.solve_refined(sym, pat, vals, Lx, D, br, kind="ldlt", max_steps=30)
    assert np.max(np.abs(x - xr)) / np.max(np.abs(xr)) < 1e-10
    ok_u, _, npert_u, xu = O.ldlt_up(pat, ident, vals, b=br)
    assert ok_u and npert_u > 0


def test_ldlt_inertia_sylvester():
    n = 300

    def lap1d(k):
        return 2 - 2 * math.cos(k * math.pi / (n + 1))

    sigma = 0.5 * (lap1d(10) + lap1d(11))
    w = W.chain(n, 2 - sigma, -1.0)
    sym = O.analyze(w.pat)
    ok_u, nneg_u, _, _ = O.ldlt_up(w.pat, sym.perm, w.values)
    assert ok_u and nneg_u == 10
    ok, _, _, nneg, _ = O.factor(sym, w.values, kind="ldlt")
    assert ok and nneg == 10


# ---- complex-symmetric LDL^T (ldlt.mjs:648-864) -------------------------------------------------------------------
def _complex_case(N=5, shift=30.0, loss=0.3):
    w = W.maxwell3d(N, 2, 12.0, shift, 5, 1)
    return w, loss * w.values


def test_complex_ldlt_solves_the_complex_symmetric_system():
    import scipy.sparse as sp
    w, im = _complex_case()
    so = O.analyze(w.pat, perm=O.nd3_order(w.pat, w.x, w.y, w.z))
    ok, Lr, Li, Dr, Di, npert = O.cfactor(so, w.values, im)
    assert ok and npert == 0
    rng = np.random.default_rng(4)
    br, bi = rng.uniform(-1, 1, w.n), rng.uniform(-1, 1, w.n)
    xr, xi = O.csolve(so, Lr, Li, Dr, Di, br, bi)
    A = sp.csr_matrix((w.values + 1j * im, w.pat.colidx, w.pat.rowptr), shape=(w.n, w.n)).toarray()
    x = np.linalg.solve(A, br + 1j * bi)
    assert np.linalg.norm(xr + 1j * xi - x) / np.linalg.norm(x) < 1e-10
    # no conjugation: A^T = A, and the factor reproduces A = L D L^T
    assert np.array_equal(A, A.T)


def test_complex_ldlt_reduces_to_the_real_one_for_real_values():
    w, _ = _complex_case(4)
    so = O.analyze(w.pat, perm=O.nd3_order(w.pat, w.x, w.y, w.z))
    ok, Lr, Li, Dr, Di, npert = O.cfactor(so, w.values, np.zeros_like(w.values))
    okr, Lx, D, nneg, nper = O.factor(so, w.values, kind="ldlt")
    assert ok and okr and npert == nper

    def lower(L):  # the lower parts of the stored blocks (the upper part of a diagonal block is never read)
        out = []
        for s in range(so.nsuper):
            nc, m = int(so.superStart[s + 1] - so.superStart[s]), int(so.Sp[s + 1] - so.Sp[s])
            blk = L[so.Lxp[s]: so.Lxp[s] + m * nc].reshape(nc, m)
            out += [blk[c, c + 1:] for c in range(nc)]
        return np.concatenate(out)

    assert not np.any(lower(Li)) and not np.any(Di)
    assert np.max(np.abs(lower(Lr) - lower(Lx))) <= 1e-10 * np.max(np.abs(lower(Lx)))
    assert np.max(np.abs(Dr - D)) <= 1e-10 * np.max(np.abs(D))


def test_complex_ldlt_perturbs_a_zero_pivot_and_fails_on_nan():
    n = 4
    rp = np.arange(0, n * n + 1, n, dtype=np.int32)
    ci = np.tile(np.arange(n, dtype=np.int32), n)
    pat = W.CsrPattern(n, rp, ci)
    A = np.eye(n) * 2.0
    A[0, 0] = 0.0  # a zero pivot: perturbed to tau
    so = O.analyze(pat, perm=np.arange(n, dtype=np.int32))
    ok, Lr, Li, Dr, Di, npert = O.cfactor(so, A.reshape(-1), np.zeros(n * n))
    assert ok and npert == 1 and Dr[0] == 1e-13 * 2.0
    A[2, 2] = np.nan
    ok, *_ = O.cfactor(so, A.reshape(-1), np.zeros(n * n))
    assert not ok
