"""GPU parity of the multi-vector solves (solveNumericMulti, sparse.mjs:1261-1310; solveMany, ldlt.mjs:595-643):
several right-hand sides swept together in the interleaved layout, in groups of up to 64, checked vector by vector
against the oracle's one-vector solves."""
import numpy as np
import pytest

import ampsolve as amp
import oracle as orc
import workloads as wl

pytestmark = pytest.mark.gpu

TOL = 1e-12  # FP64: relative error of each solution vs the oracle's


def rel(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


def _setup(w, ordering="nd3"):
    sym = amp.analyze(w.pat, ordering=ordering, x=w.x, y=w.y, z=w.z)
    so = orc.analyze(w.pat, perm=sym.perm)
    ok, Lx, *_ = orc.factor(so, w.values)
    assert ok
    return sym, so, Lx


@pytest.mark.parametrize("q", [2, 7, 64, 65, 130])
def test_fp64_multi_matches_oracle(q):
    w = wl.elastic3d(9)
    sym, so, Lx = _setup(w)
    num = amp.NumericFactor(sym, amp.CHOLESKY, amp.FP64)
    assert num.factor(w.values)
    rng = np.random.default_rng(q)
    B = rng.uniform(-1, 1, (q, w.n))
    B[q // 2] = 0.0  # a zero right-hand side solves to zero
    X = num.solve_block(B)
    assert not np.any(X[q // 2])
    for k in range(q):
        if k == q // 2:
            continue
        assert rel(X[k], orc.solve_chol(so, Lx, B[k])) <= TOL
    # the one-vector sweep and the multi-vector sweep agree to rounding
    x1 = num.solve_block(B[1:2])[0]
    assert rel(x1, X[1]) <= 1e-13


def test_multi_supernode_chains_and_ragged_blocks():
    # a 2D problem with long supernode chains (AMD) and a 3D one whose root has several 64-column blocks
    for w, ordering in [(wl.poisson2d(40), "amd"), (wl.grid27(11, 11, 11, sym=True), "amd")]:
        sym = amp.analyze(w.pat, ordering=ordering)
        so = orc.analyze(w.pat, perm=sym.perm)
        ok, Lx, *_ = orc.factor(so, w.values)
        num = amp.NumericFactor(sym, amp.CHOLESKY, amp.FP64)
        assert num.factor(w.values)
        B = np.random.default_rng(3).uniform(-1, 1, (5, w.n))
        X = num.solve_block(B)
        for k in range(5):
            assert rel(X[k], orc.solve_chol(so, Lx, B[k])) <= TOL


@pytest.mark.parametrize("q", [3, 40])
def test_mixed_multi_refined(q):
    w = wl.elastic3d(10)
    sym = amp.analyze(w.pat, ordering="nd3", x=w.x, y=w.y, z=w.z)
    num = amp.NumericFactor(sym, amp.CHOLESKY, amp.MIXED)
    assert num.factor(w.values)
    B = np.random.default_rng(11).uniform(-1, 1, (q, w.n))
    X, relres, steps = num.solve_refined_block(B, maxSteps=20, tol=1e-13)
    assert relres < 1e-13 and steps >= 1
    for k in range(q):
        r = orc.matvec(w.pat, w.values, X[k]) - B[k]
        assert np.linalg.norm(r) / np.linalg.norm(B[k]) < 1e-12


def test_multi_device_and_pinned_buffers():
    torch = pytest.importorskip("torch")
    w = wl.elastic3d(8)
    sym, so, Lx = _setup(w)
    num = amp.NumericFactor(sym, amp.CHOLESKY, amp.FP64)
    assert num.factor(w.values)
    q = 6
    B = np.random.default_rng(5).uniform(-1, 1, (q, w.n))
    Xo = np.stack([orc.solve_chol(so, Lx, B[k]) for k in range(q)])
    bd = torch.from_numpy(B.reshape(-1).copy()).cuda()
    xd = torch.empty_like(bd)
    rr, steps = num.solve_refined_device(bd.data_ptr(), xd.data_ptr(), q, maxSteps=3, tol=1e-14)
    torch.cuda.synchronize()
    assert rr < 1e-13
    assert rel(xd.cpu().numpy().reshape(q, w.n), Xo) <= TOL
    bh = torch.from_numpy(B.reshape(-1).copy()).pin_memory()
    xh = torch.empty_like(bh).pin_memory()
    num.solve_refined_host_pinned(bh.data_ptr(), xh.data_ptr(), q, 3, 1e-14)
    assert rel(xh.numpy().reshape(q, w.n), Xo) <= TOL
    num.solve_device(bd.data_ptr(), xd.data_ptr(), q)
    torch.cuda.synchronize()
    assert rel(xd.cpu().numpy().reshape(q, w.n), Xo) <= TOL


def test_ldlt_multi_matches_oracle():
    from test_gpu_ldlt import run_case, shifted

    w = wl.grid27(9, 9, 9, sym=True)
    r = run_case(w, shifted(w, 30.0), {}, nrhs=9)  # nine vectors in one interleaved sweep, each vs the oracle
    assert r["nNeg"] > 0
