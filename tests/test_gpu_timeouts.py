"""Bounded device waits: a wait that runs out ends its kernel and the call reports AMP_DEVICE_TIMEOUT, after which
the same factor object works normally (the GPU still answers). The time-out is provoked by a wait bound of one poll
(amp_factor_set_wait_limit), so waits whose dependency is not yet complete give up at once; no kernel is broken and
no wait is left unbounded. Also: amp_matvec against the oracle's matVec (sparse.mjs:219-228)."""
import numpy as np
import pytest

import ampsolve as amp
import oracle as orc
import workloads as wl

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


@pytest.fixture(scope="module")
def system():
    w = wl.elastic3d(14)
    sym = amp.analyze(w.pat, ordering="nd3", x=w.x, y=w.y, z=w.z)
    so = orc.analyze(w.pat, perm=sym.perm)
    ok, Lx, _, _, _ = orc.factor(so, w.values)
    assert ok
    b = np.random.default_rng(11).uniform(-1, 1, w.n)
    return w, sym, orc.solve_chol(so, Lx, b), b


def test_tensor_core_update_wait_times_out_then_recovers(system):
    w, sym, xo, b = system
    num = amp.NumericFactor(sym, amp.CHOLESKY, amp.MIXED)
    num.set_wait_limit(1)  # the tcgen05 update's pipeline waits give up after one poll
    with pytest.raises(amp.AmpError) as e:
        num.factor(w.values)
    assert e.value.code == amp.AMP_DEVICE_TIMEOUT
    assert not num.ok
    with pytest.raises(amp.AmpError) as e:  # no successful factorization to solve with
        amp.solveNumeric(num, b)
    assert e.value.code == amp.AMP_NO_FACTOR
    num.set_wait_limit(0)  # defaults again: the same object factors and solves correctly
    assert num.factor(w.values)
    x, relres, _ = num.solve_refined_block(b[None, :], maxSteps=10, tol=1e-13)
    assert relres < 1e-13
    assert rel(x[0], xo) <= 1e-11


def test_solve_sweep_wait_times_out_then_recovers(system):
    w, sym, xo, b = system
    num = amp.factorNumeric(sym, w.values)
    assert num.ok
    num.set_wait_limit(1)  # the sweeps' flag and counter waits give up after one poll
    timeouts = 0
    for _ in range(3):
        try:
            x = amp.solveNumeric(num, b)
        except amp.AmpError as e:
            assert e.code == amp.AMP_DEVICE_TIMEOUT, e
            timeouts += 1
        else:  # a sweep whose every wait was already satisfied is still a correct sweep
            assert rel(x, xo) <= 1e-12
    assert timeouts > 0
    B = np.stack([b, 2 * b, -b])
    timeouts = 0
    for _ in range(3):  # several right-hand sides: the multi-vector sweeps
        try:
            X = num.solve_block(B)
        except amp.AmpError as e:
            assert e.code == amp.AMP_DEVICE_TIMEOUT, e
            timeouts += 1
        else:
            assert rel(X[2], -xo) <= 1e-12
    assert timeouts > 0
    num.set_wait_limit(0)
    assert rel(amp.solveNumeric(num, b), xo) <= 1e-12
    X = num.solve_block(np.stack([b, 2 * b, -b]))
    assert rel(X[1], 2 * xo) <= 1e-12


@pytest.mark.parametrize("q", [1, 3])
def test_matvec_matches_oracle(system, q):
    w, sym, _, _ = system
    num = amp.factorNumeric(sym, w.values)
    rng = np.random.default_rng(3 + q)
    X = rng.uniform(-1, 1, (q, w.n))
    Y = num.matVec(X if q > 1 else X[0])
    Y = Y.reshape(q, w.n)
    for k in range(q):
        yo = orc.matvec(w.pat, w.values, X[k])
        assert rel(Y[k], yo) <= 1e-14
    # the module-level matVec(pat, val, x) mirror
    assert rel(amp.matVec(w.pat, w.values, X[0]), orc.matvec(w.pat, w.values, X[0])) <= 1e-14
