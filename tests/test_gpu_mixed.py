"""GPU parity of the mixed-precision factor (FP32 fronts, BF16x3 tcgen05 updates) + FP64 iterative refinement.

The refined solution must reach relative residual <= 1e-12 and agree with the oracle's FP64 solution; the FP32
factor itself stays within the accuracy BF16x3 products allow of the oracle's FP64 factor.
"""
import numpy as np
import pytest

import ampsolve as amp
import oracle as orc
import workloads as wl

pytestmark = pytest.mark.gpu

RESIDUAL = 1e-12      # refinement target (rel. residual ||b - A x|| / ||b||)
SOLUTION = 1e-10      # refined solution vs the oracle's FP64 solution (relative, max norm)
FACTOR = 1e-3         # FP32 / BF16x3 factor vs the FP64 factor (relative, max norm over each block)


def rel(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


CASES = [
    ("poisson2d-64", lambda: wl.poisson2d(64), {}),
    ("elastic3d-10", lambda: wl.elastic3d(10), {"ordering": "nd3"}),
    ("elastic3d-16", lambda: wl.elastic3d(16), {"ordering": "nd3"}),
    ("grid27-12", lambda: wl.grid27(12, 12, 12, sym=True), {}),
]


@pytest.mark.parametrize("name,make,opts", CASES, ids=[c[0] for c in CASES])
def test_mixed_refined_matches_oracle(name, make, opts):
    w = make()
    o = dict(opts)
    if o.get("ordering") == "nd3":
        o.update(x=w.x, y=w.y, z=w.z)
    sym = amp.analyze(w.pat, o)
    num = amp.NumericFactor(sym, amp.CHOLESKY, amp.MIXED)
    assert num.factor(w.values)
    b = np.random.default_rng(3).uniform(-1, 1, w.n)
    x, relres, steps = num.solve_refined_block(b.reshape(1, -1), maxSteps=20, tol=RESIDUAL)
    x = x.reshape(-1)
    assert relres <= RESIDUAL, (relres, steps)
    so = orc.analyze(w.pat, perm=sym.perm)
    ok, Lx, _, _, _ = orc.factor(so, w.values)
    xo = orc.solve_chol(so, Lx, b)
    assert rel(x, xo) <= SOLUTION, rel(x, xo)
    # the FP32 factor against the FP64 oracle factor
    Lm = num.Lx
    worst = 0.0
    for s in range(so.nsuper):
        nc, m, lo = so.superStart[s + 1] - so.superStart[s], so.Sp[s + 1] - so.Sp[s], so.Lxp[s]
        A = Lm[lo: lo + m * nc].reshape(nc, m).T
        B = Lx[lo: lo + m * nc].reshape(nc, m).T
        mask = np.tril(np.ones((m, nc), bool))
        worst = max(worst, np.max(np.abs(A[mask] - B[mask])) / max(np.max(np.abs(B[mask])), 1e-300))
    assert worst <= FACTOR, worst


def test_mixed_not_positive_definite():
    w = wl.hex_q1(4, 4, 3)
    num = amp.NumericFactor(amp.analyze(w.pat), amp.CHOLESKY, amp.MIXED)
    assert num.factor(-w.values) is False
