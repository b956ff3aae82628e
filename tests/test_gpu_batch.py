"""GPU: many uneven 2D heat problems factored and solved as one batch (FP64 and mixed precision + FP64 refinement),
each matrix's solution checked against the oracle's factor of that matrix alone."""
import numpy as np
import pytest

import ampsolve as A
import batch as B
import oracle as O
import workloads as W

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", [A.FP64, A.MIXED], ids=["fp64", "mixed"])
def test_batch_matches_per_matrix_oracle(precision):
    sizes = W.heat2d_batch_sizes(12, 7)
    ws = [W.heat2d_lognormal(N, 500 + i, q) for i, (N, q) in enumerate(sizes)]
    bc = B.BatchedCholesky([w.pat for w in ws], precision=precision)
    assert bc.factor([w.values for w in ws])
    xs, rel, steps = bc.solve_refined([w.rhs for w in ws], maxSteps=10, tol=1e-13)
    for w, x in zip(ws, xs):
        o = O.analyze(w.pat)
        ok, Lx, *_ = O.factor(o, w.values)
        assert ok
        for k in range(w.rhs.shape[0]):
            xo = O.solve_chol(o, Lx, w.rhs[k])
            assert np.linalg.norm(x[k] - xo) / np.linalg.norm(xo) < 1e-12
            r = O.matvec(w.pat, w.values, x[k]) - w.rhs[k]
            assert np.linalg.norm(r) / np.linalg.norm(w.rhs[k]) < 1e-12


def test_batch_refines_each_matrix_to_its_own_tolerance():
    # one matrix's right-hand sides are 1e-8 of the others': a residual taken over the whole batch would stop before
    # that matrix is solved to 1e-12 of its own ||b||; the per-matrix (row group) residual does not
    sizes = W.heat2d_batch_sizes(6, 9)
    ws = [W.heat2d_lognormal(N, 900 + i, q) for i, (N, q) in enumerate(sizes)]
    rhs = [w.rhs.copy() for w in ws]
    rhs[2] *= 1e-8
    bc = B.BatchedCholesky([w.pat for w in ws], precision=A.MIXED)
    assert bc.factor([w.values for w in ws])
    xs, rel, steps = bc.solve_refined(rhs, maxSteps=20, tol=1e-12)
    assert rel < 1e-12
    for w, x, b in zip(ws, xs, rhs):
        for k in range(b.shape[0]):
            r = O.matvec(w.pat, w.values, x[k]) - b[k]
            assert np.linalg.norm(r) / np.linalg.norm(b[k]) < 1e-12


def test_row_group_arguments():
    w = W.poisson2d(16)
    num = A.NumericFactor(A.analyze(w.pat), A.CHOLESKY, A.FP64)
    with pytest.raises(A.AmpError, match="from 0 to n"):
        num.set_row_groups([0, 10])
    with pytest.raises(A.AmpError, match="must not decrease"):
        num.set_row_groups([0, 100, 50, w.n])
    num.set_row_groups([0, 100, w.n])
    assert num.factor(w.values)
    X, rel, _ = num.solve_refined_block(w.rhs, maxSteps=3, tol=1e-14)
    assert rel < 1e-13
    num.set_row_groups(None)
