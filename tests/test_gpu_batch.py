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
