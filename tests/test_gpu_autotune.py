"""The schedule autotuner (amp_plan_autotune) and the schedule parameters it searches (group width, whole-front
cut-off, deferral of the update beyond the next group): every candidate schedule must give the same factor to round-off (parity with the oracle at the FP64 bar), the tuner must return one of its
candidates, keep it, and hand it to a second plan of the same pattern from its cache without timing again."""
import numpy as np
import pytest

import ampsolve as A
import oracle as O
import workloads as W

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.mark.parametrize("gb,sf,dfr", [(1, 32, 1), (2, 64, 1), (8, 128, 1), (16, 96, 1), (1, 64, 3), (2, 128, 2),
                                       (2, 64, 8), (4, 128, 4)])
@pytest.mark.parametrize("precision", [A.FP64, A.MIXED], ids=["fp64", "mixed"])
def test_every_schedule_matches_the_oracle(gb, sf, dfr, precision):
    w = W.elastic3d(14)
    sym = A.analyze(w.pat, ordering="nd3", x=w.x, y=w.y, z=w.z, groupBlocks=gb, smallFront=sf, deferUpdates=dfr)
    so = O.analyze(w.pat, perm=sym.perm)
    ok, Lx, *_ = O.factor(so, w.values)
    b = w.rhs[0]
    xo = O.solve_chol(so, Lx, b)
    num = A.NumericFactor(sym, A.CHOLESKY, precision)
    assert num.factor(w.values)
    if precision == A.FP64:
        assert rel(A.solveNumeric(num, b), xo) <= 1e-12
    else:
        X, rr, _ = num.solve_refined_block(b[None, :], maxSteps=10, tol=1e-12)
        assert rr <= 1e-12 and rel(X[0], xo) <= 1e-10


def test_ldlt_schedule_parameters():
    w = W.maxwell3d(8, 2, 12.0, 40.0, 5, 1)
    for gb, sf, dfr in ((1, 32, 1), (8, 64, 1), (1, 32, 4)):
        sym = A.analyze(w.pat, ordering="nd3", x=w.x, y=w.y, z=w.z, groupBlocks=gb, smallFront=sf, deferUpdates=dfr)
        f = A.SupernodalLDLT(sym)
        r = f.factor(w.values)
        so = O.analyze(w.pat, perm=sym.perm)
        ok, Lx, D, nneg, npert = O.factor(so, w.values, kind="ldlt")
        assert r["ok"] and (r["nNeg"], r["nPerturbed"]) == (nneg, npert)
        assert f.solveRefined(w.pat, w.values, w.rhs[0], maxSteps=5, tol=1e-14)["relResidual"] < 1e-12


def test_autotune_picks_caches_and_keeps_a_candidate():
    w = W.elastic3d(16)
    sym = A.analyze(w.pat, ordering="nd3", x=w.x, y=w.y, z=w.z)
    r = A.autotune(sym, w.values, A.CHOLESKY, A.MIXED)
    assert not r["cached"] and r["candidates"] == 11
    assert r["groupBlocks"] in (1, 2, 4, 8) and r["smallFront"] in (64, 128) and r["deferUpdates"] in (1, 2, 4, 8)
    assert 0 < r["msBest"] <= r["msDefault"]
    num = A.NumericFactor(sym, A.CHOLESKY, A.MIXED)  # the tuned schedule factors correctly
    assert num.factor(w.values)
    X, rr, _ = num.solve_refined_block(w.rhs[:1], maxSteps=10, tol=1e-12)
    assert rr <= 1e-12
    with pytest.raises(A.AmpError, match="already has a factor"):
        A.autotune(sym, w.values, A.CHOLESKY, A.MIXED)
    sym2 = A.analyze(w.pat, ordering="nd3", x=w.x, y=w.y, z=w.z)
    r2 = A.autotune(sym2, w.values, A.CHOLESKY, A.MIXED)
    assert r2["cached"] and (r2["groupBlocks"], r2["smallFront"], r2["deferUpdates"]) == \
        (r["groupBlocks"], r["smallFront"], r["deferUpdates"])
