"""GPU parity at the benchmark systems' full sizes (the sizes bench.py measures), against the oracle.

  cfg2  3D P1 elasticity 40^3 (201,720 DOF, nd3Order): FP64 factor + solve against the oracle's FP64 factor + solve
        to 1e-12 relative; the mixed factor (FP32 fronts, BF16x3 tensor-core updates) + FP64 GMRES-IR to relative
        residual 1e-12 and to 1e-10 of the oracle's solution.
  cfg3  the 256 batched 2D heat problems as one block-diagonal factorization, FP64 and mixed + FP64 refinement, every
        matrix's right-hand sides against the oracle's factor of that matrix alone.
  cfg4  3D P2 heat 48^3 (893,855 DOF): too large for the oracle on one core (12.7 TFLOP), so checked through
        properties: both precisions refined to relative residual <= 1e-12, the normwise backward error small, and the
        mixed solution within 1e-10 of the FP64 one; the same system at 16^3 against the oracle in both precisions.
  cfg5  3D Nedelec Maxwell 32^3, LDL^T (indefinite): inertia and perturbation count exact against the oracle, the
        solution within the oracle's own sensitivity (its change under a 1-ulp symmetric perturbation of A, times
        100; the bound of test_gpu_ldlt.py), refined residual <= 1e-12.
"""
import numpy as np
import pytest

import ampsolve as A
import batch as BT
import oracle as O
import workloads as W
from test_gpu_ldlt import lower_parts, rel as rel2, ulp_perturbed

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12    # FP64 GPU solution vs the oracle's (relative, max norm)
MIXED_TOL = 1e-10   # refined mixed solution vs the oracle's FP64 solution
RESIDUAL = 1e-12    # refinement target ||b - A x|| / ||b||


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def residual(pat, vals, x, b):
    return float(np.linalg.norm(O.matvec(pat, vals, x) - b) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def cfg2():
    w = W.elastic3d(40)
    sym = A.analyze(w.pat, ordering="nd3", x=w.x, y=w.y, z=w.z)
    so = O.analyze(w.pat, perm=sym.perm)
    ok, Lx, _, _, _ = O.factor(so, w.values, simd=True)  # bitwise equal to the scalar restatement
    assert ok
    b = w.rhs[0]
    return w, sym, O.solve_chol(so, Lx, b), b


def test_cfg2_elastic3d_40_fp64_matches_oracle(cfg2):
    w, sym, xo, b = cfg2
    num = A.factorNumeric(sym, w.values)
    assert num.ok
    x = A.solveNumeric(num, b)
    assert rel(x, xo) <= FP64_TOL, rel(x, xo)
    assert residual(w.pat, w.values, x, b) <= RESIDUAL


def test_cfg2_elastic3d_40_mixed_gmres_ir_matches_oracle(cfg2):
    w, sym, xo, b = cfg2
    num = A.NumericFactor(sym, A.CHOLESKY, A.MIXED)
    assert num.factor(w.values)
    out = num.solve_gmres(b, tol=1e-12, restart=40, maxIter=300)
    assert out["converged"] and out["relres"] <= RESIDUAL
    assert rel(out["x"], xo) <= MIXED_TOL, rel(out["x"], xo)
    assert residual(w.pat, w.values, out["x"], b) <= RESIDUAL
    # plain FP64 refinement (solveRefined) reaches the same bar with more steps
    X, rr, steps = num.solve_refined_block(b[None, :], maxSteps=10, tol=RESIDUAL)
    assert rr <= RESIDUAL and rel(X[0], xo) <= MIXED_TOL


@pytest.mark.parametrize("precision", [A.FP64, A.MIXED], ids=["fp64", "mixed"])
def test_cfg3_batch_256_matches_per_matrix_oracle(precision):
    ws = W.heat2d_batch(256)
    bc = BT.BatchedCholesky([w.pat for w in ws], precision=precision)
    assert bc.factor([w.values for w in ws])
    xs, rr, steps = bc.solve_refined([w.rhs for w in ws], maxSteps=10, tol=RESIDUAL)
    assert rr <= RESIDUAL
    worst = 0.0
    for w, x in zip(ws, xs):
        o = O.analyze(w.pat)
        ok, Lx, *_ = O.factor(o, w.values, simd=True)
        assert ok
        for k in range(w.rhs.shape[0]):
            xo = O.solve_chol(o, Lx, w.rhs[k])
            worst = max(worst, float(np.linalg.norm(x[k] - xo) / np.linalg.norm(xo)))
    assert worst <= FP64_TOL, worst


def test_cfg4_heat3d_p2_48_properties():
    w = W.heat3d_p2(48, q=16)
    assert w.n == 893855
    sym = A.analyze(w.pat, ordering="nd3", x=w.x, y=w.y, z=w.z)
    B = w.rhs[:16]
    anorm = float(np.linalg.norm(w.values))
    out = {}
    for prec in (A.FP64, A.MIXED):
        num = A.NumericFactor(sym, A.CHOLESKY, prec)
        assert num.factor(w.values)
        X, rr, _ = num.solve_refined_block(B, maxSteps=10, tol=RESIDUAL)
        assert rr <= RESIDUAL, (prec, rr)
        for k in (0, 7, 15):
            r = np.linalg.norm(O.matvec(w.pat, w.values, X[k]) - B[k])
            assert r / (anorm * np.linalg.norm(X[k]) + np.linalg.norm(B[k])) <= 1e-15
        out[prec] = X
        del num
    fe = max(float(np.linalg.norm(out[A.MIXED][k] - out[A.FP64][k]) / np.linalg.norm(out[A.FP64][k]))
             for k in range(16))
    assert fe <= MIXED_TOL, fe


@pytest.mark.parametrize("precision", [A.FP64, A.MIXED], ids=["fp64", "mixed"])
def test_cfg4_system_at_16_matches_oracle(precision):
    w = W.heat3d_p2(16, q=4)
    sym = A.analyze(w.pat, ordering="nd3", x=w.x, y=w.y, z=w.z)
    so = O.analyze(w.pat, perm=sym.perm)
    ok, Lx, *_ = O.factor(so, w.values, simd=True)
    assert ok
    num = A.NumericFactor(sym, A.CHOLESKY, precision)
    assert num.factor(w.values)
    B = w.rhs[:4]
    if precision == A.FP64:
        X = num.solve_block(B)
        tol = FP64_TOL
    else:
        X, rr, _ = num.solve_refined_block(B, maxSteps=10, tol=RESIDUAL)
        assert rr <= RESIDUAL
        tol = MIXED_TOL
    for k in range(4):
        assert rel(X[k], O.solve_chol(so, Lx, B[k])) <= tol


def test_cfg5_maxwell3d_32_ldlt_matches_oracle():
    w = W.maxwell3d(32, q=2)
    sym = A.analyze(w.pat, ordering="nd3", x=w.x, y=w.y, z=w.z)
    so = O.analyze(w.pat, perm=sym.perm)
    ok_o, Lx_o, D_o, nneg_o, npert_o = O.factor(so, w.values, kind="ldlt", simd=True)
    ok_p, Lx_p, D_p, _, _ = O.factor(so, ulp_perturbed(w.pat, w.values), kind="ldlt", simd=True)
    assert ok_o and ok_p
    f = A.SupernodalLDLT(sym)
    r = f.factor(w.values)
    assert r["ok"] and r["nNeg"] > 0
    assert (r["nNeg"], r["nPerturbed"]) == (nneg_o, npert_o)
    assert rel2(f.D, D_o) <= max(1e-11, 100 * rel2(D_p, D_o))
    Lo = lower_parts(so, Lx_o)
    assert rel2(lower_parts(so, f.Lx), Lo) <= max(1e-11, 100 * rel2(lower_parts(so, Lx_p), Lo))
    b = w.rhs[0]
    xo = O.solve_ldlt(so, Lx_o, D_o, b)
    tol_x = max(1e-11, 100 * rel2(O.solve_ldlt(so, Lx_p, D_p, b), xo))
    assert rel2(f.solve(b), xo) <= tol_x
    ref = f.solveRefined(w.pat, w.values, b, maxSteps=5, tol=1e-14)
    assert ref["relResidual"] <= RESIDUAL
