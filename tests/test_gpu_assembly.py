"""On-device assembly of the CSR values (assembleCells, physics/src/common/scalar.ts:96-146, with the element slots of
la/sparse.mjs:113-185 and the Dirichlet restriction of fem/tri.mjs:192-225): the device values must be the same bits
as the host assembly of the same mesh and coefficients (tests' and benchmark's generators, which follow the
reference's element formulas and add the element entries in element order). Then the factorization of the
device-assembled values solves the system like the host values do."""
import numpy as np
import pytest

import ampsolve as A
import workloads as W

pytestmark = pytest.mark.gpu


def _assembly(kind, w, m):
    return A.Assembly(kind, w.pat, m.coords, m.conn, m.dofs)


@pytest.mark.parametrize("N,seed", [(64, 0), (20, 4711), (127, 9)])
def test_p1_heat_values_bit_exact(N, seed):
    w = W.poisson2d(N) if seed == 0 else W.heat2d_lognormal(N, seed, 1)
    m = W.mesh(0, N, seed)
    v = _assembly(A.AMP_ELEM_P1_TRI_SCALAR, w, m).assemble(m.coef)
    assert np.array_equal(v.view(np.uint64), w.values.view(np.uint64))


@pytest.mark.parametrize("N", [6, 40])
def test_p1_elasticity_values_bit_exact(N):
    w = W.elastic3d(N)
    m = W.mesh(1, N, E=1.0, nu=0.3)
    a = _assembly(A.AMP_ELEM_P1_TET_ELASTIC, w, m)
    v = a.assemble(m.coef)
    assert np.array_equal(v.view(np.uint64), w.values.view(np.uint64))
    # new coefficients (a stiffer half): assembled again on the device, the same as assembling with them on the host
    c2 = m.coef.copy()
    c2[0::2][: len(c2) // 4] = 3.0
    v2 = a.assemble(c2)
    assert not np.array_equal(v2, v) and np.all(np.isfinite(v2))


def test_assembled_values_factor_and_solve():
    torch = pytest.importorskip("torch")
    w = W.elastic3d(12)
    m = W.mesh(1, 12)
    a = _assembly(A.AMP_ELEM_P1_TET_ELASTIC, w, m)
    vals = torch.empty(w.pat.nnz, dtype=torch.float64, device="cuda")
    coef = torch.from_numpy(m.coef).cuda()
    torch.cuda.synchronize()
    a.assemble_device(coef.data_ptr(), True, vals.data_ptr())
    sym = A.analyze(w.pat, ordering="nd3", x=w.x, y=w.y, z=w.z)
    num = A.NumericFactor(sym, A.CHOLESKY, A.FP64)
    assert num.factor((vals.data_ptr(), vals.numel()), on_device=True)
    ref = A.factorNumeric(sym, w.values)
    b = w.rhs[0]
    x, xr = A.solveNumeric(num, b), A.solveNumeric(ref, b)
    assert np.array_equal(x, xr)  # same bits in, same bits out


def test_pattern_mismatch_is_reported():
    w = W.poisson2d(8)
    m = W.mesh(0, 8)
    rp = w.pat.rowptr.copy()
    ci = w.pat.colidx.copy()
    # drop the first off-diagonal entry of row 0 (and keep the arrays consistent by moving the diagonal in its place)
    row0 = ci[rp[0]:rp[1]]
    keep = np.concatenate([ci[:rp[0]], row0[row0 == 0], ci[rp[1]:]])
    rp2 = rp.copy()
    rp2[1:] -= len(row0) - 1
    bad = W.CsrPattern(w.n, rp2.astype(np.int32), keep.astype(np.int32))
    with pytest.raises(A.AmpError) as e:
        A.Assembly(A.AMP_ELEM_P1_TRI_SCALAR, bad, m.coords, m.conn, m.dofs)
    assert e.value.code == A.AMP_PATTERN_MISMATCH
