"""The product's host symbolic phase against the oracle, bit for bit, on the five benchmark systems at their full sizes:

  cfg1  2D P1 Poisson, 64 x 64 cells (AMD)
  cfg2  3D P1 elasticity, 40^3 hexes x 6 tets (nd3Order, leaf 2000)
  cfg3  256 batched 2D P1 heat problems (AMD per matrix)
  cfg4  3D P2 heat, 48^3 hexes x 6 tets (nd3Order)
  cfg5  3D Nedelec Maxwell, 32^3 hexes x 6 tets (nd3Order on edge midpoints)

Every array of the analysis (permutation, elimination tree, column counts, lower CSC with its source slots,
supernode partition and tree, row structures, Lxp) and every scalar must be identical: the numeric phase's parity
and the benchmark's flop counts rest on it. CPU only (the analysis runs on the host inside libampsolve.so).
"""
import numpy as np
import pytest

import ampsolve as A
import oracle as O
import workloads as W
from test_symbolic_and_abi import assert_same_symbolic


def _nd3(w):
    operm = O.nd3_order(w.pat, w.x, w.y, w.z)
    assert np.array_equal(A.nd3Order(w.pat, w.x, w.y, w.z), operm)
    osym = O.analyze(w.pat, perm=operm)
    ps = A.analyze(w.pat, ordering="nd3", x=w.x, y=w.y, z=w.z)
    assert_same_symbolic(ps, osym)
    return ps


def test_cfg1_poisson2d_64_amd():
    w = W.poisson2d(64)
    assert w.n == 63 * 63
    assert np.array_equal(A.amdOrder(w.pat), O.amd_order(w.pat))
    assert_same_symbolic(A.analyze(w.pat), O.analyze(w.pat))


def test_cfg2_elastic3d_40_nd3():
    w = W.elastic3d(40)
    assert w.n == 201720
    ps = _nd3(w)
    assert ps.maxFront == 7539


def test_cfg3_batch_256_amd_per_matrix():
    for i, w in enumerate(W.heat2d_batch(256)):
        perm = A.amdOrder(w.pat)
        assert np.array_equal(perm, O.amd_order(w.pat)), i
        assert_same_symbolic(A.analyze(w.pat, perm=perm), O.analyze(w.pat, perm=perm))


@pytest.mark.parametrize("name,make,n", [
    ("cfg4-heat3d-p2-48", lambda: W.heat3d_p2(48, q=1), 893855),
    ("cfg5-maxwell3d-32", lambda: W.maxwell3d(32, q=1), None),
])
def test_cfg4_cfg5_nd3(name, make, n):
    w = make()
    if n is not None:
        assert w.n == n
    _nd3(w)
