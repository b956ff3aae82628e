"""Golden fixtures (tests/golden/structure_*.json, made by tests/golden/make_golden.py from the definitions with
numpy only): permutation after the etree postorder, elimination tree, column counts, nnzL, flops, fingerprint and the
dense Cholesky factor. The oracle and the product's host symbolic phase are both checked against them on CPU; the
product's device factor is checked against the dense factor on the GPU.
"""
import glob
import json
import os

import numpy as np
import pytest

import ampsolve as A
import oracle as O
import workloads as W

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURES = sorted(glob.glob(os.path.join(HERE, "golden", "structure_*.json")))


def load(path):
    d = json.load(open(path))
    pat = W.CsrPattern(d["n"], np.array(d["rowptr"], np.int32), np.array(d["colidx"], np.int32))
    return d, pat


def check_structure(d, sym):
    assert np.array_equal(sym.perm, d["perm"])
    assert np.array_equal(sym.parent, d["parent"])
    assert np.array_equal(sym.colCount, d["colCount"])
    assert sym.nnzL == d["nnzL"] and sym.flops == d["flops"]
    assert sym.patternKey == d["fingerprint"]
    # every supernode's row list covers exactly the union of its columns' nonzero rows in the dense factor
    n = d["n"]
    Ld = np.array(d["L_dense_rowmajor"]).reshape(n, n)
    for s in range(sym.nsuper):
        f, l = sym.superStart[s], sym.superStart[s + 1]
        rows = set(sym.Si[sym.Sp[s]:sym.Sp[s + 1]].tolist())
        for j in range(f, l):
            assert set(np.nonzero(Ld[j:, j])[0] + j) <= rows


def dense_from_supernodes(sym, Lx):
    n = sym.n
    Ld = np.zeros((n, n))
    for s in range(sym.nsuper):
        f, nc = sym.superStart[s], sym.superStart[s + 1] - sym.superStart[s]
        rows = sym.Si[sym.Sp[s]:sym.Sp[s + 1]]
        m = len(rows)
        blk = np.asarray(Lx[sym.Lxp[s]:sym.Lxp[s] + m * nc]).reshape(nc, m)  # column-major m x nc
        for c in range(nc):
            for r in range(c, m):
                Ld[rows[r], f + c] = blk[c, r]
    return Ld


@pytest.mark.parametrize("path", FIXTURES, ids=[os.path.basename(p)[10:-5] for p in FIXTURES])
def test_oracle_against_golden(path):
    d, pat = load(path)
    sym = O.analyze(pat, perm=np.array(d["perm0"], np.int32))
    check_structure(d, sym)
    ok, Lx, *_ = O.factor(sym, np.array(d["values"]))
    assert ok
    Lref = np.array(d["L_dense_rowmajor"]).reshape(d["n"], d["n"])
    assert np.max(np.abs(dense_from_supernodes(sym, Lx) - Lref)) <= 1e-12 * np.max(np.abs(Lref))


@pytest.mark.parametrize("path", FIXTURES, ids=[os.path.basename(p)[10:-5] for p in FIXTURES])
def test_product_symbolic_against_golden(path):
    d, pat = load(path)
    sym = A.analyze(pat, perm=np.array(d["perm0"], np.int32))
    check_structure(d, sym)


@pytest.mark.gpu
@pytest.mark.parametrize("path", FIXTURES, ids=[os.path.basename(p)[10:-5] for p in FIXTURES])
def test_product_factor_against_golden(path):
    d, pat = load(path)
    sym = A.analyze(pat, perm=np.array(d["perm0"], np.int32))
    num = A.NumericFactor(sym)
    assert num.factor(np.array(d["values"]))
    Lref = np.array(d["L_dense_rowmajor"]).reshape(d["n"], d["n"])
    assert np.max(np.abs(dense_from_supernodes(sym, num.Lx) - Lref)) <= 1e-12 * np.max(np.abs(Lref))
