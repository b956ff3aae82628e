"""The orderings (amdOrder, ndOrder, nd3Order) and the supernode structure pinned against fixtures derived from the
reference's JavaScript source, for the oracle and for the product.

The fixtures (tests/golden/ordering_*.json) come from tests/golden/js_transcription.py, a statement-by-statement
Python transcription of sparse.mjs:231-283, 297-592, 597-902 and order3d.mjs:11-77 written from the JS text alone
(with Int32Array's out-of-range read / ignored write semantics emulated), separately from the C oracle and from the
product's C++. Three cases were also traced by hand through amdOrder (sparse.mjs line numbers):

  path of 8 (0-1-...-7): no dense rows (dense = min(6, max(16, 10 sqrt 8)) = 6 > degrees). The degree-1 list holds
  7 -> 0 (later insertions go first, :350-352), so 7 is the first pivot; its only neighbour 6 drops to degree 1 and
  is pushed in front of 0 (:549-556); the pivots run 7, 6, ..., 2, 1, and eliminating 1 leaves 0 with no external
  degree, so 0 is absorbed by mass elimination (:497-505). Absorbed elements point to their absorber (:416-419),
  1 is the root, its children are linked 2 then 0 (:567-580), and the depth-first postorder (:581-597) gives
  [7, 6, 5, 4, 3, 2, 0, 1].
  arrow of 6, hub last (edges i-5): the hub's degree 5 exceeds dense = min(4, 16) = 4, so it is removed up front
  with parent n (:344-349); the leaves 4, 3, 2, 1, 0 are pivots with empty elements (roots, :563-566); the
  postorder visits the roots 0..4, then n's child 5: [0, 1, 2, 3, 4, 5].
  arrow of 6, hub first (edges 0-i): the same with the hub at 0: [1, 2, 3, 4, 5, 0].
"""
import glob
import json
import os

import numpy as np
import pytest

import ampsolve as A
import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
FILES = sorted(glob.glob(os.path.join(HERE, "golden", "ordering_*.json")))
HAND = {"path8-amd": [7, 6, 5, 4, 3, 2, 0, 1], "arrow6-hub-last-amd": [0, 1, 2, 3, 4, 5],
        "arrow6-hub-first-amd": [1, 2, 3, 4, 5, 0]}


class _Pat:
    def __init__(self, d):
        self.n = d["n"]
        self.rowptr = np.asarray(d["rowptr"], np.int32)
        self.colidx = np.asarray(d["colidx"], np.int32)

    @property
    def nnz(self):
        return int(self.rowptr[-1])


def _orders(d, p):
    c = {k: np.asarray(v, np.float64) for k, v in d["coords"].items()}
    leaf = d["params"].get("leaf")
    if d["ordering"] == "amd":
        return O.amd_order(p), A.amdOrder(p)
    if d["ordering"] == "nd":
        return O.nd_order(p, c["x"], c["y"], leaf), A.ndOrder(p, c["x"], c["y"], leaf)
    return O.nd3_order(p, c["x"], c["y"], c["z"], leaf), A.nd3Order(p, c["x"], c["y"], c["z"], leaf)


def test_fixtures_present():
    names = {json.load(open(f))["name"] for f in FILES}
    assert set(HAND) <= names and len(names) >= 9


@pytest.mark.parametrize("path", FILES, ids=[os.path.basename(f)[9:-5] for f in FILES])
def test_ordering_and_structure_match_js_derivation(path):
    d = json.load(open(path))
    if d["name"] in HAND:
        assert d["order"] == HAND[d["name"]]
    p = _Pat(d)
    o_order, p_order = _orders(d, p)
    assert list(o_order) == d["order"]
    assert list(p_order) == d["order"]
    for sym in (O.analyze(p, perm=o_order), A.analyze(p, perm=np.asarray(p_order, np.int32))):
        for f in ("perm", "parent", "colCount", "superStart", "superParent", "Sp", "Si", "Lxp"):
            assert [int(v) for v in np.asarray(getattr(sym, f))] == d[f], f
        assert (sym.nnzL, sym.flops, sym.maxFront) == (d["nnzL"], d["flops"], d["maxFront"])
