"""CPU tests of the batched path's host side: a block-diagonal batch analyzed with the concatenated per-matrix AMD
orders gives every matrix exactly the structure the oracle gives it alone (permutation, elimination tree, column
counts, supernode partition), offset by its first row."""
import numpy as np

import batch as B
import oracle as O
import workloads as W


def test_block_diagonal_keeps_per_matrix_structure():
    ws = [W.heat2d_lognormal(N, 10 + i, 2) for i, N in enumerate((8, 13, 5, 20, 11, 16))]
    bc_pat, offs, slots = B.block_diagonal([w.pat for w in ws])
    import ampsolve as A
    perm = np.concatenate([A.amdOrder(w.pat) + offs[i] for i, w in enumerate(ws)]).astype(np.int32)
    sym = A.analyze(bc_pat, perm=perm)
    starts = list(sym.superStart)
    for i, w in enumerate(ws):
        o = O.analyze(w.pat)  # the reference's own per-matrix analysis (AMD)
        a, b = int(offs[i]), int(offs[i + 1])
        assert np.array_equal(sym.perm[a:b] - a, o.perm)
        par = sym.parent[a:b]
        assert np.array_equal(np.where(par < 0, -1, par - a), o.parent)
        assert np.array_equal(sym.colCount[a:b], o.colCount)
        mine = [s - a for s in starts if a <= s <= b]
        assert mine == list(o.superStart)
    assert sym.nnzL == sum(O.analyze(w.pat).nnzL for w in ws)


def test_batch_sizes_are_seeded_and_in_range():
    sz = W.heat2d_batch_sizes(256, 3)
    assert sz == W.heat2d_batch_sizes(256, 3) and len(sz) == 256
    assert all(16 <= N <= 128 and 1 <= q <= 64 for N, q in sz)
    assert len({N for N, _ in sz}) > 50
