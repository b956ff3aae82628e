"""Many independent sparse systems factored and solved together (the batched 2D heat set: 256 uneven problems).

The batch is one block-diagonal system whose fill-reducing order is the concatenation of each matrix's own order
(amdOrder per matrix, as the reference analyzes each one). Its elimination forest is then the union of the matrices'
trees, and the etree postorder visits the roots in increasing index, so every matrix keeps exactly the permutation,
column counts and supernodes it has alone, offset by its first row. Each etree level of all the matrices goes in one
launch, and the whole numeric factorization of the batch is one captured CUDA graph.

Right-hand sides: matrix i has q_i of them; the batch solves max q_i vectors together (zeros where a matrix has
fewer) and refines them in FP64 against the block-diagonal values until every matrix's relative residual
||b_i - A_i x_i|| / ||b_i|| is below the tolerance for each of its right-hand sides.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Sequence

import numpy as np

import ampsolve as amp


@dataclass
class _Pat:
    n: int
    rowptr: np.ndarray
    colidx: np.ndarray

    @property
    def nnz(self) -> int:
        return int(self.rowptr[self.n])


def block_diagonal(pats: Sequence) -> tuple[_Pat, np.ndarray, np.ndarray]:
    """(pattern, row offsets [len + 1], CSR slot offsets [len + 1]) of the block-diagonal union of the patterns."""
    offs = np.zeros(len(pats) + 1, np.int64)
    nnz = np.zeros(len(pats) + 1, np.int64)
    for i, p in enumerate(pats):
        offs[i + 1] = offs[i] + int(p.n)
        nnz[i + 1] = nnz[i] + int(p.rowptr[p.n])
    rowptr = np.zeros(int(offs[-1]) + 1, np.int64)
    colidx = np.zeros(int(nnz[-1]), np.int32)
    for i, p in enumerate(pats):
        rp = np.asarray(p.rowptr[: p.n + 1], np.int64)
        rowptr[offs[i] + 1: offs[i + 1] + 1] = rp[1:] + nnz[i]
        colidx[nnz[i]: nnz[i + 1]] = np.asarray(p.colidx[: rp[-1]], np.int64) + offs[i]
    if nnz[-1] >= 2 ** 31:
        raise ValueError("batch has more than 2^31 - 1 pattern entries")
    return _Pat(int(offs[-1]), rowptr.astype(np.int32), colidx), offs, nnz


class BatchedCholesky:
    """Cholesky of many SPD systems at once (FP64 or mixed precision), per-matrix AMD orders."""

    def __init__(self, pats: Sequence, precision: int = amp.MIXED, perms: Sequence | None = None):
        self.count = len(pats)
        self.pat, self.offs, self.slots = block_diagonal(pats)
        orders = perms if perms is not None else [amp.amdOrder(p) for p in pats]
        perm = np.concatenate([np.asarray(o, np.int64) + self.offs[i] for i, o in enumerate(orders)]) \
            if self.count else np.zeros(0, np.int64)
        self.sym = amp.analyze(self.pat, perm=perm.astype(np.int32))
        self.num = amp.NumericFactor(self.sym, amp.CHOLESKY, precision)
        self.num.set_row_groups(self.offs)  # refinement measures each matrix's residual on its own
        self.values = None

    def factor(self, values: Sequence) -> bool:
        """values[i]: the CSR values of matrix i. True when every matrix is positive definite."""
        self.values = np.concatenate([np.asarray(v, np.float64) for v in values]) if self.count else np.zeros(0)
        return self.num.factor(self.values)

    def solve_refined(self, rhs: Sequence, maxSteps: int = 10, tol: float = 1e-12):
        """rhs[i]: (q_i, n_i) array. Returns ([x_i (q_i, n_i)], worst per-matrix relative residual, refinement
        steps)."""
        q = max((np.asarray(r).reshape(-1, int(self.offs[i + 1] - self.offs[i])).shape[0] for i, r in enumerate(rhs)),
                default=0)
        N = self.pat.n
        B = np.zeros((q, N))
        for i, r in enumerate(rhs):
            ni = int(self.offs[i + 1] - self.offs[i])
            r = np.asarray(r, np.float64).reshape(-1, ni)
            B[: r.shape[0], self.offs[i]: self.offs[i + 1]] = r
        X, rel, steps = self.num.solve_refined_block(B, maxSteps=maxSteps, tol=tol)
        out = []
        for i, r in enumerate(rhs):
            ni = int(self.offs[i + 1] - self.offs[i])
            qi = np.asarray(r).reshape(-1, ni).shape[0]
            out.append(X[:qi, self.offs[i]: self.offs[i + 1]].copy())
        return out, rel, steps
