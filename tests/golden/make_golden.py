"""Generate tests/golden/structure_*.json: small SPD systems with a fixed permutation and their factor structure,
computed from the definitions, independently of both the oracle and the product.

For P A P^T (P from the given new->old permutation) the script runs a dense boolean symbolic elimination (the
filled graph, by definition), then reads off
  parent[j]   = min { i > j : L[i, j] != 0 }, or -1         (elimination tree, sparse.mjs:597-625)
  colCount[j] = #{ i >= j : L[i, j] != 0 }                 (column counts incl. the diagonal, sparse.mjs:719-759)
  nnzL = sum colCount, flops = sum colCount^2               (sparse.mjs:754-759)
  fingerprint = "n:nnz:fnv1a(rowptr bytes, colidx bytes)"   (sparse.mjs:908-925)
with the permutation analyze() returns (the given one followed by the etree postorder), and stores the dense
Cholesky factor of P A P^T from numpy (LAPACK) for a numeric cross-check.

The matrices: a path (tridiagonal), an arrow with the hub first (fill everywhere) and last (no fill), a 4x4 5-point
grid and a 3x3x3 27-point grid with a scrambled order, a block-diagonal pair and a 1x1. Run from the repo root:
    python tests/golden/make_golden.py
"""
import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def csr_from_dense(Ad):
    n = Ad.shape[0]
    rowptr, colidx, vals = [0], [], []
    for i in range(n):
        for j in range(n):
            if Ad[i, j] != 0 or i == j:
                colidx.append(j)
                vals.append(float(Ad[i, j]))
        rowptr.append(len(colidx))
    return rowptr, colidx, vals


def fnv1a(rowptr, colidx):
    h = 0x811C9DC5
    for arr in (rowptr, colidx):
        for byte in np.asarray(arr, "<i4").tobytes():
            h = ((h ^ byte) * 0x01000193) & 0xFFFFFFFF
    return f"{len(rowptr) - 1}:{len(colidx)}:{h:x}"


def structure(Ad, perm):
    n = Ad.shape[0]
    B = (Ad[np.ix_(perm, perm)] != 0) | np.eye(n, dtype=bool)
    F = B.copy()
    for k in range(n):  # eliminate k: its later neighbours become a clique
        nb = [i for i in range(k + 1, n) if F[i, k]]
        for a in nb:
            for b in nb:
                F[a, b] = True
    L = np.tril(F)
    parent = [int(next((i for i in range(j + 1, n) if L[i, j]), -1)) for j in range(n)]
    cc = [int(L[j:, j].sum()) for j in range(n)]
    return parent, cc


def postorder(parent):
    """Etree postorder (sparse.mjs:626-645): roots in increasing index, each subtree's children in increasing index,
    a node after its children. Written recursively here, from that definition."""
    n = len(parent)
    kids = [[] for _ in range(n)]
    for j in range(n):
        if parent[j] >= 0:
            kids[parent[j]].append(j)
    out = []

    def visit(v):
        for c in kids[v]:
            visit(c)
        out.append(v)

    for j in range(n):
        if parent[j] < 0:
            visit(j)
    return out


def spd_from_pattern(P, seed):
    """Values on a symmetric boolean pattern: off-diagonals in -(0.5, 1.5), diagonal = row sum + 1 (SPD)."""
    rng = np.random.default_rng(seed)
    n = P.shape[0]
    A = np.zeros((n, n))
    for i in range(n):
        for j in range(i):
            if P[i, j]:
                A[i, j] = A[j, i] = -(0.5 + rng.random())
    for i in range(n):
        A[i, i] = -A[i].sum() + 1.0
    return A


def grid_pattern(nx, ny, nz, stencil27):
    n = nx * ny * nz
    P = np.zeros((n, n), bool)
    idx = lambda i, j, k: i + nx * (j + ny * k)
    for k in range(nz):
        for j in range(ny):
            for i in range(nx):
                for dk in (-1, 0, 1):
                    for dj in (-1, 0, 1):
                        for di in (-1, 0, 1):
                            if not stencil27 and abs(di) + abs(dj) + abs(dk) > 1:
                                continue
                            a, b, c = i + di, j + dj, k + dk
                            if 0 <= a < nx and 0 <= b < ny and 0 <= c < nz:
                                P[idx(i, j, k), idx(a, b, c)] = True
    return P


def cases():
    out = []
    n = 8
    P = np.eye(n, dtype=bool) | np.eye(n, k=1, dtype=bool) | np.eye(n, k=-1, dtype=bool)
    out.append(("path8", spd_from_pattern(P, 1), list(range(n))))
    n = 6
    P = np.eye(n, dtype=bool)
    P[0, :] = P[:, 0] = True
    A = spd_from_pattern(P, 2)
    out.append(("arrow6-hub-first", A, list(range(n))))
    out.append(("arrow6-hub-last", A, list(range(1, n)) + [0]))
    P = grid_pattern(4, 4, 1, False)
    out.append(("grid5pt-4x4", spd_from_pattern(P, 3), list(range(16))))
    P = grid_pattern(3, 3, 3, True)
    scrambled = [int(v) for v in np.random.default_rng(5).permutation(27)]
    out.append(("grid27-3x3x3-scrambled", spd_from_pattern(P, 4), scrambled))
    P = np.zeros((6, 6), bool)
    P[:3, :3] = True
    P[3:, 3:] = np.eye(3, dtype=bool) | np.eye(3, k=1, dtype=bool) | np.eye(3, k=-1, dtype=bool)
    out.append(("two-blocks", spd_from_pattern(P, 6), [3, 0, 4, 1, 5, 2]))
    out.append(("one", np.array([[2.5]]), [0]))
    return out


def main():
    for name, Ad, perm in cases():
        rowptr, colidx, vals = csr_from_dense(Ad)
        parent0, _ = structure(Ad, np.array(perm))
        post = postorder(parent0)  # analyze() returns perm0 followed by the etree postorder (sparse.mjs:687-696)
        final = [perm[k] for k in post]
        parent, cc = structure(Ad, np.array(final))
        Lden = np.linalg.cholesky(Ad[np.ix_(final, final)])
        rec = {
            "name": name, "n": Ad.shape[0], "rowptr": rowptr, "colidx": colidx, "values": vals, "perm0": perm,
            "perm": final,
            "parent": parent, "colCount": cc, "nnzL": int(sum(cc)), "flops": float(sum(c * c for c in cc)),
            "fingerprint": fnv1a(rowptr, colidx), "L_dense_rowmajor": [float(v) for v in Lden.ravel()],
            "how": "tests/golden/make_golden.py: dense boolean elimination (definition) + numpy Cholesky",
        }
        with open(os.path.join(HERE, f"structure_{name}.json"), "w") as f:
            json.dump(rec, f, indent=None, separators=(",", ":"))
            f.write("\n")


if __name__ == "__main__":
    main()
