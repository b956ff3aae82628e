"""Writes tests/golden/ordering_*.json: the orderings and supernode structures of small patterns as the reference's
JavaScript computes them, derived with js_transcription.py (a statement-by-statement Python transcription of
amdOrder, ndOrder, nd3Order and analyze from sparse.mjs / order3d.mjs). The path of 8 was also traced by hand through
amdOrder (tests/test_ordering_golden.py gives the trace). Run from the repository root:

    python tests/golden/make_ordering_golden.py
"""
from __future__ import annotations

import json
import os
import random
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

import js_transcription as js  # noqa: E402


def csr(n, edges):
    adj = [set([i]) for i in range(n)]
    for a, b in edges:
        adj[a].add(b)
        adj[b].add(a)
    rowptr, colidx = [0], []
    for i in range(n):
        colidx.extend(sorted(adj[i]))
        rowptr.append(len(colidx))
    return {"n": n, "rowptr": rowptr, "colidx": colidx}


def grid2d(nx, ny):
    idx = lambda i, j: j * nx + i  # noqa: E731
    e = []
    for j in range(ny):
        for i in range(nx):
            if i + 1 < nx:
                e.append((idx(i, j), idx(i + 1, j)))
            if j + 1 < ny:
                e.append((idx(i, j), idx(i, j + 1)))
    x = [float(i) / (nx - 1) for j in range(ny) for i in range(nx)]
    y = [float(j) / (ny - 1) for j in range(ny) for i in range(nx)]
    return csr(nx * ny, e), x, y


def grid27(N, dofs=1):
    """27-point stencil on N^3 nodes (coordinates i / (N - 1)), `dofs` unknowns per node sharing its coordinates."""
    nodes = [(i, j, k) for k in range(N) for j in range(N) for i in range(N)]
    nid = {p: t for t, p in enumerate(nodes)}
    e = []
    for (i, j, k), a in nid.items():
        for di in (-1, 0, 1):
            for dj in (-1, 0, 1):
                for dk in (-1, 0, 1):
                    b = nid.get((i + di, j + dj, k + dk))
                    if b is None or b < a:
                        continue
                    for c1 in range(dofs):
                        for c2 in range(dofs):
                            u, v = a * dofs + c1, b * dofs + c2
                            if u != v:
                                e.append((u, v))
    n = len(nodes) * dofs
    xs = [nodes[t // dofs][0] / (N - 1) for t in range(n)]
    ys = [nodes[t // dofs][1] / (N - 1) for t in range(n)]
    zs = [nodes[t // dofs][2] / (N - 1) for t in range(n)]
    return csr(n, e), xs, ys, zs


def random_with_dense_row(n=40, seed=7):
    """Random edges, one row joined to every other (above amdOrder's dense threshold min(n - 2, max(16, 10 sqrt n)))
    and one isolated row (degree 0)."""
    rnd = random.Random(seed)
    e = set()
    while len(e) < 3 * n:
        a, b = rnd.randrange(n - 1), rnd.randrange(n - 1)
        if a != b and a != 5 and b != 5:
            e.add((min(a, b), max(a, b)))
    hub = n - 1
    e |= {(i, hub) for i in range(n - 1) if i != 5}
    return csr(n, sorted(e))


def cases():
    out = []
    out.append(("path8-amd", csr(8, [(i, i + 1) for i in range(7)]), "amd", {}))
    g, x, y = grid2d(4, 4)
    out.append(("grid5pt-4x4-amd", g, "amd", {}))
    g, x, y = grid2d(6, 6)
    out.append(("grid5pt-6x6-nd-leaf4", g, "nd", {"x": x, "y": y, "leaf": 4}))
    out.append(("arrow6-hub-first-amd", csr(6, [(0, i) for i in range(1, 6)]), "amd", {}))
    out.append(("arrow6-hub-last-amd", csr(6, [(i, 5) for i in range(5)]), "amd", {}))
    g, x, y, z = grid27(3)
    out.append(("grid27-3x3x3-nd3-leaf4", g, "nd3", {"x": x, "y": y, "z": z, "leaf": 4}))
    g, x, y, z = grid27(4, dofs=3)
    out.append(("grid27-4x4x4-3dof-nd3-leaf20", g, "nd3", {"x": x, "y": y, "z": z, "leaf": 20}))
    out.append(("random40-dense-row-amd", random_with_dense_row(), "amd", {}))
    g, x, y = grid2d(9, 7)
    out.append(("grid5pt-9x7-amd", g, "amd", {}))
    return out


def main():
    for name, pat, ordering, o in cases():
        if ordering == "amd":
            perm0 = js.amdOrder(pat)
        elif ordering == "nd":
            perm0 = js.ndOrder(pat, o["x"], o["y"], o["leaf"])
        else:
            perm0 = js.nd3Order(pat, o["x"], o["y"], o["z"], o["leaf"])
        a = js.analyze(pat, perm=perm0)
        doc = {"name": name, "how": "js_transcription.py (line-by-line transcription of sparse.mjs / order3d.mjs)",
               "ordering": ordering, "params": {k: v for k, v in o.items() if k == "leaf"},
               "n": pat["n"], "rowptr": pat["rowptr"], "colidx": pat["colidx"],
               "coords": {k: o[k] for k in ("x", "y", "z") if k in o}, "order": perm0, **a}
        with open(os.path.join(HERE, f"ordering_{name}.json"), "w") as f:
            json.dump(doc, f, separators=(",", ":"))
        print(name, "n", pat["n"], "nsuper", len(a["superStart"]) - 1, "perm", perm0[:12])


if __name__ == "__main__":
    main()
