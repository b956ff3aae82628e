"""k^2 of the driven Maxwell system: midway between the 10th and 11th nonzero eigenvalues of the curl-curl pencil.

A(k2) = K - k2 M (lowest-order Nedelec edges, PEC boundary; workloads.maxwell3d). The inertia of A(sigma) counts the
eigenvalues of (K, M) below sigma (Sylvester). The gradients of the (N - 1)^3 interior nodes span K's null space, so
for sigma > 0

    nNeg(K - sigma M) = (N - 1)^3 + #{nonzero eigenvalues < sigma}.

Bisection on that count with the GPU LDL^T gives lambda_10 and lambda_11; k2 is their midpoint. Run on a GPU:

    python tests/golden/maxwell_k2.py 32

This is the recipe of the stored constant workloads.MAXWELL_K2_32; nothing imports it.
"""
from __future__ import annotations

import os
import sys

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "..", "..", "applied-multiphysics_b200"))

import ampsolve as amp  # noqa: E402
import workloads as wl  # noqa: E402


def inertia_counter(N: int, nbox: int = 8, eps_in: float = 12.0, seed: int = 5):
    w0 = wl.maxwell3d(N, nbox, eps_in, 0.0, seed, 1)
    w1 = wl.maxwell3d(N, nbox, eps_in, 1.0, seed, 1)
    K, M = w0.values, w0.values - w1.values  # A(k2) = K - k2 M, linear in k2
    sym = amp.analyze(w0.pat, ordering="nd3", x=w0.x, y=w0.y, z=w0.z)
    f = amp.SupernodalLDLT(sym)
    null_dim = (N - 1) ** 3

    def count(sigma: float) -> int:
        r = f.factor(K - sigma * M)
        if not r["ok"]:
            raise RuntimeError(f"LDL^T failed at sigma = {sigma}")
        return r["nNeg"] - null_dim

    return count, null_dim, w0.n


def bisect_eigenvalue(count, k: int, lo: float, hi: float, rel: float = 1e-10) -> float:
    """Smallest sigma with count(sigma) >= k, to relative precision rel, given count(lo) < k <= count(hi)."""
    while hi - lo > rel * hi:
        mid = 0.5 * (lo + hi)
        if count(mid) >= k:
            hi = mid
        else:
            lo = mid
    return 0.5 * (lo + hi)


def k2_between(N: int, i: int = 10) -> tuple[float, float, float]:
    count, null_dim, n = inertia_counter(N)
    lo = 1e-8
    c0 = count(lo)
    if c0 != 0:
        raise RuntimeError(f"count at sigma = {lo} is {c0}, expected 0 (null space {null_dim} of n = {n})")
    hi = 1.0
    while count(hi) < i + 1:
        hi *= 2.0
    li = bisect_eigenvalue(count, i, lo, hi)
    lj = bisect_eigenvalue(count, i + 1, li, hi)
    return 0.5 * (li + lj), li, lj


if __name__ == "__main__":
    N = int(sys.argv[1]) if len(sys.argv) > 1 else 32
    k2, l10, l11 = k2_between(N)
    print(f"N={N} lambda10={l10!r} lambda11={l11!r} k2={k2!r}")
