"""Shift-invert eigen solver for the symmetric pencil K x = lambda M x on the GPU factor: the solve-heavy caller of
the sparse direct solver (the reference's shiftInvertEigen, packages/physics/src/common/eigen.ts:116-230).

K - sigma M is factored once on the device (Cholesky when the caller states that it is positive definite and sigma
is below the spectrum, else LDL^T, whose negative pivots give the inertia), and the Krylov iteration runs on the
device too: every block of the basis is one operator application op(X) = (K - sigma M)^-1 M X (SpMV with M plus one
multi-vector solve), orthogonalised against the basis in device memory (amp_eigen_block_arnoldi); only the small
projected matrix crosses to the host. Ritz values mu of largest modulus give lambda = sigma + 1 / mu. The Ritz
vectors are then refined as the reference does (eigen.ts:190-222): one more operator application, Rayleigh
quotients, M-orthonormalisation within clusters of equal eigenvalues, and the relative residuals
||K x - lambda M x|| / (||K x|| + |lambda| ||M x||).

Differences from the reference: the Krylov basis is M-orthonormal (the operator is self-adjoint in the M inner
product), so the projected matrix is symmetric and the iteration is block Lanczos with full reorthogonalisation and
thick restart; the reference's blockArnoldi (la/arnoldi.mjs) orthogonalises in the Euclidean inner product with a
general Hessenberg matrix. Both find the same eigenpairs. The projector hook, the iterative-solver path and the
inertia completeness check of the reference are not part of this device path.
"""
from __future__ import annotations

import time

import numpy as np

import ampsolve as amp


def shiftInvertEigen(pat, K, M, sigma: float, nWant: int, tol: float = 1e-10, blockSize: int = 1,
                     maxBasis: int | None = None, maxRestarts: int = 60, seed: int = 20261106, factor: str = "auto",
                     kPsd: bool = False, sym=None, attempts: int = 3) -> dict:
    """Eigenpairs of K x = lambda M x nearest sigma (EigenInput / EigenResult of eigen.ts:14-106).

    The explicit relative residuals of the refined pairs are checked against max(1e3 tol, 1e-9): a run whose Krylov
    iteration reported convergence with a pair above that bound (seen intermittently on an indefinite Maxwell pencil,
    cause not found) is repeated, factorization included, with the next seed, up to `attempts` runs; the result with
    the smallest worst residual is returned, and stats["attempts"] counts the runs."""
    best = None
    for a in range(max(1, attempts)):
        r = _shift_invert_once(pat, K, M, sigma, nWant, tol, blockSize, maxBasis, maxRestarts, seed + a, factor, kPsd,
                               sym)
        worst = float(np.max(r["residual"])) if len(r["residual"]) else 0.0
        if best is None or worst < best[0]:
            best = (worst, r)
        if r["stats"]["converged"] and worst <= max(1e3 * tol, 1e-9):
            break
    r = best[1]
    r["stats"]["attempts"] = a + 1
    return r


def _shift_invert_once(pat, K, M, sigma, nWant, tol, blockSize, maxBasis, maxRestarts, seed, factor, kPsd, sym):
    K = np.ascontiguousarray(K, np.float64)
    M = np.ascontiguousarray(M, np.float64)
    n = int(pat.n)
    A = K - sigma * M
    kind = "cholesky" if factor == "cholesky" or (factor != "ldlt" and sigma < 0 and kPsd) else "ldlt"
    sym = sym if sym is not None else amp.analyze(pat)
    t0 = time.perf_counter()
    num = amp.NumericFactor(sym, amp.CHOLESKY if kind == "cholesky" else amp.LDLT, amp.FP64)
    ok = num.factor(A)
    if not ok:
        raise RuntimeError("eigen: K - sigma M is not positive definite (sigma not below the spectrum?)"
                           if kind == "cholesky" else "eigen: LDL^T of K - sigma M failed (sigma on an eigenvalue?)")
    factorMs = (time.perf_counter() - t0) * 1e3
    num.set_mass(M)
    t1 = time.perf_counter()
    mb = maxBasis if maxBasis is not None else max(30, 2 * nWant + 12)
    mu, ritz, st = num.block_arnoldi(nWant, blockSize=blockSize, maxBasis=mb, tol=tol, maxRestarts=maxRestarts,
                                     seed=seed)
    arnoldiMs = (time.perf_counter() - t1) * 1e3
    # refine: one inverse-iteration step, Rayleigh quotients, M-orthonormalise clusters (eigen.ts:190-222)
    t2 = time.perf_counter()
    vecs = num.shift_invert_apply(ritz).reshape(len(mu), n)
    KX = amp.matVec(pat, K, vecs).reshape(len(mu), n)
    MX = amp.matVec(pat, M, vecs).reshape(len(mu), n)
    lam = np.einsum("ij,ij->i", vecs, KX) / np.einsum("ij,ij->i", vecs, MX)
    order = sorted(range(len(lam)), key=lambda i: lam[i])
    vecs, lam = vecs[order], lam[order]
    done = []
    for i in range(len(vecs)):
        x = vecs[i].copy()
        for j in range(i):
            if abs(lam[j] - lam[i]) > 1e-6 * max(abs(lam[i]), 1e-300):
                continue
            y = done[j]
            x -= float(np.dot(x, amp.matVec(pat, M, y))) * y
        x /= np.sqrt(float(np.dot(x, amp.matVec(pat, M, x))))
        done.append(x)
    X = np.array(done) if done else np.zeros((0, n))
    KX = amp.matVec(pat, K, X).reshape(len(done), n) if done else X
    MX = amp.matVec(pat, M, X).reshape(len(done), n) if done else X
    lam = np.einsum("ij,ij->i", X, KX) / np.einsum("ij,ij->i", X, MX) if done else np.zeros(0)
    res = np.array([np.linalg.norm(KX[i] - lam[i] * MX[i]) /
                    ((np.linalg.norm(KX[i]) + abs(lam[i]) * np.linalg.norm(MX[i])) or 1.0) for i in range(len(done))])
    refineMs = (time.perf_counter() - t2) * 1e3
    return {"lambda": lam, "vecs": list(X), "residual": res, "mu": mu,
            "stats": {"n": n, "nnz": int(pat.rowptr[n]), "factor": kind, "nnzL": sym.nnzL,
                      "nNegative": num.nNeg if kind == "ldlt" else 0, "nPerturbed": num.nPerturbed,
                      "factorMs": factorMs, "arnoldiMs": arnoldiMs, "refineMs": refineMs,
                      "opApplications": st["opVectors"] + len(mu), "restarts": st["restarts"],
                      "converged": st["converged"], "ritzResidual": st["maxResidual"]}}
