"""The solve-heavy caller on the GPU: shift-invert eigenpairs of K x = lambda M x with the Krylov iteration on the
device (amp_eigen_block_arnoldi over amp_shift_invert_apply), against scipy's shift-invert Lanczos (ARPACK with a
sparse LU on the host) as the checker. The eigenpairs are defined by the pencil alone, so they must agree to the
tolerance whatever the Krylov method. Pencils: the Nedelec Maxwell curl-curl / mass pair (indefinite K - sigma M,
LDL^T, the reference's em3d use) and a P1 Laplacian with its consistent mass (sigma below the spectrum, Cholesky)."""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as sla

import ampsolve as A
import eigen as E
import workloads as W

pytestmark = pytest.mark.gpu


class _Pat:
    def __init__(self, n, rowptr, colidx):
        self.n, self.rowptr, self.colidx = n, np.asarray(rowptr, np.int32), np.asarray(colidx, np.int32)

    @property
    def nnz(self):
        return int(self.rowptr[-1])


def p1_laplace_pencil(N):
    """P1 stiffness and consistent mass on N x N cells of the unit square (2 triangles each), Dirichlet boundary."""
    h = 1.0 / N
    nid = lambda i, j: j * (N + 1) + i  # noqa: E731
    tris = []
    for j in range(N):
        for i in range(N):
            a, b, c, d = nid(i, j), nid(i + 1, j), nid(i, j + 1), nid(i + 1, j + 1)
            tris += [(a, b, d), (a, d, c)]
    nn = (N + 1) ** 2
    xy = np.array([[i * h, j * h] for j in range(N + 1) for i in range(N + 1)])
    rows, cols, kv, mv = [], [], [], []
    for t in tris:
        P = xy[list(t)]
        B = np.array([[P[1, 0] - P[0, 0], P[2, 0] - P[0, 0]], [P[1, 1] - P[0, 1], P[2, 1] - P[0, 1]]])
        area = abs(np.linalg.det(B)) / 2
        G = np.linalg.solve(B.T, np.array([[-1.0, 1.0, 0.0], [-1.0, 0.0, 1.0]]))
        Ke = area * G.T @ G
        Me = area / 12 * (np.ones((3, 3)) + np.eye(3))
        for a in range(3):
            for b in range(3):
                rows.append(t[a]); cols.append(t[b]); kv.append(Ke[a, b]); mv.append(Me[a, b])
    Kd = sp.coo_matrix((kv, (rows, cols)), shape=(nn, nn)).toarray()
    Md = sp.coo_matrix((mv, (rows, cols)), shape=(nn, nn)).toarray()
    free = [k for k in range(nn) if 0 < k % (N + 1) < N and 0 < k // (N + 1) < N]
    Kd, Md = Kd[np.ix_(free, free)], Md[np.ix_(free, free)]
    P = sp.csr_matrix(Md > 0)  # the consistent mass couples every pair of nodes of a triangle: the pattern
    P.sort_indices()
    r = np.repeat(np.arange(P.shape[0]), np.diff(P.indptr))
    return _Pat(P.shape[0], P.indptr, P.indices), Kd[r, P.indices].copy(), Md[r, P.indices].copy()


def maxwell_pencil(N):
    w0 = W.maxwell3d(N, 2, 12.0, 0.0, 5, 1)
    w1 = W.maxwell3d(N, 2, 12.0, 1.0, 5, 1)
    return w0.pat, w0.values, w0.values - w1.values  # A(k2) = K - k2 M


def scipy_eigs(pat, K, M, sigma, k):
    Ks = sp.csr_matrix((K, pat.colidx, pat.rowptr), shape=(pat.n, pat.n))
    Ms = sp.csr_matrix((M, pat.colidx, pat.rowptr), shape=(pat.n, pat.n))
    return np.sort(sla.eigsh(Ks, k=k, M=Ms, sigma=sigma, which="LM", tol=1e-13)[0])


@pytest.mark.parametrize("block", [1, 3])
def test_laplace_cholesky_shift_invert(block):
    pat, K, M = p1_laplace_pencil(24)
    r = E.shiftInvertEigen(pat, K, M, sigma=-1.0, nWant=6, kPsd=True, blockSize=block, tol=1e-12)
    assert r["stats"]["factor"] == "cholesky" and r["stats"]["converged"]
    ref = scipy_eigs(pat, K, M, -1.0, 6)
    assert np.max(np.abs(np.sort(r["lambda"]) - ref) / np.abs(ref)) <= 1e-9
    assert np.max(r["residual"]) <= 1e-9
    # the continuous -Laplace eigenvalues of the unit square: 2 pi^2, 5 pi^2 (twice), ... to discretisation accuracy
    assert abs(r["lambda"][0] / (2 * np.pi ** 2) - 1) < 0.02


def test_maxwell_ldlt_shift_invert():
    pat, K, M = maxwell_pencil(8)
    sigma = 30.0
    r = E.shiftInvertEigen(pat, K, M, sigma=sigma, nWant=6, tol=1e-12, maxBasis=48)
    assert r["stats"]["factor"] == "ldlt" and r["stats"]["converged"]
    assert r["stats"]["nNegative"] > 0  # indefinite: the null space (gradients) and the modes below sigma
    ref = scipy_eigs(pat, K, M, sigma, 6)
    got = np.sort(r["lambda"])
    assert np.max(np.abs(got - ref) / np.abs(ref)) <= 1e-9, (got, ref)
    assert np.max(r["residual"]) <= 1e-9


def test_shift_invert_apply_matches_host():
    pat, K, M = p1_laplace_pencil(16)
    sigma = -2.0
    sym = A.analyze(pat)
    num = A.NumericFactor(sym, A.CHOLESKY, A.FP64)
    assert num.factor(K - sigma * M)
    num.set_mass(M)
    X = np.random.default_rng(2).uniform(-1, 1, (3, pat.n))
    Y = num.shift_invert_apply(X)
    As = sp.csr_matrix((K - sigma * M, pat.colidx, pat.rowptr), shape=(pat.n, pat.n)).tocsc()
    Ms = sp.csr_matrix((M, pat.colidx, pat.rowptr), shape=(pat.n, pat.n))
    for k in range(3):
        y = sla.spsolve(As, Ms @ X[k])
        assert np.max(np.abs(Y[k] - y)) <= 1e-12 * np.max(np.abs(y))
