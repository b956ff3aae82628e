"""amp_front_factor_noalloc: the entry point for callers that cannot allocate device memory.

Applications that give all device memory to their own pool at start-up, or that must not let a cudaMalloc stall
their other streams, factor a front they own through this entry point; its scratch is a static device array. This
test calls it through the C ABI and checks its factor against the regular entry point's (amp_factor_numeric on the
same dense SPD matrix, whose analysis is one supernode holding the whole front), on two calls in a row: the second
call reuses the scratch the first one left behind. Collected last (file name) so that a failure here leaves every
other test already run.
"""
import ctypes as C

import numpy as np
import pytest

import ampsolve as amp
import workloads as wl

pytestmark = pytest.mark.gpu

TOL = 1e-12  # the FP64 parity bar of the other GPU tests


def _dense_spd(n, seed):
    rng = np.random.default_rng(seed)
    M = rng.uniform(-1, 1, (n, n))
    return M @ M.T + n * np.eye(n)


def _noalloc(F_dev_ptr, m, nc, stream=None):
    fn = amp.lib().amp_front_factor_noalloc
    fn.restype = C.c_int
    fn.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.c_void_p, C.POINTER(C.c_int32)]
    fail = C.c_int32(-2)
    code = fn(C.c_void_p(F_dev_ptr), m, nc, None if stream is None else C.c_void_p(stream), C.byref(fail))
    return code, fail.value


def test_noalloc_front_matches_regular_factor_twice():
    torch = pytest.importorskip("torch")
    n = 300
    rp = np.arange(0, n * n + 1, n, dtype=np.int32)
    ci = np.tile(np.arange(n, dtype=np.int32), n)
    pat = wl.CsrPattern(n, rp, ci)
    sym = amp.analyze(pat)
    assert sym.nsuper == 1 and sym.maxFront == n
    perm = sym.perm
    for call, seed in enumerate((11, 12)):
        A = _dense_spd(n, seed)
        num = amp.factorNumeric(sym, A.reshape(-1).copy())  # regular entry point (allocates its factor)
        assert num.ok
        Lref = num.Lx.reshape(n, n).T  # column-major m x nc block of the single supernode
        Ap = A[np.ix_(perm, perm)]
        F = torch.from_numpy(np.asfortranarray(Ap).T.copy().reshape(-1)).cuda()  # column-major, ld = n
        torch.cuda.synchronize()
        code, fail = _noalloc(F.data_ptr(), n, n)
        assert code == amp.AMP_OK, amp.lib().amp_last_error()
        assert fail == -1
        Lna = F.cpu().numpy().reshape(n, n).T
        low = np.tril(np.ones((n, n), bool))
        err = np.max(np.abs(Lna[low] - Lref[low])) / np.max(np.abs(Lref[low]))
        assert err <= TOL, (call, err)


def test_noalloc_partial_front_schur_and_failure():
    torch = pytest.importorskip("torch")
    m, nc = 200, 70
    A = _dense_spd(m, 3)
    F = torch.from_numpy(A.T.copy().reshape(-1)).cuda()
    code, fail = _noalloc(F.data_ptr(), m, nc)
    assert code == amp.AMP_OK and fail == -1
    R = F.cpu().numpy().reshape(m, m).T
    L11 = np.linalg.cholesky(A[:nc, :nc])
    L21 = np.linalg.solve(L11, A[:nc, nc:]).T
    S = A[nc:, nc:] - L21 @ L21.T
    low = np.tril(np.ones((m - nc, m - nc), bool))
    assert np.max(np.abs(np.tril(R[:nc, :nc]) - L11)) <= 1e-12 * np.max(np.abs(L11))
    assert np.max(np.abs(R[nc:, :nc] - L21)) <= 1e-12 * np.max(np.abs(L21))
    assert np.max(np.abs(R[nc:, nc:][low] - S[low])) <= 1e-12 * np.max(np.abs(S))
    # an indefinite front reports its first non-positive pivot
    B = -np.eye(64)
    Fb = torch.from_numpy(B.copy().reshape(-1)).cuda()
    code, fail = _noalloc(Fb.data_ptr(), 64, 64)
    assert code == amp.AMP_OK and fail == 0


@pytest.mark.parametrize("m,nc", [(1024, 512), (1100, 640)])
def test_noalloc_on_a_stream_multi_chunk(m, nc):
    """A caller's own stream, several 256-row panel chunks per pivot block (the last-reader counter with more than
    two readers), nc a multiple of 64 and not, two calls in a row against numpy's Cholesky and Schur complement."""
    torch = pytest.importorskip("torch")
    st = torch.cuda.Stream()
    for seed in (21, 22):
        A = _dense_spd(m, seed)
        with torch.cuda.stream(st):
            F = torch.from_numpy(A.T.copy().reshape(-1)).to("cuda", non_blocking=False)
        st.synchronize()
        code, fail = _noalloc(F.data_ptr(), m, nc, stream=st.cuda_stream)
        assert code == amp.AMP_OK and fail == -1, amp.lib().amp_last_error()
        R = F.cpu().numpy().reshape(m, m).T
        L11 = np.linalg.cholesky(A[:nc, :nc])
        L21 = np.linalg.solve(L11, A[:nc, nc:]).T
        S = A[nc:, nc:] - L21 @ L21.T
        low = np.tril(np.ones((m - nc, m - nc), bool))
        assert np.max(np.abs(np.tril(R[:nc, :nc]) - L11)) <= TOL * np.max(np.abs(L11))
        assert np.max(np.abs(R[nc:, :nc] - L21)) <= TOL * np.max(np.abs(L21))
        assert np.max(np.abs(R[nc:, nc:][low] - S[low])) <= TOL * np.max(np.abs(S))


def test_noalloc_rejects_oversized_front():
    torch = pytest.importorskip("torch")
    F = torch.zeros(4, dtype=torch.float64, device="cuda")
    code, _ = _noalloc(F.data_ptr(), 16385, 16)
    assert code == amp.AMP_INVALID
    assert "exceeds the maximum" in amp.lib().amp_last_error().decode()


def test_noalloc_on_every_device():
    # the per-device set-up (scratch address, kernel attributes): a front factored on each visible GPU in turn, the
    # calling thread's current device being the front's; skipped with one GPU
    torch = pytest.importorskip("torch")
    ndev = torch.cuda.device_count()
    if ndev < 2:
        pytest.skip("one GPU: the second device's set-up is not reachable")
    m = nc = 200
    A = _dense_spd(m, 5)
    L = np.linalg.cholesky(A)
    low = np.tril(np.ones((m, m), bool))
    for dev in range(ndev):
        with torch.cuda.device(dev):
            F = torch.from_numpy(np.asfortranarray(A).T.copy().reshape(-1)).to(f"cuda:{dev}")
            torch.cuda.synchronize()
            code, fail = _noalloc(F.data_ptr(), m, nc)
            assert code == amp.AMP_OK, (dev, amp.lib().amp_last_error())
            assert fail == -1
            R = F.cpu().numpy().reshape(m, m).T
        assert np.max(np.abs(R[low] - L[low])) <= TOL * np.max(np.abs(L)), dev
