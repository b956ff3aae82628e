"""Seeded synthetic FEM systems (ctypes over libampwork.so, built from csrc/workloads.cpp).

Each generator returns a :class:`Workload` with the CSR pattern (full symmetric storage, sorted rows, diagonal present),
the FP64 values aligned with it, DOF coordinates (for the nested-dissection orderings) and right-hand sides.
The five benchmark systems follow the shapes of the reference's own assembly code; see csrc/workloads.cpp.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "libampwork.so")
_lib = None


class _W(C.Structure):
    _fields_ = [("n", C.c_int), ("nnz", C.c_int64), ("rowptr", C.POINTER(C.c_int)), ("colidx", C.POINTER(C.c_int)),
                ("values", C.POINTER(C.c_double)), ("x", C.POINTER(C.c_double)), ("y", C.POINTER(C.c_double)),
                ("z", C.POINTER(C.c_double)), ("nrhs", C.c_int), ("rhs", C.POINTER(C.c_double))]


@dataclass
class CsrPattern:
    """Symmetric CSR pattern, full storage (both triangles, diagonal present), rows sorted ascending."""
    n: int
    rowptr: np.ndarray
    colidx: np.ndarray

    @property
    def nnz(self) -> int:
        return int(self.rowptr[self.n])


@dataclass
class Workload:
    name: str
    pat: CsrPattern
    values: np.ndarray
    x: np.ndarray | None
    y: np.ndarray | None
    z: np.ndarray | None
    rhs: np.ndarray  # shape (nrhs, n)

    @property
    def n(self) -> int:
        return self.pat.n


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB):
            raise RuntimeError(f"{_LIB} is missing: run __graft_entry__.build() first")
        L = C.CDLL(_LIB)
        for name, args in [("amp_wl_poisson2d", [C.c_int, C.c_uint32]),
                           ("amp_wl_heat2d_lognormal", [C.c_int, C.c_uint32, C.c_int]),
                           ("amp_wl_elastic3d", [C.c_int, C.c_double, C.c_double, C.c_uint32, C.c_int]),
                           ("amp_wl_heat3d_p2", [C.c_int, C.c_int, C.c_double, C.c_uint32, C.c_int]),
                           ("amp_wl_maxwell3d", [C.c_int, C.c_int, C.c_double, C.c_double, C.c_uint32, C.c_int]),
                           ("amp_wl_grid27", [C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, C.c_int]),
                           ("amp_wl_hex_q1", [C.c_int, C.c_int, C.c_int]),
                           ("amp_wl_chain", [C.c_int, C.c_double, C.c_double])]:
            f = getattr(L, name)
            f.argtypes = args
            f.restype = C.POINTER(_W)
        L.amp_wl_free.argtypes = [C.POINTER(_W)]
        _lib = L
    return _lib


def _take(name: str, wp) -> Workload:
    w = wp.contents
    n, nnz = w.n, int(w.nnz)

    def arr(p, ln, dt):
        if not p or ln == 0:
            return np.zeros(ln, dt)
        return np.ctypeslib.as_array(p, shape=(ln,)).astype(dt, copy=True)

    pat = CsrPattern(n, arr(w.rowptr, n + 1, np.int32), arr(w.colidx, nnz, np.int32))
    vals = arr(w.values, nnz, np.float64)
    x = arr(w.x, n, np.float64) if w.x else None
    y = arr(w.y, n, np.float64) if w.y else None
    z = arr(w.z, n, np.float64) if w.z else None
    rhs = arr(w.rhs, w.nrhs * n, np.float64).reshape(w.nrhs, n) if w.nrhs else np.zeros((0, n))
    lib().amp_wl_free(wp)
    return Workload(name, pat, vals, x, y, z, rhs)


def poisson2d(N: int = 64, seed: int = 1) -> Workload:
    """2D P1 Poisson on the unit square, N x N cells x 2 triangles, Dirichlet; RHS f = 1 and seeded U(-1,1)."""
    return _take(f"poisson2d-{N}", lib().amp_wl_poisson2d(N, seed))


def heat2d_lognormal(N: int, seed: int, q: int) -> Workload:
    """One member of the batched 2D heat set: lognormal(0,1) conductivity per triangle, q seeded RHS."""
    return _take(f"heat2d-{N}", lib().amp_wl_heat2d_lognormal(N, seed, q))


def elastic3d(N: int = 40, E: float = 1.0, nu: float = 0.3, seed: int = 2, q: int = 1) -> Workload:
    """3D P1 linear elasticity on N^3 hexes x 6 Kuhn tets, x = 0 face clamped, seeded U(-1,1) body load."""
    return _take(f"elastic3d-{N}", lib().amp_wl_elastic3d(N, E, nu, seed, q))


def heat3d_p2(N: int = 48, nsph: int = 64, radius: float = 0.05, seed: int = 4, q: int = 16) -> Workload:
    """3D P2 (tet10) heat, k = 100 in seeded spheres else 1, Dirichlet on x = 0 and x = 1."""
    return _take(f"heat3d-p2-{N}", lib().amp_wl_heat3d_p2(N, nsph, radius, seed, q))


# k^2 of the 32^3 driven Maxwell system: midway between its 10th (34.3115) and 11th (36.2170) nonzero eigenvalues,
# found by inertia bisection with the GPU LDL^T (tests/golden/maxwell_k2.py 32, on a B200).
MAXWELL_K2_32 = 35.2642118891234


def maxwell3d(N: int = 32, nbox: int = 8, eps_in: float = 12.0, k2: float | None = None, seed: int = 5,
              q: int = 64) -> Workload:
    """Lowest-order Nedelec curl-curl - k2 eps_r mass on N^3 hexes x 6 tets, PEC boundary, port-like RHS.
    k2 defaults to MAXWELL_K2_32 for N = 32 (indefinite: 10 eigenvalues below it besides the gradient null space)."""
    if k2 is None:
        k2 = MAXWELL_K2_32 if N == 32 else 0.0
    return _take(f"maxwell3d-{N}", lib().amp_wl_maxwell3d(N, nbox, eps_in, k2, seed, q))


def grid27(Nx: int, Ny: int, Nz: int, zero_every: int = 0, shift: float = 0.0, sym: bool = False) -> Workload:
    """27-point grid fixture of the reference's WASM front / solve tests."""
    return _take("grid27", lib().amp_wl_grid27(Nx, Ny, Nz, zero_every, shift, 1 if sym else 0))


def hex_q1(nx: int = 6, ny: int = 5, nz: int = 4) -> Workload:
    """Graded Q1 hex Laplacian of the reference's la-sparse tests (x = 0 face fixed)."""
    return _take("hex-q1", lib().amp_wl_hex_q1(nx, ny, nz))


def chain(n: int, diag: float = 2.0, off: float = -1.0) -> Workload:
    """1D chain tridiag(off, diag, off) of the reference's core-solvers tests."""
    return _take("chain", lib().amp_wl_chain(n, diag, off))


def heat2d_batch_sizes(count: int = 256, seed: int = 3) -> list[tuple[int, int]]:
    """(N, q) of the batched 2D heat set: N ~ U{16..128} cells per side, q ~ U{1..64} right-hand sides, from the
    uint32 LCG s = s * 1664525 + 1013904223."""
    s = seed & 0xFFFFFFFF
    out = []
    for _ in range(count):
        s = (s * 1664525 + 1013904223) & 0xFFFFFFFF
        N = 16 + (s >> 8) % 113
        s = (s * 1664525 + 1013904223) & 0xFFFFFFFF
        q = 1 + (s >> 8) % 64
        out.append((int(N), int(q)))
    return out


def heat2d_batch(count: int = 256, seed: int = 3) -> list[Workload]:
    """The batched 2D heat set: `count` lognormal-conductivity P1 problems of uneven size with q_i seeded RHS each."""
    return [heat2d_lognormal(N, seed * 1000 + i, q) for i, (N, q) in enumerate(heat2d_batch_sizes(count, seed))]


@dataclass
class Mesh:
    """The mesh behind a workload (inputs of on-device assembly): node coordinates (nnodes, dim), connectivity
    (nelem, k), DOF map (nnodes * bs, -1 for Dirichlet DOFs) and per-element coefficients."""
    kind: int
    coords: np.ndarray
    conn: np.ndarray
    dofs: np.ndarray
    coef: np.ndarray


def mesh(kind: int, N: int, seed: int = 0, E: float = 1.0, nu: float = 0.3) -> Mesh:
    """kind 0: the triangles of heat2d_lognormal(N, seed) (seed 0: conductivity 1, the Poisson system); kind 1: the
    tets of elastic3d(N, E, nu) (3 DOFs per node, x = 0 clamped, (E, nu) per tet)."""
    L = lib()
    f = L.amp_wl_mesh
    f.restype = C.c_int
    f.argtypes = [C.c_int, C.c_int, C.c_uint32, C.c_double, C.c_double, C.POINTER(C.c_int), C.POINTER(C.c_int),
                  C.POINTER(C.POINTER(C.c_double)), C.POINTER(C.c_int64), C.POINTER(C.c_int),
                  C.POINTER(C.POINTER(C.c_int)), C.POINTER(C.c_int), C.POINTER(C.POINTER(C.c_int)),
                  C.POINTER(C.POINTER(C.c_double)), C.POINTER(C.c_int)]
    L.amp_wl_free_array.argtypes = [C.c_void_p]
    nn, dim, k, bs, nco = C.c_int(), C.c_int(), C.c_int(), C.c_int(), C.c_int()
    ne = C.c_int64()
    xy, cf = C.POINTER(C.c_double)(), C.POINTER(C.c_double)()
    cn, dm = C.POINTER(C.c_int)(), C.POINTER(C.c_int)()
    if f(kind, N, seed, E, nu, C.byref(nn), C.byref(dim), C.byref(xy), C.byref(ne), C.byref(k), C.byref(cn),
         C.byref(bs), C.byref(dm), C.byref(cf), C.byref(nco)) != 0:
        raise ValueError(f"unknown mesh kind {kind}")

    def take(p, ln, dt):
        a = np.ctypeslib.as_array(p, shape=(ln,)).astype(dt, copy=True)
        L.amp_wl_free_array(C.cast(p, C.c_void_p))
        return a

    coords = take(xy, nn.value * dim.value, np.float64).reshape(nn.value, dim.value)
    conn = take(cn, ne.value * k.value, np.int32).reshape(ne.value, k.value)
    dofs = take(dm, nn.value * bs.value, np.int32)
    coef = take(cf, nco.value, np.float64)
    return Mesh(kind, coords, conn, dofs, coef)
