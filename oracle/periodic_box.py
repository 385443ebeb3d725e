"""Assembled-operator oracle for undeformed periodic boxes (test
infrastructure only: the product never imports it).

The reference's Poisson and Helmholtz operators on an undeformed box of
nx x ny x nz equal hexahedra, written with a correct global numbering of
the GLL nodes (periodic images identified) and solved with scipy.
It exists for boxes with one or two elements along a direction, where the
reference's own first-match face pairing (src/init.c:68-130, 298-320) pairs
a face with the neighbour's face on the same side and so solves a different
system: results there are "reference-incorrect" and this oracle, not the
reference, is the check.  On boxes with three or more elements per
direction both agree (tests/test_oracle_pins.py pins it against the
reference there).

Discretisation (the reference's, for affine elements): GLL points and
weights x, w and the 1-D derivative matrix D of n points; per element of
size hx x hy x hz the weak Laplacian (src/poisson.c:34-56 with
G = J^-1 J^-T diagonal)
    A_e = (hy hz / 2 hx) Mz x My x Kx + (hx hz / 2 hy) Mz x Ky x Mx
        + (hx hy / 2 hz) Kz x My x Mx,   K = D^T diag(w) D,  M = diag(w),
and the mass B_e = (hx hy hz / 8) Mz x My x Mx (src/poisson.c:58-66); the
Helmholtz operator is A + lambda B (src/helmholtz.c:33-49, svva = 0).  The
assembled system is solved by Jacobi-preconditioned CG to a relative
residual of 1e-14.  Local
index (k, j, i) with i fastest, element e = ex + nx (ey + ny ez), as
ssenss_b200.mesh.box_mesh numbers them.
"""
import math

import numpy as np


def gll(n):
    """GLL points, weights and derivative matrix D[i, j] = l_j'(x_i) of n
    points (Newton on the Legendre polynomial; the published formulas)."""
    N = n - 1
    x = -np.cos(np.pi * np.arange(n) / N)
    for _ in range(100):
        P = np.zeros((n, n))
        P[:, 0] = 1.0
        P[:, 1] = x
        for k in range(2, n):
            P[:, k] = ((2 * k - 1) * x * P[:, k - 1] - (k - 1) * P[:, k - 2]) / k
        dx = (x * P[:, N] - P[:, N - 1]) / (n * P[:, N])
        x = x - dx
        if np.max(np.abs(dx)) < 1e-16:
            break
    P = np.zeros((n, n))
    P[:, 0] = 1.0
    P[:, 1] = x
    for k in range(2, n):
        P[:, k] = ((2 * k - 1) * x * P[:, k - 1] - (k - 1) * P[:, k - 2]) / k
    LN = P[:, N]
    w = 2.0 / (N * n * LN ** 2)
    D = np.zeros((n, n))
    for i in range(n):
        for j in range(n):
            if i != j:
                D[i, j] = LN[i] / LN[j] / (x[i] - x[j])
    D[0, 0] = -N * n / 4.0
    D[N, N] = N * n / 4.0
    return x, w, D


def global_ids(shape, n):
    """Global node id of every local node, (nel, n, n, n), periodic images
    identified."""
    nx, ny, nz = shape
    m = n - 1
    e = np.arange(nx * ny * nz)
    ex, ey, ez = e % nx, (e // nx) % ny, e // (nx * ny)
    ar = np.arange(n)
    gx = (ex[:, None, None, None] * m + ar[None, None, None, :]) % (nx * m)
    gy = (ey[:, None, None, None] * m + ar[None, None, :, None]) % (ny * m)
    gz = (ez[:, None, None, None] * m + ar[None, :, None, None]) % (nz * m)
    return gx + nx * m * (gy + ny * m * gz)


def assembled_operator(shape, n, lam=0.0, length=2 * math.pi):
    """Assembled A + lam B (scipy CSR) and the global ids of the local
    nodes."""
    import scipy.sparse as sp
    nx, ny, nz = shape
    hx, hy, hz = length / nx, length / ny, length / nz
    _, w, D = gll(n)
    K = sp.csr_matrix(D.T @ np.diag(w) @ D)
    M = sp.diags(w)
    kron = lambda a, b, c: sp.kron(a, sp.kron(b, c))   # noqa: E731  (k, j, i) order
    Ae = (hy * hz / (2 * hx)) * kron(M, M, K) + (hx * hz / (2 * hy)) * kron(M, K, M) + \
        (hx * hy / (2 * hz)) * kron(K, M, M)
    if lam:
        Ae = Ae + lam * (hx * hy * hz / 8.0) * kron(M, M, M)
    Ae = sp.coo_matrix(Ae)
    gid = global_ids(shape, n).reshape(nx * ny * nz, -1)
    ndof = int(gid.max()) + 1
    rows = gid[:, Ae.row].ravel()
    cols = gid[:, Ae.col].ravel()
    vals = np.tile(Ae.data, gid.shape[0])
    A = sp.coo_matrix((vals, (rows, cols)), shape=(ndof, ndof)).tocsr()
    return A, gid


def solve(shape, n, f_local, lam=0.0, length=2 * math.pi):
    """Solution (local layout) of the assembled system for the assembled
    weak right-hand side f_local (nel, n, n, n): every local copy of a node
    holds the node's value.  Poisson (lam = 0, singular on a periodic box):
    the solution with zero mean over the nodes."""
    import scipy.sparse as sp
    import scipy.sparse.linalg as spla
    A, gid = assembled_operator(shape, n, lam, length)
    ndof = A.shape[0]
    f = np.zeros(ndof)
    f[gid.ravel()] = np.asarray(f_local).reshape(gid.shape).ravel()
    if not lam:
        # periodic Poisson: project f onto the range (the constants span the
        # null space of the symmetric A), solve, keep the zero-mean solution
        f = f - f.mean()
    # Jacobi-preconditioned CG to a relative residual of 1e-14 (the
    # assembled system is SPD, or SPD on the zero-mean subspace)
    dinv = 1.0 / A.diagonal()
    Mj = spla.LinearOperator(A.shape, matvec=lambda v: dinv * v)
    u, info = spla.cg(A, f, rtol=1e-14, atol=0.0, maxiter=100000, M=Mj)
    if info != 0:
        raise RuntimeError(f"assembled CG did not converge ({info})")
    if not lam:
        u -= u.mean()
    return u[gid].reshape(np.shape(f_local))
