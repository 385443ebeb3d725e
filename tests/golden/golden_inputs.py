"""Inputs of the golden fixtures, rebuilt bit for bit from integers on any
machine (integer hashing and IEEE +, -, *, / only; no libm calls, whose
last bit may depend on the CPU's vector extensions).

Used by make_golden.py (which runs the reference) and by the tests that
compare against its output.
"""
from __future__ import annotations

import numpy as np

from ssenss_b200.mesh import channel_mesh, tgv_box

CASES = {
    # name: (mesh builder, order n)
    "tgv3_n6": (lambda: tgv_box(3), 6),
    "channel433_n5": (lambda: channel_mesh((4, 3, 3), seed=7), 5),
    # the benchmark's order: the FP64 tensor-core operator and the n = 4 /
    # n = 2 cooperative levels
    "tgv3_n8": (lambda: tgv_box(3), 8),
}
PARTICLE_CASE = "tgv3_n6"
DT, VISC, DENS = 1e-3, 1.0 / 1600.0, 1.0
PART_T, PART_DT = 0.1, 0.05


def hash_field(shape, salt: int) -> np.ndarray:
    """Values in [-0.5, 0.5) from a 64-bit mix of (index, salt); exact."""
    q = np.arange(int(np.prod(shape)), dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = q * np.uint64(0x9E3779B97F4A7C15) + np.uint64(salt) * np.uint64(0xBF58476D1CE4E5B9)
        z ^= z >> np.uint64(31)
        z *= np.uint64(0x94D049BB133111EB)
        z ^= z >> np.uint64(29)
    return ((z >> np.uint64(11)).astype(np.float64) / float(1 << 53) - 0.5).reshape(shape)


def affine_nodes(mesh, points):
    """Physical coordinates (3, nel, n, n, n) of an axis-aligned box mesh's
    GLL nodes: x = x0 + (1 + xi) / 2 * h, from the element's corner
    vertices."""
    v = np.asarray(mesh.vertices)
    lo = v.min(axis=2)             # (nel, 3)
    hi = v.max(axis=2)
    n = len(points)
    out = np.empty((3, mesh.nel, n, n, n))
    half = (1.0 + np.asarray(points)) / 2.0
    for a in range(3):
        c = lo[:, a][:, None] + half[None, :] * (hi[:, a] - lo[:, a])[:, None]   # (nel, n)
        shp = [mesh.nel, 1, 1, 1]
        shp[3 - a] = n                 # a = 0 -> i (last axis)
        out[a] = np.broadcast_to(c.reshape(shp), (mesh.nel, n, n, n))
    return out


def particle_factors(mesh, n):
    """Exact jac / tinv_jac of the axis-aligned box map, rounded once:
    J = diag(h/2), tinv = diag(2/h), (9, nel, n, n, n)."""
    v = np.asarray(mesh.vertices)
    h = v.max(axis=2) - v.min(axis=2)    # (nel, 3)
    jac = np.zeros((9, mesh.nel, n, n, n))
    tinv = np.zeros((9, mesh.nel, n, n, n))
    for a in range(3):
        jac[4 * a] = (h[:, a] / 2.0)[:, None, None, None]
        tinv[4 * a] = (2.0 / h[:, a])[:, None, None, None]
    return jac, tinv


def particle_velocity(mesh, points, t, dt):
    """Reference-domain velocity snapshots (3 levels, 3 comps, nel, n, n, n)
    at t - 2 dt, t - dt, t: low-order polynomials of the node coordinates."""
    X = affine_nodes(mesh, points)
    L = 2.0 * 3.141592653589793
    x, y, z = (X[a] / L - 0.5 for a in range(3))
    n = len(points)
    ur = np.empty((3, 3, mesh.nel, n, n, n))
    for lev in range(3):
        tt = t - (2 - lev) * dt
        ur[lev, 0] = 12.0 * (y * (1.0 - 4.0 * y * y) + 0.5 * tt)
        ur[lev, 1] = -12.0 * (x * (1.0 - 4.0 * x * x)) + 3.0 * z
        ur[lev, 2] = 9.0 * (x * y - 0.25 * tt) + 4.0
    return ur


def particle_states(mesh, npart: int, salt: int):
    t, dt = PART_T, PART_DT
    state = np.zeros((npart, 8))
    state[:, :3] = 1.98 * hash_field((npart, 3), salt)
    state[:, 3:6] = 40.0 * hash_field((npart, 3), salt + 1)
    state[:, 6] = t - dt
    state[:, 7] = 0.05 + 2.0 * (hash_field((npart,), salt + 2) + 0.5)
    ints = np.zeros((npart, 3), np.int32)
    el = (np.floor((hash_field((npart,), salt + 3) + 0.5) * mesh.nel)).astype(np.int32)
    ints[:, 0] = np.minimum(el, mesh.nel - 1)
    ints[:, 1] = ints[:, 0]
    return state, ints
