"""Synthetic hexahedral meshes in the SSENSS grid-record form.

A mesh is what one grid file of the reference holds (src/dataio.c:34-62,
misc/rectangular_grid.py:21-135): per element the 8 trilinear vertices of an
n=2 GLL element (vertex index a + 2b + 4c, x fastest) and 26 neighbour ids --
6 faces (w, e, s, n, b, t), 12 edges (sw, se, nw, ne, bw, be, tw, te, bs, bn,
ts, tn) and 8 corners (x fastest) -- with a negative code on walls (-1
no-slip, -2 free-slip).  Elements are numbered x fastest (index order 'xyz').

The box generator follows the rules of misc/rectangular_grid.py (neighbours
wrap periodically, wall faces and their edges/corners carry the wall code)
and adds the deformations the channel workload needs: a per-axis vertex
coordinate list (tanh stretching) and a seeded random displacement of
interior vertices, shared by periodic images.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

# neighbour slots: faces, then edges, then corners (src/structs.h:25-54)
FACE_DIRS = [(-1, 0, 0), (1, 0, 0), (0, -1, 0), (0, 1, 0), (0, 0, -1), (0, 0, 1)]
EDGE_DIRS = [
    (-1, -1, 0), (1, -1, 0), (-1, 1, 0), (1, 1, 0),
    (-1, 0, -1), (1, 0, -1), (-1, 0, 1), (1, 0, 1),
    (0, -1, -1), (0, 1, -1), (0, -1, 1), (0, 1, 1),
]
CORNER_DIRS = [((c & 1) * 2 - 1, ((c >> 1) & 1) * 2 - 1, ((c >> 2) & 1) * 2 - 1)
               for c in range(8)]
ALL_DIRS = FACE_DIRS + EDGE_DIRS + CORNER_DIRS

NO_SLIP = -1
FREE_SLIP = -2


@dataclasses.dataclass
class Mesh:
    """Grid records of `nel` elements (see module docstring)."""

    vertices: np.ndarray   # (nel, 3, 8) float64: x[8], y[8], z[8]
    neigh: np.ndarray      # (nel, 26) int32
    shape: tuple           # (nx, ny, nz) for box meshes
    description: str = ""

    @property
    def nel(self) -> int:
        return int(self.neigh.shape[0])

    def unique_nodes(self, n: int) -> int:
        """Unique GLL nodes of order n (the DSS equivalence classes)."""
        nx, ny, nz = self.shape
        per = [self._periodic(a) for a in range(3)]
        cnt = 1
        for a, na in enumerate((nx, ny, nz)):
            cnt *= na * (n - 1) + (0 if per[a] else 1)
        return cnt

    def _periodic(self, axis: int) -> bool:
        # a box is periodic along `axis` when its first element's low face
        # neighbour is not a wall
        return int(self.neigh[0, 2 * axis]) >= 0


class SplitMix64:
    """splitmix64 (Steele, Lea, Flood 2014): the seeded stream behind every
    synthetic mesh deformation and right-hand side."""

    MASK = (1 << 64) - 1

    def __init__(self, seed: int):
        self.state = seed & self.MASK

    def next(self) -> int:
        self.state = (self.state + 0x9E3779B97F4A7C15) & self.MASK
        z = self.state
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & self.MASK
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & self.MASK
        return z ^ (z >> 31)

    def uniform(self) -> float:
        """Uniform in [0, 1) with 53 random bits."""
        return (self.next() >> 11) * (1.0 / 9007199254740992.0)


def box_mesh(shape, lo=(0.0, 0.0, 0.0), hi=(2 * math.pi,) * 3,
             periodic=(True, True, True), wall=NO_SLIP, coords=None,
             perturb: float = 0.0, seed: int = 0) -> Mesh:
    """Box of nx x ny x nz hexahedra.

    coords: optional per-axis vertex coordinate arrays (length n_a + 1)
    replacing the equidistant spacing.  perturb: interior vertices move by
    perturb * h_local * U(-1, 1) per coordinate, h_local the smaller adjacent
    spacing along that axis; vertices on walls stay put and periodic images
    share their displacement.
    """
    nx, ny, nz = (int(s) for s in shape)
    dims = (nx, ny, nz)
    axes = []
    for a in range(3):
        if coords is not None and coords[a] is not None:
            c = np.asarray(coords[a], dtype=np.float64)
            assert c.shape == (dims[a] + 1,)
        else:
            c = np.array([lo[a] + i * (hi[a] - lo[a]) / dims[a]
                          for i in range(dims[a] + 1)], dtype=np.float64)
        axes.append(c)

    # lattice of vertices (nx+1, ny+1, nz+1, 3)
    X = np.empty((nx + 1, ny + 1, nz + 1, 3), dtype=np.float64)
    X[..., 0] = axes[0][:, None, None]
    X[..., 1] = axes[1][None, :, None]
    X[..., 2] = axes[2][None, None, :]

    if perturb > 0.0:
        rng = SplitMix64(seed)
        # one displacement per distinct vertex: periodic image planes share it
        nv = [dims[a] if periodic[a] else dims[a] + 1 for a in range(3)]
        disp = np.zeros((nv[0], nv[1], nv[2], 3))
        on_wall = [np.zeros(nv[a], dtype=bool) for a in range(3)]
        for a in range(3):
            if not periodic[a]:
                on_wall[a][0] = True
                on_wall[a][-1] = True
        hloc = []
        for a in range(3):
            c = axes[a]
            h = np.empty(nv[a])
            for i in range(nv[a]):
                left = c[i] - c[i - 1] if i > 0 else (
                    c[-1] - c[-2] if periodic[a] else np.inf)
                right = c[i + 1] - c[i] if i < dims[a] else np.inf
                h[i] = min(left, right)
            hloc.append(h)
        for k in range(nv[2]):
            for j in range(nv[1]):
                for i in range(nv[0]):
                    if on_wall[0][i] or on_wall[1][j] or on_wall[2][k]:
                        continue
                    idx = (i, j, k)
                    for a in range(3):
                        u = 2.0 * rng.uniform() - 1.0
                        disp[i, j, k, a] = perturb * hloc[a][idx[a]] * u
        for k in range(nz + 1):
            for j in range(ny + 1):
                for i in range(nx + 1):
                    ii = i % nx if periodic[0] else i
                    jj = j % ny if periodic[1] else j
                    kk = k % nz if periodic[2] else k
                    X[i, j, k] += disp[ii, jj, kk]

    nel = nx * ny * nz
    vert = np.empty((nel, 3, 8), dtype=np.float64)
    neigh = np.empty((nel, 26), dtype=np.int32)
    for k in range(nz):
        for j in range(ny):
            for i in range(nx):
                e = i + j * nx + k * nx * ny
                for v in range(8):
                    a, b, c = v & 1, (v >> 1) & 1, (v >> 2) & 1
                    vert[e, :, v] = X[i + a, j + b, k + c]
                for s, (di, dj, dk) in enumerate(ALL_DIRS):
                    idx = [i + di, j + dj, k + dk]
                    code = None
                    for a in range(3):
                        if idx[a] < 0 or idx[a] >= dims[a]:
                            if periodic[a]:
                                idx[a] %= dims[a]
                            else:
                                code = wall
                    neigh[e, s] = code if code is not None else (
                        idx[0] + idx[1] * nx + idx[2] * nx * ny)
    return Mesh(np.ascontiguousarray(vert), np.ascontiguousarray(neigh),
                (nx, ny, nz))


def concat_meshes(meshes) -> tuple:
    """Independent meshes as one mesh: elements of mesh k follow those of
    meshes 0 .. k-1, neighbour ids shifted by the element offset, wall codes
    kept.  Returns (mesh, seg_first) with seg_first[k] the first element of
    mesh k and seg_first[-1] the total (the segment table of
    ssg_solve_helmholtz_segments)."""
    first = [0]
    verts, neigh = [], []
    for m in meshes:
        off = first[-1]
        verts.append(np.asarray(m.vertices, dtype=np.float64))
        nb = np.asarray(m.neigh, dtype=np.int32).copy()
        nb[nb >= 0] += off
        neigh.append(nb)
        first.append(off + m.nel)
    mesh = Mesh(np.concatenate(verts), np.concatenate(neigh), (first[-1], 1, 1),
                "concatenation of " + ", ".join(m.description or "mesh" for m in meshes))
    return mesh, np.array(first, dtype=np.int32)


def tgv_box(nel_per_dir: int) -> Mesh:
    """Triply periodic [0, 2 pi]^3 box of equal hexahedra (Taylor-Green)."""
    m = box_mesh((nel_per_dir,) * 3)
    m.description = f"TGV periodic [0,2pi]^3, {nel_per_dir}^3 elements"
    return m


def channel_mesh(shape=(32, 16, 16), stretch: float = 2.0,
                 perturb: float = 0.1, seed: int = 20241203) -> Mesh:
    """Deformed channel [0,4 pi] x [-1,1] x [0,2 pi]: periodic in x and z,
    no-slip walls at y = -1, 1, tanh-stretched wall-normal vertices
    y_j = tanh(s (2j/ny - 1)) / tanh(s), interior vertices perturbed by
    perturb * h_local * U(-1,1) from splitmix64(seed)."""
    nx, ny, nz = shape
    ys = np.array([math.tanh(stretch * (2.0 * j / ny - 1.0)) / math.tanh(stretch)
                   for j in range(ny + 1)])
    ys[0], ys[-1] = -1.0, 1.0
    m = box_mesh(shape, lo=(0.0, -1.0, 0.0), hi=(4 * math.pi, 1.0, 2 * math.pi),
                 periodic=(True, False, True), coords=(None, ys, None),
                 perturb=perturb, seed=seed)
    m.description = (f"channel {nx}x{ny}x{nz}, tanh({stretch}) y-stretch, "
                     f"perturb {perturb}, seed {seed}")
    return m


def factor3(e: int) -> tuple:
    """Factor e into three integers as close to a cube as possible."""
    best = None
    for a in range(1, int(round(e ** (1 / 3))) + 2):
        if e % a:
            continue
        r = e // a
        for b in range(a, int(math.isqrt(r)) + 1):
            if r % b:
                continue
            c = r // b
            cand = tuple(sorted((a, b, c)))
            score = max(cand) - min(cand)
            if best is None or score < best[0]:
                best = (score, cand)
    if best is None:
        return (1, 1, e)
    return best[1]


def gll(n: int):
    """GLL points and weights of n points (the library's gll_basis)."""
    from . import _lib
    x, w = np.empty(n), np.empty(n)
    st = _lib.load().ssg_gll(int(n), x.ctypes.data_as(_lib._dp), w.ctypes.data_as(_lib._dp))
    if st != 0:
        raise ValueError(f"no GLL basis of {n} points")
    return x, w


def periodic_box_fourier_rhs(shape, n: int, seed: int, modes: int = 8, kmax: int = 3,
                             length: float = 2 * math.pi) -> np.ndarray:
    """Weak, assembled right-hand side on the undeformed periodic box
    box_mesh(shape) (element e = ex + nx (ey + ny ez), local i along x) of
    `modes` seeded Fourier modes g = sum a cos(k.x + phi), a ~ N(0, 1),
    k integer in [-kmax, kmax]^3 (k != 0, so mean zero): DSS(rho J g), the
    local products summed over the copies of each global node."""
    nx, ny, nz = shape
    x, w = gll(n)
    h = length / np.array([nx, ny, nz], dtype=float)
    e = np.arange(nx * ny * nz)
    ex, ey, ez = e % nx, (e // nx) % ny, e // (nx * ny)
    m = n - 1
    ar = np.arange(n)
    gx = (ex[:, None, None, None] * m + ar[None, None, None, :]) % (nx * m)
    gy = (ey[:, None, None, None] * m + ar[None, None, :, None]) % (ny * m)
    gz = (ez[:, None, None, None] * m + ar[None, :, None, None]) % (nz * m)
    gid = (gx + nx * m * (gy + ny * m * gz)).ravel()
    X = (ex[:, None, None, None] + (1 + x[None, None, None, :]) / 2) * h[0]
    Y = (ey[:, None, None, None] + (1 + x[None, None, :, None]) / 2) * h[1]
    Z = (ez[:, None, None, None] + (1 + x[None, :, None, None]) / 2) * h[2]
    rng = np.random.default_rng(seed)
    g = np.zeros((nx * ny * nz, n, n, n))
    for _ in range(modes):
        k = rng.integers(-kmax, kmax + 1, 3)
        if not k.any():
            k[0] = 1
        g += rng.standard_normal() * np.cos(k[0] * X + k[1] * Y + k[2] * Z +
                                            rng.uniform(0, 2 * math.pi))
    rho = w[None, None, None, :] * w[None, None, :, None] * w[None, :, None, None]
    loc = (rho * (h[0] * h[1] * h[2] / 8.0) * g).ravel()
    tot = np.bincount(gid, weights=loc, minlength=int(gid.max()) + 1)
    return tot[gid].reshape(nx * ny * nz, n, n, n)

