"""Test-infrastructure oracles for the SSENSS solve path.

TEST INFRASTRUCTURE ONLY -- imported by tests/, __graft_entry__.smoke() and
bench.py's CPU baseline, never by the product (ssenss_b200/).

Two CPU implementations with one Python face:

* Oracle     -- ssg_oracle.c, the plain-C restatement of the reference's
                algorithm (libssg_oracle.so, always built).
* Reference  -- the reference SSENSS sources compiled in place with a
                single-rank MPI stand-in and an in-memory mesh
                (_ref/libssenss_ref.so, built only where the reference source
                tree is present, see oracle/Makefile).  It is not re-entrant:
                one Reference object at a time.

Fields are L-vectors of shape (nel, n, n, n) (u[e][k][j][i]); vector fields
are (3, nel, n, n, n).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "libssg_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libssenss_ref.so")
# the same reference with its solve path bound to libssenss_b200 through the
# C binding ssenss_b200/shim/ssenss_gpu_shim.c (needs a GPU to run)
REF_GPU_SO = os.path.join(HERE, "_ref", "libssenss_ref_gpu.so")

PRESSURE, X_VELOCITY, Y_VELOCITY, Z_VELOCITY = 0, 1, 2, 3

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


def _d(a):
    return a.ctypes.data_as(_dp)


def _i(a):
    return a.ctypes.data_as(_ip)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def build(quiet: bool = True) -> None:
    """Build the oracle (and the reference library where its sources are
    present) with oracle/Makefile."""
    import subprocess
    out = subprocess.run(["make", "-C", HERE], capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + out.stdout + out.stderr)


def reference_available() -> bool:
    return os.path.exists(REF_SO)


class _Common:
    """Shared shape bookkeeping."""

    n: int
    nel: int

    def _shape(self, n=None):
        n = self.n if n is None else n
        return (self.nel, n, n, n)

    @staticmethod
    def gll(n):
        """The oracle's GLL points and weights of order n."""
        x, w = np.empty(n), np.empty(n)
        Oracle.lib().og_gll(n, _d(x), _d(w))
        return x, w

    def _vshape(self, n=None):
        n = self.n if n is None else n
        return (3, self.nel, n, n, n)


class Oracle(_Common):
    """ssg_oracle.c restatement (see module docstring)."""

    _lib = None

    @classmethod
    def lib(cls):
        if cls._lib is None:
            if not os.path.exists(ORACLE_SO):
                build()
            L = C.CDLL(ORACLE_SO)
            L.og_create.restype = C.c_void_p
            L.og_create.argtypes = [C.c_int, C.c_int, _dp, _ip, C.c_double,
                                    C.c_double, C.c_double]
            L.og_destroy.argtypes = [C.c_void_p]
            L.og_set_params.argtypes = [C.c_void_p, C.c_double, C.c_double,
                                        C.c_double]
            for f in ("og_nlevels", "og_conv_n"):
                getattr(L, f).argtypes = [C.c_void_p]
                getattr(L, f).restype = C.c_int
            L.og_level_n.argtypes = [C.c_void_p, C.c_int]
            L.og_level_n.restype = C.c_int
            L.og_level_geometry.argtypes = [C.c_void_p, C.c_int, C.c_int, _dp]
            L.og_level_precon.argtypes = [C.c_void_p, C.c_int, C.c_int, _dp]
            L.og_dss_pairs.argtypes = [C.c_void_p, _ip]
            L.og_conv_geometry.argtypes = [C.c_void_p, C.c_int, _dp]
            L.og_local_opeval.argtypes = [C.c_void_p, C.c_int, C.c_int, _dp, _dp]
            L.og_global_opeval.argtypes = [C.c_void_p, C.c_int, C.c_int, _dp, _dp]
            L.og_dss.argtypes = [C.c_void_p, C.c_int, _dp]
            L.og_dot.argtypes = [C.c_void_p, C.c_int, _dp, _dp]
            L.og_dot.restype = C.c_double
            L.og_set_dot_perturbation.argtypes = [C.c_void_p, C.c_double, C.c_ulonglong]
            L.og_solve_poisson.argtypes = [C.c_void_p, _dp, _dp, C.c_double,
                                           C.c_int, _dp, C.c_int]
            L.og_solve_poisson.restype = C.c_int
            L.og_solve_helmholtz.argtypes = [C.c_void_p, C.c_int, _dp, _dp,
                                             C.c_double, C.c_int, _dp, C.c_int]
            L.og_solve_helmholtz.restype = C.c_int
            L.og_mg_precon.argtypes = [C.c_void_p, _dp, _dp, C.c_double]
            L.og_convection.argtypes = [C.c_void_p, _dp, _dp, _dp]
            L.og_particles_advance.argtypes = [C.c_void_p, C.c_size_t, _dp, _ip,
                                               _dp]
            L.og_particles_advance.restype = C.c_int
            L.og_set_particle_basis.argtypes = [C.c_void_p, _dp, _dp, _dp]
            L.og_point_interp.argtypes = [C.c_int, _dp, _dp, C.c_double,
                                          C.c_double, C.c_double]
            L.og_point_interp.restype = C.c_double
            L.og_gll.argtypes = [C.c_int, _dp, _dp]
            L.og_deriv.argtypes = [C.c_int, _dp, _dp]
            L.og_svv_deriv.argtypes = [C.c_int, _dp, _dp, C.c_int, C.c_double, _dp]
            L.og_interp.argtypes = [C.c_int, _dp, C.c_int, _dp, _dp]
            L.og_set_svv.argtypes = [C.c_int, C.c_double]
            cls._lib = L
        return cls._lib

    def __init__(self, mesh, n, dt=1e-3, visc=1.0 / 1600.0, dens=1.0, svv=(-1, 0.0)):
        """svv: (svvn, svva) of the SVV Helmholtz operator (svvn < 0: 2n/3)."""
        L = self.lib()
        self.n, self.nel = int(n), int(mesh.nel)
        self._vert = _f64(mesh.vertices)
        self._neigh = np.ascontiguousarray(mesh.neigh, dtype=np.int32)
        L.og_set_svv(int(svv[0]), float(svv[1]))
        self.h = L.og_create(self.n, self.nel, _d(self._vert), _i(self._neigh),
                             dt, visc, dens)
        if not self.h:
            raise ValueError("unsupported order")
        self.nlevels = L.og_nlevels(self.h)
        self.orders = [L.og_level_n(self.h, l) for l in range(self.nlevels)]
        self.nconv = L.og_conv_n(self.h)
        self.dt, self.visc, self.t = dt, visc, 0.0

    def close(self):
        if getattr(self, "h", None):
            self.lib().og_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def set_params(self, t, dt, visc):
        self.t, self.dt, self.visc = t, dt, visc
        self.lib().og_set_params(self.h, t, dt, visc)

    # -- data -------------------------------------------------------------
    def geometry(self, level, comp):
        out = np.empty(self._shape(self.orders[level]))
        self.lib().og_level_geometry(self.h, level, comp, _d(out))
        return out

    def precon(self, level, which):
        out = np.empty(self._shape(self.orders[level]))
        self.lib().og_level_precon(self.h, level, which, _d(out))
        return out

    def dss_pairs(self):
        out = np.empty((self.nel, 26, 2), dtype=np.int32)
        self.lib().og_dss_pairs(self.h, _i(out))
        return out

    def conv_geometry(self, comp):
        out = np.empty(self._shape(self.nconv))
        self.lib().og_conv_geometry(self.h, comp, _d(out))
        return out

    # -- operators ----------------------------------------------------------
    def local_opeval(self, var, p, level=0):
        p = _f64(p)
        out = np.empty_like(p)
        self.lib().og_local_opeval(self.h, level, var, _d(p), _d(out))
        return out

    def global_opeval(self, var, p, level=0):
        p = _f64(p)
        out = np.empty_like(p)
        self.lib().og_global_opeval(self.h, level, var, _d(p), _d(out))
        return out

    def dss(self, u, level=0):
        u = _f64(u).copy()
        self.lib().og_dss(self.h, level, _d(u))
        return u

    def dot(self, x, y, level=0):
        return self.lib().og_dot(self.h, level, _d(_f64(x)), _d(_f64(y)))

    # -- solvers ------------------------------------------------------------
    def solve_poisson(self, f, u0, eps=1e-10, max_iter=5000):
        f, u = _f64(f), _f64(u0).copy()
        hist = np.zeros(max_iter + 1)
        k = self.lib().og_solve_poisson(self.h, _d(f), _d(u), eps, max_iter,
                                        _d(hist), len(hist))
        return u, hist[:min(k, len(hist))]

    def solve_helmholtz(self, var, f, u0, eps=1e-10, max_iter=5000):
        f, u = _f64(f), _f64(u0).copy()
        hist = np.zeros(max_iter + 1)
        k = self.lib().og_solve_helmholtz(self.h, var, _d(f), _d(u), eps,
                                          max_iter, _d(hist), len(hist))
        return u, hist[:min(k, len(hist))]

    def rounding_spread(self, solve, f, seeds=8, rel_pert=2e-16):
        """How far the solution of solve(f, 0) (a bound method of this
        oracle, e.g. self.solve_poisson) is determined by the arithmetic:
        the largest relative difference (max |du| / max |u|) between the
        plain solve and `seeds` solves whose every global dot product is
        scaled by (1 + rel_pert * xi), xi in [-1, 1) (og_set_dot_perturbation).
        Any other correct summation order lands inside this spread."""
        u0, _ = solve(f, np.zeros_like(f))
        scale = max(float(np.max(np.abs(u0))), 1e-300)
        worst = 0.0
        try:
            for s in range(1, seeds + 1):
                self.lib().og_set_dot_perturbation(self.h, rel_pert, s)
                u, _ = solve(f, np.zeros_like(f))
                worst = max(worst, float(np.max(np.abs(u - u0))) / scale)
        finally:
            self.lib().og_set_dot_perturbation(self.h, 0.0, 1)
        return worst

    def mg_precon(self, r, eps=1e-10):
        r = _f64(r)
        z = np.empty_like(r)
        self.lib().og_mg_precon(self.h, _d(r), _d(z), eps)
        return z

    def convection(self, u, v):
        u, v = _f64(u), _f64(v)
        out = np.empty_like(u)
        self.lib().og_convection(self.h, _d(u), _d(v), _d(out))
        return out

    def particle_geometry(self):
        """(points, jac, tinv) the particle walk reads; jac/tinv (9, nel, n, n, n)."""
        x, _ = self.gll(self.n)
        jac = np.stack([self.geometry(0, 10 + a) for a in range(9)])
        tinv = np.stack([self.geometry(0, 19 + a) for a in range(9)])
        return x, jac, tinv

    def set_particle_basis(self, points, jac, tinv):
        """Walk particles on these GLL points and level-0 factors (bitwise
        parity with a caller whose points differ in the last bit)."""
        self._pb = (_f64(points), _f64(jac), _f64(tinv))
        self.lib().og_set_particle_basis(self.h, *(_d(a) for a in self._pb))

    def particles_advance(self, state, ints, ur):
        state = _f64(state).copy()
        ints = np.ascontiguousarray(ints, dtype=np.int32).copy()
        ur = _f64(ur)
        passes = self.lib().og_particles_advance(self.h, state.shape[0],
                                                 _d(state), _i(ints), _d(ur))
        return state, ints, passes


class Reference(_Common):
    """The reference sources compiled in place (see module docstring)."""

    _lib = None
    _path = REF_SO

    @classmethod
    def lib(cls):
        if cls._lib is None:
            if not os.path.exists(cls._path):
                raise FileNotFoundError(cls._path)
            L = C.CDLL(cls._path)
            L.ssgref_step_log_count.restype = C.c_int
            L.ssgref_step_log_entry.argtypes = [C.c_int, _ip, _ip, _dp, C.c_int]
            L.ssgref_step_log_entry.restype = C.c_int
            L.ssgref_setup.argtypes = [C.c_int, C.c_int, _dp, _ip, C.c_double,
                                       C.c_double, C.c_double]
            L.ssgref_setup.restype = C.c_int
            L.ssgref_set_time.argtypes = [C.c_double, C.c_double, C.c_double]
            L.ssgref_level_order.argtypes = [C.c_int]
            L.ssgref_level_order.restype = C.c_int
            L.ssgref_conv_order.restype = C.c_int
            L.ssgref_level_basis.argtypes = [C.c_int, _dp, _dp, _dp, _dp]
            L.ssgref_level_interp.argtypes = [C.c_int, _dp]
            L.ssgref_level_geometry.argtypes = [C.c_int, C.c_int, _dp]
            L.ssgref_level_precon.argtypes = [C.c_int, C.c_int, _dp]
            L.ssgref_conv_geometry.argtypes = [C.c_int, _dp]
            L.ssgref_conv_basis.argtypes = [_dp, _dp, _dp]
            L.ssgref_global_opeval.argtypes = [C.c_int, _dp, _dp]
            L.ssgref_local_opeval.argtypes = [C.c_int, _dp, _dp]
            L.ssgref_dss.argtypes = [_dp]
            L.ssgref_dss_level.argtypes = [C.c_int, _dp]
            L.ssgref_dot.argtypes = [_dp, _dp]
            L.ssgref_dot.restype = C.c_double
            L.ssgref_solve_poisson.argtypes = [_dp, _dp, C.c_double, _dp, C.c_int]
            L.ssgref_solve_poisson.restype = C.c_int
            L.ssgref_solve_helmholtz.argtypes = [C.c_int, _dp, _dp, C.c_double,
                                                 _dp, C.c_int]
            L.ssgref_solve_helmholtz.restype = C.c_int
            L.ssgref_fcg_mg.argtypes = [_dp, _dp, C.c_double, C.c_int]
            L.ssgref_fcg_mg.restype = C.c_double
            L.ssgref_cg_jacobi.argtypes = [C.c_int, _dp, _dp, C.c_double, C.c_int]
            L.ssgref_cg_jacobi.restype = C.c_double
            L.ssgref_mg_precon.argtypes = [_dp, _dp, C.c_double]
            L.ssgref_convection.argtypes = [_dp, _dp, _dp]
            L.ssgref_time.restype = C.c_double
            L.ssgref_get_field.argtypes = [C.c_int, C.c_int, _dp]
            L.ssgref_set_field.argtypes = [C.c_int, C.c_int, _dp]
            L.ssgref_particles_advance.argtypes = [C.c_size_t, _dp, _ip]
            L.ssgref_set_level0_factor.argtypes = [C.c_int, _dp]
            L.ssgref_set_svv.argtypes = [C.c_int, C.c_double]
            L.ssgref_stokes_operator.argtypes = [C.c_int, _dp, _dp, _dp]
            L.ssgref_integrate_convection_rk4.argtypes = [_dp, C.c_double, C.c_double,
                                                          C.c_double, C.c_double]
            L.ssgref_particles_advance.restype = C.c_int
            cls._lib = L
        return cls._lib

    def __init__(self, mesh, n, dt=1e-3, visc=1.0 / 1600.0, dens=1.0, svv=(-1, 0.0)):
        """svv: (svvn, svva) of the SVV Helmholtz operator (svvn < 0: 2n/3,
        the reference's src/main.c:54-55 values are (2n/3, 0))."""
        L = self.lib()
        self.n, self.nel = int(n), int(mesh.nel)
        # the reference keeps pointers into these during setup only
        self._vert = _f64(mesh.vertices)
        self._neigh = np.ascontiguousarray(mesh.neigh, dtype=np.int32)
        L.ssgref_set_svv(int(svv[0]), float(svv[1]))
        self.nlevels = L.ssgref_setup(self.n, self.nel, _d(self._vert),
                                      _i(self._neigh), dt, visc, dens)
        self.orders = [L.ssgref_level_order(l) for l in range(self.nlevels)]
        self.nconv = L.ssgref_conv_order()
        self.dt, self.visc, self.t = dt, visc, 0.0

    def close(self):
        self.lib().ssgref_teardown()

    def set_params(self, t, dt, visc):
        self.t, self.dt, self.visc = t, dt, visc
        self.lib().ssgref_set_time(t, dt, visc)

    # -- data -------------------------------------------------------------
    def basis(self, level):
        m = self.orders[level]
        x, w = np.empty(m), np.empty(m)
        d, s = np.empty((m, m)), np.empty((m, m))
        self.lib().ssgref_level_basis(level, _d(x), _d(w), _d(d), _d(s))
        # stored d[j][i] = D_ij: transpose to D[i, j]
        return x, w, d.T.copy(), s.T.copy()

    def interp(self, level):
        nf, nc = self.orders[level - 1], self.orders[level]
        a = np.empty((nc, nf))
        self.lib().ssgref_level_interp(level, _d(a))
        return a.T.copy()   # [i_fine, p_coarse]

    def geometry(self, level, comp):
        out = np.empty(self._shape(self.orders[level]))
        self.lib().ssgref_level_geometry(level, comp, _d(out))
        return out

    def precon(self, level, which):
        out = np.empty(self._shape(self.orders[level]))
        self.lib().ssgref_level_precon(level, which, _d(out))
        return out

    def conv_geometry(self, comp):
        out = np.empty(self._shape(self.nconv))
        self.lib().ssgref_conv_geometry(comp, _d(out))
        return out

    # -- operators ----------------------------------------------------------
    def global_opeval(self, var, p, level=0):
        assert level == 0
        p = _f64(p)
        out = np.empty_like(p)
        self.lib().ssgref_global_opeval(var, _d(p), _d(out))
        return out

    def local_opeval(self, var, p, level=0):
        assert level == 0
        p = _f64(p)
        out = np.empty_like(p)
        self.lib().ssgref_local_opeval(var, _d(p), _d(out))
        return out

    def dss(self, u, level=0):
        u = _f64(u).copy()
        if level == 0:
            self.lib().ssgref_dss(_d(u))
        else:
            self.lib().ssgref_dss_level(level, _d(u))
        return u

    def dot(self, x, y, level=0):
        assert level == 0
        return self.lib().ssgref_dot(_d(_f64(x)), _d(_f64(y)))

    # -- solvers ------------------------------------------------------------
    def solve_poisson(self, f, u0, eps=1e-10, max_iter=5000):
        f, u = _f64(f), _f64(u0).copy()
        hist = np.zeros(5001)
        k = self.lib().ssgref_solve_poisson(_d(f), _d(u), eps, _d(hist),
                                            len(hist))
        return u, hist[:min(k, len(hist))]

    def solve_helmholtz(self, var, f, u0, eps=1e-10, max_iter=5000):
        f, u = _f64(f), _f64(u0).copy()
        hist = np.zeros(5001)
        k = self.lib().ssgref_solve_helmholtz(var, _d(f), _d(u), eps, _d(hist),
                                              len(hist))
        return u, hist[:min(k, len(hist))]

    def mg_precon(self, r, eps=1e-10):
        r = _f64(r)
        z = np.empty_like(r)
        self.lib().ssgref_mg_precon(_d(r), _d(z), eps)
        return z

    def convection(self, u, v):
        u, v = _f64(u), _f64(v)
        out = np.empty_like(u)
        self.lib().ssgref_convection(_d(u), _d(v), _d(out))
        return out

    # -- time stepping / particles -------------------------------------------
    def init_tgv(self):
        self.lib().ssgref_init_tgv()

    def integrate_convection_rk4(self, u, t0, t, dt, beta):
        """integrate_convection_rk4 (src/time.c:84-130) on u (3, nel, n, n,
        n), returned updated; the history from set_field, the solver time
        from set_params."""
        u = _f64(u).copy()
        self.lib().ssgref_integrate_convection_rk4(_d(u), t0, t, dt, beta)
        return u

    def init_ethier_steinman(self):
        """The reference's analytic test case (src/test.c:202-214):
        Ethier-Steinman velocity and time-dependent Dirichlet walls."""
        self.lib().ssgref_init_ethier_steinman()

    def ns_step(self):
        self.lib().ssgref_ns_step()

    def stokes_operator(self, which, u, g=None):
        """The Stokes operators of a step, element by element (no DSS):
        which 0 = double_curl_operator(u); 1 = the pressure right-hand side
        of u~ = u with the surface terms of g (3 fields) on the walls; 2 =
        the velocity right-hand sides of u~ = u and the pressure g."""
        u = _f64(u)
        shape = self._shape()
        out = np.zeros(shape if which == 1 else (3,) + shape)
        if g is None:
            g = np.zeros((3,) + shape)
        self.lib().ssgref_stokes_operator(which, _d(u), _d(_f64(g)), _d(out))
        return out

    def step_log(self, clear=True):
        """Every solve the Navier-Stokes steps ran since the last clear:
        list of (kind 0 Poisson / 1 Helmholtz, var, residual history)."""
        L = self.lib()
        out = []
        hist = np.zeros(5001)
        kind, var = C.c_int(), C.c_int()
        for i in range(L.ssgref_step_log_count()):
            k = L.ssgref_step_log_entry(i, C.byref(kind), C.byref(var), _d(hist), len(hist))
            out.append((kind.value, var.value, hist[:min(k, len(hist))].copy()))
        if clear:
            L.ssgref_step_log_clear()
        return out

    def time(self):
        return self.lib().ssgref_time()

    def get_field(self, which, hist_level=0):
        out = np.empty(self._shape())
        self.lib().ssgref_get_field(which, hist_level, _d(out))
        return out

    def set_field(self, which, hist_level, src):
        self.lib().ssgref_set_field(which, hist_level, _d(_f64(src)))

    def particle_geometry(self):
        """(points, jac, tinv) the reference's particle walk reads."""
        x = self.basis(0)[0]
        jac = np.stack([self.geometry(0, 10 + a) for a in range(9)])
        tinv = np.stack([self.geometry(0, 19 + a) for a in range(9)])
        return x, jac, tinv

    def set_particle_factors(self, jac, tinv):
        """Overwrite the level-0 jac / tinv_jac (9, nel, n, n, n) the
        reference's particle walk reads."""
        for a in range(9):
            self.lib().ssgref_set_level0_factor(10 + a, _d(_f64(jac[a])))
            self.lib().ssgref_set_level0_factor(19 + a, _d(_f64(tinv[a])))

    def particles_advance(self, state, ints, ur):
        """ur: (3 levels, 3 comps, nel, n, n, n), oldest level first."""
        for lev in range(3):
            for comp in range(3):
                self.set_field(4 + comp, 2 - lev, ur[lev, comp])
        state = _f64(state).copy()
        ints = np.ascontiguousarray(ints, dtype=np.int32).copy()
        self.lib().ssgref_particles_advance(state.shape[0], _d(state), _i(ints))
        return state, ints


class ReferenceGPU(Reference):
    """The reference with its solve path on the GPU: the same harness and
    entry points as Reference, built against the library's C binding
    (ssenss_b200/shim/ssenss_gpu_shim.c).  Its library and Reference's can
    live in one process (each resolves its own symbols), but a failure inside
    the binding ends the process through the reference's fatal_error, so
    tests run it in a child process."""

    _lib = None
    _path = REF_GPU_SO

    def device_step(self, on):
        """integrate_navier_stokes as one library step on the device (True,
        the binding's default) or the reference's own step with its solves
        bound to the library (False)."""
        self.lib().ssgref_gpu_device_step(1 if on else 0)
