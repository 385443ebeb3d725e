"""B200 (sm_100a) implementation of the SSENSS per-timestep solve path.

Python mirror of the reference's solver call surface (src/solver.h,
src/global.h, src/convection.h, src/particles.h) over the C ABI in
include/ssenss_b200.h.  Fields are numpy arrays (host memory; copied through
the library's staging) or CUDA tensors (device memory, used in place) in the
reference's L-vector layout u[e][k][j][i].

    ctx = Context(device=0)
    ctx.setup_mesh(mesh, n=8)          # ssenss_b200.mesh.box_mesh(...)
    ap = ctx.global_opeval(PRESSURE, p)
    u, info = ctx.solve_poisson_cg(f, u0, eps=1e-10)

Every compute call runs CUDA kernels; without a usable GPU the context
cannot be created (SsgError with SSG_ERR_CUDA).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import SolveInfo

PRESSURE, X_VELOCITY, Y_VELOCITY, Z_VELOCITY = 0, 1, 2, 3
FP64, MIXED = 0, 1

STATUS = {
    0: "SSG_OK", 1: "SSG_ERR_ARG", 2: "SSG_ERR_CUDA", 3: "SSG_ERR_NOMEM",
    4: "SSG_ERR_BUDGET", 5: "SSG_MAXITER", 6: "SSG_NONFINITE", 7: "SSG_ERR_MESH",
    8: "SSG_ERR_STATE", 9: "SSG_ERR_TIMEOUT", 10: "SSG_ERR_CANCELLED",
}


class SsgError(RuntimeError):
    def __init__(self, status, detail=""):
        self.status = status
        super().__init__(f"{STATUS.get(status, status)}: {detail}")


def _ptr(a):
    """Pointer to a numpy array's data or a CUDA tensor's storage."""
    if isinstance(a, np.ndarray):
        if not a.flags.c_contiguous:
            raise ValueError("array must be C-contiguous")
        return C.c_void_p(a.ctypes.data)
    if hasattr(a, "data_ptr"):
        if not a.is_contiguous():
            raise ValueError("tensor must be contiguous")
        return C.c_void_p(a.data_ptr())
    raise TypeError(f"unsupported field type {type(a)}")


def tuning(n: int) -> dict:
    """Launch shapes in use for order n (ssg_tuning)."""
    lib = _lib.load()
    a, d, v = C.c_int(), C.c_int(), C.c_int()
    st = lib.ssg_tuning(int(n), C.byref(a), C.byref(d), C.byref(v))
    if st != 0:
        raise SsgError(st, "tuning")
    return {"ax_elements_per_block": a.value, "dss_blocks_per_sm": d.value,
            "vector_blocks_per_sm": v.value}


def kernel_launch_count() -> int:
    """Kernel launches of the library in this process so far."""
    return int(_lib.load().ssg_kernel_launch_count())


class Context:
    """One GPU context (ssg_context): mesh, factors, workspace, stream."""

    def __init__(self, device: int = 0, stream=None):
        self.lib = _lib.load()
        h = C.c_void_p()
        if stream is None:
            st = self.lib.ssg_create(device, C.byref(h))
        else:
            st = self.lib.ssg_create_on_stream(device, C.c_void_p(stream), C.byref(h))
        if st != 0:
            raise SsgError(st, "ssg_create")
        self.h = h
        self.n = self.nel = self.nlevels = 0
        self.orders = []

    def close(self):
        if getattr(self, "h", None):
            self.lib.ssg_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st, what, ok=(0,)):
        if st not in ok:
            raise SsgError(st, f"{what}: {self.lib.ssg_last_error(self.h).decode()}")
        return st

    @property
    def stream(self) -> int:
        return self.lib.ssg_stream(self.h) or 0

    # -- set-up ---------------------------------------------------------------
    def set_parameters(self, dt, visc, dens=1.0):
        self._check(self.lib.ssg_set_parameters(self.h, dt, visc, dens), "set_parameters")

    def set_precision(self, precision):
        p = {"fp64": FP64, "mixed": MIXED}.get(precision, precision)
        self._check(self.lib.ssg_set_precision(self.h, int(p)), "set_precision")

    def set_graphs(self, enable: bool):
        self._check(self.lib.ssg_set_graphs(self.h, int(bool(enable))), "set_graphs")

    def time_operator(self, var=PRESSURE, reps: int = 50) -> float:
        """Device microseconds per level-0 operator apply (ssg_time_operator)."""
        us = C.c_double()
        self._check(self.lib.ssg_time_operator(self.h, int(var), int(reps), C.byref(us)),
                    "time_operator")
        return float(us.value)

    def time_smoother(self, level: int = 0, reps: int = 50) -> dict:
        """Device microseconds per launch of the smoother CG kernels at a
        level (ssg_time_smoother): operator, DSS + dot, CG update."""
        us = (C.c_double * 3)()
        self._check(self.lib.ssg_time_smoother(self.h, int(level), int(reps), us),
                    "time_smoother")
        return {"operator": us[0], "dss_dot": us[1], "cg_update": us[2]}

    def autotune(self, reps: int = 10):
        """ssg_autotune: time the launch-shape candidates on this mesh and
        keep the fastest (process-wide, per order); returns the shapes."""
        self._check(self.lib.ssg_autotune(self.h, int(reps)), "autotune")
        return {n: tuning(n) for n in sorted(set(self.orders))}

    def set_setup_options(self, no_dealias=False, no_particles=False, opposite_pairing=False):
        """ssg_set_setup_options for the next setup_mesh (opposite_pairing:
        SSG_SETUP_OPPOSITE_PAIRING, the correct pairing of meshes with one or
        two elements along a periodic direction)."""
        flags = (1 if no_dealias else 0) | (2 if no_particles else 0) | \
            (4 if opposite_pairing else 0)
        self._check(self.lib.ssg_set_setup_options(self.h, flags), "set_setup_options")

    def set_svv(self, svvn=-1, svva=0.0):
        """ssg_set_svv: SVV cut-off mode and amplitude of the Helmholtz
        operator for the next setup_mesh (svvn < 0: 2n/3)."""
        self._check(self.lib.ssg_set_svv(self.h, int(svvn), float(svva)), "set_svv")

    def memory_bytes(self) -> int:
        b = C.c_size_t()
        self._check(self.lib.ssg_memory_info(self.h, C.byref(b)), "memory_info")
        return int(b.value)

    def setup_mesh(self, mesh, n: int):
        vert = np.ascontiguousarray(mesh.vertices, dtype=np.float64)
        neigh = np.ascontiguousarray(mesh.neigh, dtype=np.int32)
        self._check(self.lib.ssg_setup_mesh(
            self.h, int(n), int(mesh.nel), vert.ctypes.data_as(_lib._dp),
            neigh.ctypes.data_as(_lib._ip)), "setup_mesh")
        self._info()

    # -- drop-in set-up from the caller's own discretisation -------------------
    @staticmethod
    def _dbl(a):
        if a is None:
            return None, None
        a = np.ascontiguousarray(a, dtype=np.float64)
        return a, a.ctypes.data_as(_lib._dp)

    def setup_connectivity(self, neigh):
        """ssg_setup_connectivity: the reference's 26-neighbour table (nel, 26)."""
        neigh = np.ascontiguousarray(neigh, dtype=np.int32)
        self._check(self.lib.ssg_setup_connectivity(
            self.h, int(neigh.shape[0]), neigh.ctypes.data_as(_lib._ip)), "setup_connectivity")

    def setup_level(self, level, n, deriv, svv_deriv, weights, geom, jac_det, interp=None):
        """ssg_setup_level with the reference's stored arrays (deriv d[j][i],
        geom (6, nel, n, n, n), jac_det (nel, n, n, n), interp n_coarse x n_fine)."""
        keep = [self._dbl(a) for a in (deriv, svv_deriv, weights, geom, jac_det, interp)]
        self._check(self.lib.ssg_setup_level(self.h, int(level), int(n),
                                             *(k[1] for k in keep)), "setup_level")

    def setup_finish(self):
        self._check(self.lib.ssg_setup_finish(self.h), "setup_finish")
        self._info()

    def setup_dealias(self, m, deriv, weights, tinv_jac, jac_det, interp):
        """ssg_setup_dealias: conv_basis order m and its stored factors."""
        keep = [self._dbl(a) for a in (deriv, weights, tinv_jac, jac_det, interp)]
        self._check(self.lib.ssg_setup_dealias(self.h, int(m), *(k[1] for k in keep)),
                    "setup_dealias")

    def setup_particle_geometry(self, points, jac, tinv_jac):
        """ssg_setup_particle_geometry: the walk's GLL points (None: the
        library's) and level-0 jac / tinv_jac (9, nel, n, n, n)."""
        keep = [self._dbl(a) for a in (points, jac, tinv_jac)]
        self._check(self.lib.ssg_setup_particle_geometry(self.h, *(k[1] for k in keep)),
                    "setup_particle_geometry")

    def _info(self):
        n, nel, nl = C.c_int(), C.c_int(), C.c_int()
        orders = (C.c_int * 8)()
        self._check(self.lib.ssg_mesh_info(self.h, C.byref(n), C.byref(nel), C.byref(nl),
                                           orders), "mesh_info")
        self.n, self.nel, self.nlevels = n.value, nel.value, nl.value
        self.orders = [orders[i] for i in range(nl.value)]

    def level_data(self, level, which):
        m = self.orders[level]
        out = np.empty((self.nel, m, m, m))
        self._check(self.lib.ssg_level_data(self.h, level, which,
                                            out.ctypes.data_as(_lib._dp)), "level_data")
        return out

    def shape(self):
        return (self.nel, self.n, self.n, self.n)

    # -- operators (src/solver.c:191-198, src/global.c) ---------------------
    def _out_like(self, a, out):
        if out is not None:
            return out
        if isinstance(a, np.ndarray):
            return np.empty_like(a, dtype=np.float64)
        return a.new_empty(a.shape)

    def global_opeval(self, var, p, out=None):
        out = self._out_like(p, out)
        self._check(self.lib.ssg_global_opeval(self.h, var, _ptr(p), _ptr(out)),
                    "global_opeval")
        return out

    def local_opeval(self, var, p, out=None):
        out = self._out_like(p, out)
        self._check(self.lib.ssg_local_opeval(self.h, var, _ptr(p), _ptr(out)),
                    "local_opeval")
        return out

    def direct_stiffness_summation(self, u):
        """In place, like the reference."""
        self._check(self.lib.ssg_direct_stiffness_summation(self.h, _ptr(u)), "dss")
        return u

    def global_dot_product(self, x, y):
        r = C.c_double()
        self._check(self.lib.ssg_global_dot_product(self.h, _ptr(x), _ptr(y), C.byref(r)),
                    "global_dot_product")
        return r.value

    def inverse_mass(self, u):
        self._check(self.lib.ssg_inverse_mass(self.h, _ptr(u)), "inverse_mass")
        return u

    # -- solves (src/solver.c:33-189) ---------------------------------------
    def _solve(self, fn, args, what, history, max_iter):
        info = SolveInfo()
        hist = None
        if history:
            hist = np.zeros(min(max_iter, 8192))
            info.history = hist.ctypes.data_as(_lib._dp)
            info.history_cap = len(hist)
        st = fn(*args, C.byref(info))
        self._check(st, what, ok=(0, 5))
        res = {
            "status": STATUS[st],
            "iterations": info.iterations,
            "residual": info.residual,
            "initial_residual": info.initial_residual,
            "solve_ms": info.solve_ms,
        }
        if hist is not None:
            res["history"] = hist[:info.history_len].copy()
        return res

    def solve_poisson_cg(self, f, u, eps=1e-10, max_iter=5000, history=True):
        """u: initial guess, overwritten with the solution (as the reference
        overwrites sel->p)."""
        info = self._solve(self.lib.ssg_solve_poisson_cg,
                           (self.h, _ptr(f), _ptr(u), eps, max_iter),
                           "solve_poisson_cg", history, max_iter)
        return u, info

    def solve_helmholtz_cg(self, var, f, u, eps=1e-10, max_iter=5000, history=True):
        info = self._solve(self.lib.ssg_solve_helmholtz_cg,
                           (self.h, var, _ptr(f), _ptr(u), eps, max_iter),
                           "solve_helmholtz_cg", history, max_iter)
        return u, info

    def solve_helmholtz_segments(self, var, seg_first, lambdas, f, u, eps, max_iter=5000):
        """ssg_solve_helmholtz_segments: Helmholtz solves of the independent
        meshes concatenated in this context's mesh, in shared launches.
        seg_first: nseg + 1 element offsets; lambdas, eps: one per segment.
        Returns u and one info dict per segment."""
        seg = np.ascontiguousarray(seg_first, dtype=np.int32)
        lam = np.ascontiguousarray(lambdas, dtype=np.float64)
        ep = np.ascontiguousarray(np.broadcast_to(np.asarray(eps, dtype=np.float64),
                                                  lam.shape))
        nseg = len(lam)
        infos = (SolveInfo * nseg)()
        st = self.lib.ssg_solve_helmholtz_segments(
            self.h, int(var), nseg, seg.ctypes.data, lam.ctypes.data, _ptr(f), _ptr(u),
            ep.ctypes.data, int(max_iter), infos)
        self._check(st, "solve_helmholtz_segments", ok=(0, 5))
        return u, [{"status": STATUS[st], "iterations": i.iterations, "residual": i.residual,
                    "initial_residual": i.initial_residual} for i in infos]

    def conjugate_gradient(self, var, f, u, eps=1e-10, max_iter=5000, history=True):
        info = self._solve(self.lib.ssg_conjugate_gradient,
                           (self.h, var, _ptr(f), _ptr(u), eps, max_iter),
                           "conjugate_gradient", history, max_iter)
        return u, info

    def jacobi_preconditioner(self, var, r, z=None):
        """ssg_jacobi_preconditioner: z = r .* diag^-1 of var's operator."""
        z = self._out_like(r, z)
        self._check(self.lib.ssg_jacobi_preconditioner(self.h, int(var), _ptr(r), _ptr(z)),
                    "jacobi_preconditioner")
        return z

    def multigrid_preconditioner(self, r, z=None, eps=1e-10):
        z = self._out_like(r, z)
        self._check(self.lib.ssg_multigrid_preconditioner(self.h, _ptr(r), _ptr(z), eps),
                    "multigrid_preconditioner")
        return z

    # -- convection, particles ------------------------------------------------
    def convection_operator(self, u, v, out=None):
        out = self._out_like(u, out)
        self._check(self.lib.ssg_convection_operator(self.h, _ptr(u), _ptr(v), _ptr(out)),
                    "convection_operator")
        return out

    def set_velocity_history(self, u, u_old, u_oldold, t, dt):
        """ssg_set_velocity_history: the three velocity levels (3, nel, n,
        n, n each) at solver time t with step dt."""
        self._check(self.lib.ssg_set_velocity_history(self.h, _ptr(u), _ptr(u_old),
                                                      _ptr(u_oldold), float(t), float(dt)),
                    "set_velocity_history")

    def integrate_convection_rk4(self, u, t0, t, dt, beta):
        """ssg_integrate_convection_rk4 on u (3, nel, n, n, n), in place."""
        self._check(self.lib.ssg_integrate_convection_rk4(self.h, _ptr(u), float(t0), float(t),
                                                          float(dt), float(beta)),
                    "integrate_convection_rk4")
        return u

    # -- the whole time step (src/navier_stokes.c:224-235) -------------------
    def flow_set(self, u, conv, rot, p, f=None, t=0.0):
        """ssg_flow_set: u, conv, rot: three levels (newest first) of (3,
        nel, n, n, n); p: three levels of (nel, n, n, n); f: (3, nel, n, n,
        n) or None (zero); t: solver time."""
        ff = _lib.FlowFields()
        for l in range(3):
            ff.u[l] = _ptr(u[l])
            ff.conv[l] = _ptr(conv[l])
            ff.rot[l] = _ptr(rot[l])
            ff.p[l] = _ptr(p[l])
        ff.f = _ptr(f) if f is not None else None
        self._check(self.lib.ssg_flow_set(self.h, C.byref(ff), float(t)), "flow_set")

    def flow_get(self):
        """ssg_flow_get: dict of u, conv, rot (3 levels each, newest first),
        p (3 levels), f and t, as numpy arrays."""
        sh = self.shape()
        out = {k: [np.empty((3,) + sh) for _ in range(3)] for k in ("u", "conv", "rot")}
        out["p"] = [np.empty(sh) for _ in range(3)]
        out["f"] = np.empty((3,) + sh)
        ff = _lib.FlowFields()
        for l in range(3):
            ff.u[l] = _ptr(out["u"][l])
            ff.conv[l] = _ptr(out["conv"][l])
            ff.rot[l] = _ptr(out["rot"][l])
            ff.p[l] = _ptr(out["p"][l])
        ff.f = _ptr(out["f"])
        t = C.c_double()
        self._check(self.lib.ssg_flow_get(self.h, C.byref(ff), C.byref(t)), "flow_get")
        out["t"] = t.value
        return out

    def navier_stokes_step(self, f=None, bc_u=None, bc_dudt=None, history=True):
        """ssg_navier_stokes_step: one step on the resident fields.  Returns
        the four solves (pressure, then u, v, w) as dicts."""
        infos = (SolveInfo * 4)()
        hists = []
        if history:
            for k in range(4):
                h = np.zeros(5001)
                hists.append(h)
                infos[k].history = h.ctypes.data_as(_lib._dp)
                infos[k].history_cap = len(h)
        st = self.lib.ssg_navier_stokes_step(
            self.h, _ptr(f) if f is not None else None,
            _ptr(bc_u) if bc_u is not None else None,
            _ptr(bc_dudt) if bc_dudt is not None else None, infos)
        self._check(st, "navier_stokes_step", ok=(0, 5))
        res = []
        for k in range(4):
            i = infos[k]
            d = {"iterations": i.iterations, "residual": i.residual,
                 "initial_residual": i.initial_residual, "solve_ms": i.solve_ms}
            if history:
                d["history"] = hists[k][:i.history_len].copy()
            res.append(d)
        return res

    def stokes_operator(self, which, u, g=None, out=None):
        """ssg_stokes_operator: which 0 = double curl of u; 1 = pressure
        right-hand side of u~ = u and g (3 fields); 2 = velocity right-hand
        sides of u~ = u and the pressure g (no DSS)."""
        if out is None:
            sh = self.shape()
            out = np.empty(sh if which == 1 else (3,) + sh)
        self._check(self.lib.ssg_stokes_operator(self.h, int(which), _ptr(u),
                                                 _ptr(g) if g is not None else None,
                                                 _ptr(out)), "stokes_operator")
        return out

    def convection_elements(self, first, u, v, out=None):
        """ssg_convection_elements: convection of the elements first ..
        first + count - 1, fields shaped (3, count, n, n, n)."""
        out = self._out_like(u, out)
        self._check(self.lib.ssg_convection_elements(self.h, int(first), int(u.shape[1]),
                                                     _ptr(u), _ptr(v), _ptr(out)),
                    "convection_elements")
        return out

    def set_particle_velocity(self, ur):
        self._check(self.lib.ssg_set_particle_velocity(self.h, _ptr(ur)),
                    "set_particle_velocity")

    def integrate_particle_equations(self, state, ints, t, dt):
        passes = C.c_int()
        self._check(self.lib.ssg_integrate_particle_equations(
            self.h, state.shape[0], _ptr(state), _ptr(ints), t, dt, C.byref(passes)),
            "integrate_particle_equations")
        return state, ints, passes.value


# ---------------------------------------------------------------------------
# serving loop (ssg_server_*)
# ---------------------------------------------------------------------------
def request_bytes(n: int, nel: int, precision="mixed") -> int:
    """Admission estimate (bytes) of a request's resident context."""
    p = {"fp64": FP64, "mixed": MIXED}.get(precision, precision)
    return int(_lib.load().ssg_request_bytes(int(n), int(nel), int(p)))


def mesh_key(mesh, n: int) -> int:
    """Stable 64-bit identity of (mesh, order) for the server's context cache."""
    import hashlib
    h = hashlib.blake2b(digest_size=8)
    h.update(np.ascontiguousarray(mesh.vertices, dtype=np.float64).tobytes())
    h.update(np.ascontiguousarray(mesh.neigh, dtype=np.int32).tobytes())
    h.update(int(n).to_bytes(4, "little"))
    return int.from_bytes(h.digest(), "little") or 1


class Server:
    """Continuous-batching solve server on one GPU (ssg_server)."""

    def __init__(self, device: int = 0, hbm_budget: float = 150e9, max_active: int = 8):
        self.lib = _lib.load()
        h = C.c_void_p()
        st = self.lib.ssg_server_create(int(device), C.c_size_t(int(hbm_budget)),
                                        int(max_active), C.byref(h))
        if st != 0:
            raise SsgError(st, "ssg_server_create")
        self.h = h
        self._pending = {}

    def submit(self, mesh, n, rhs, lam=0.0, eps=1e-10, relative=False, precision="mixed",
               max_iter=0, deadline_ms=0.0, key=None):
        vert = np.ascontiguousarray(mesh.vertices, dtype=np.float64)
        neigh = np.ascontiguousarray(mesh.neigh, dtype=np.int32)
        rhs = np.ascontiguousarray(rhs, dtype=np.float64)
        out = np.zeros_like(rhs)
        r = _lib.Request()
        r.nel = int(mesh.nel)
        r.vertices = vert.ctypes.data_as(_lib._dp)
        r.neigh = neigh.ctypes.data_as(_lib._ip)
        r.mesh_key = int(mesh_key(mesh, n) if key is None else key)
        r.n = int(n)
        r.lam = float(lam)
        r.eps = float(eps)
        r.relative = int(bool(relative))
        r.precision = {"fp64": FP64, "mixed": MIXED}.get(precision, precision)
        r.max_iter = int(max_iter)
        r.deadline_ms = float(deadline_ms)
        rid = C.c_ulonglong()
        st = self.lib.ssg_server_submit(self.h, C.byref(r), rhs.ctypes.data_as(_lib._dp),
                                        out.ctypes.data_as(_lib._dp), C.byref(rid))
        if st != 0:
            raise SsgError(st, "ssg_server_submit")
        self._pending[rid.value] = out
        return rid.value

    def wait(self, rid, timeout_ms=-1.0):
        """(solution, status name, info) of request rid."""
        res = C.c_int()
        info = _lib.SolveInfo()
        st = self.lib.ssg_server_wait(self.h, C.c_ulonglong(rid), float(timeout_ms),
                                      C.byref(res), C.byref(info))
        if st != 0:
            raise SsgError(st, "ssg_server_wait")
        out = self._pending.pop(rid, None)
        return out, STATUS.get(res.value, res.value), {
            "iterations": info.iterations, "residual": info.residual,
            "initial_residual": info.initial_residual, "latency_ms": info.solve_ms}

    def set_batching(self, max_batch=16, max_points=65536):
        """ssg_server_set_batching: shared-launch batches of up to max_batch
        small (<= max_points points) Helmholtz requests of one order
        (max_batch 1: off, the default)."""
        self._check(self.lib.ssg_server_set_batching(self.h, int(max_batch),
                                                     C.c_size_t(int(max_points))),
                    "set_batching")

    def cancel(self, rid):
        self._check(self.lib.ssg_server_cancel(self.h, C.c_ulonglong(rid)), "cancel")

    def drain(self, timeout_ms=-1.0):
        self._check(self.lib.ssg_server_drain(self.h, float(timeout_ms)), "drain")

    def stats(self) -> dict:
        s = _lib.ServerStats()
        self._check(self.lib.ssg_server_get_stats(self.h, C.byref(s)), "stats")
        return {name: getattr(s, name) for name, _ in s._fields_}

    def _check(self, st, what):
        if st != 0:
            raise SsgError(st, what)

    def close(self):
        if getattr(self, "h", None):
            self.lib.ssg_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

