"""Regenerate the golden fixtures (tests/golden/*.npz) from the reference
itself: the unmodified SSENSS sources compiled by oracle/Makefile into
oracle/_ref/libssenss_ref.so.

    make -C oracle && python tests/golden/make_golden.py

Per case (golden_inputs.CASES) the fixture holds the reference's outputs on
inputs that golden_inputs.py rebuilds exactly:

  dss         direct_stiffness_summation of hash field u      (bitwise)
  op_p, op_h  global_opeval, Poisson / Helmholtz (x velocity), of u
  dot         global_dot_product(u, v)
  f           weak right-hand side DSS(rho J g), g a hash field
  sol_p, it_p, hist_p   flexible CG + p-multigrid Poisson solve of f
  sol_h, it_h, hist_h   Jacobi CG Helmholtz solve of f (x velocity)
  mg          one multigrid_preconditioner application to f
  conv        convection_operator(u3, v3), hash-field vectors
and for the particle case the reference's GLL points and its particle walk
(integrate_particle_equations) from golden_inputs.particle_states on the
factors of golden_inputs.particle_factors.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
sys.path.insert(0, HERE)

import oracle as O  # noqa: E402
import golden_inputs as G  # noqa: E402

NPART = 600


def make(name):
    mk, n = G.CASES[name]
    mesh = mk()
    ref = O.Reference(mesh, n, dt=G.DT, visc=G.VISC, dens=G.DENS)
    ref.set_params(0.0, G.DT, G.VISC)
    shp = (mesh.nel, n, n, n)
    u = G.hash_field(shp, 1)
    v = G.hash_field(shp, 2)
    out = {"n": n, "nel": mesh.nel, "orders": np.array(ref.orders)}
    out["dss"] = ref.dss(u)
    out["op_p"] = ref.global_opeval(O.PRESSURE, u)
    out["op_h"] = ref.global_opeval(O.X_VELOCITY, u)
    out["dot"] = ref.dot(u, v)
    x, w = ref.basis(0)[:2]
    rho = w[None, None, None, :] * w[None, None, :, None] * w[None, :, None, None]
    f = ref.dss(rho * ref.geometry(0, 6) * G.hash_field(shp, 3))
    out["f"] = f
    sol, hist = ref.solve_poisson(f, np.zeros(shp))
    out["sol_p"], out["hist_p"], out["it_p"] = sol, hist, len(hist)
    sol, hist = ref.solve_helmholtz(O.X_VELOCITY, f, np.zeros(shp))
    out["sol_h"], out["hist_h"], out["it_h"] = sol, hist, len(hist)
    out["mg"] = ref.mg_precon(f)
    u3 = G.hash_field((3,) + shp, 4)
    v3 = G.hash_field((3,) + shp, 5)
    out["conv"] = ref.convection(u3, v3)
    if name == G.PARTICLE_CASE:
        jac, tinv = G.particle_factors(mesh, n)
        ref.set_particle_factors(jac, tinv)
        ref.set_params(G.PART_T, G.PART_DT, G.VISC)
        ur = G.particle_velocity(mesh, x, G.PART_T, G.PART_DT)
        state, ints = G.particle_states(mesh, NPART, 7)
        s, i = ref.particles_advance(state, ints, ur)
        out["points"] = x
        out["p_state"], out["p_ints"] = s, i
    path = os.path.join(HERE, f"{name}.npz")
    np.savez_compressed(path, **out)
    print(name, os.path.getsize(path), "bytes;", "iters", out["it_p"], out["it_h"])


if __name__ == "__main__":
    if not O.reference_available():
        sys.exit("oracle/_ref/libssenss_ref.so missing: run make -C oracle first")
    for name in G.CASES:
        make(name)
