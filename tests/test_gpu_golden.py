"""GPU path against the reference's own outputs (tests/golden/*.npz, written
by tests/golden/make_golden.py from the reference compiled in place), through
the C ABI.  Same bars as the oracle pins: DSS and the particle walk bitwise,
operators and the inner product 1e-13, solve iteration counts exact and
solutions 1e-11 (Helmholtz 1e-12), multigrid 1e-9, convection 1e-13.
"""
import os
import sys

import numpy as np
import pytest

import oracle as O
from conftest import same_stop

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import golden_inputs as G  # noqa: E402

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


_ctx = {}


def golden_case(name, factory):
    if name not in _ctx:
        mk, n = G.CASES[name]
        mesh = mk()
        ctx = factory(mesh, n, dt=G.DT, visc=G.VISC)
        g = dict(np.load(os.path.join(HERE, "golden", f"{name}.npz")))
        _ctx[name] = (mesh, n, ctx, g)
    return _ctx[name]


@pytest.mark.parametrize("name", list(G.CASES))
def test_golden_operators(name, gpu_ctx_factory):
    mesh, n, ctx, g = golden_case(name, gpu_ctx_factory)
    assert ctx.orders == list(g["orders"])
    shp = (mesh.nel, n, n, n)
    u, v = G.hash_field(shp, 1), G.hash_field(shp, 2)
    assert np.array_equal(ctx.direct_stiffness_summation(u.copy()), g["dss"])
    assert rel(ctx.global_opeval(O.PRESSURE, u), g["op_p"]) < 1e-13
    assert rel(ctx.global_opeval(O.X_VELOCITY, u), g["op_h"]) < 1e-13
    assert abs(ctx.global_dot_product(u, v) - float(g["dot"])) <= 1e-13 * float(
        ctx.global_dot_product(u, u))
    u3, v3 = G.hash_field((3,) + shp, 4), G.hash_field((3,) + shp, 5)
    assert rel(ctx.convection_operator(u3, v3), g["conv"]) < 1e-13


@pytest.mark.parametrize("name", list(G.CASES))
def test_golden_solves(name, gpu_ctx_factory):
    mesh, n, ctx, g = golden_case(name, gpu_ctx_factory)
    f = g["f"]
    sol, info = ctx.solve_poisson_cg(f, np.zeros_like(f))
    assert info["status"] == "SSG_OK"
    if same_stop(info["iterations"], info["history"], g["hist_p"]):
        assert rel(sol, g["sol_p"]) < 1e-11
    k = min(info["iterations"], int(g["it_p"]))
    assert np.all(np.abs(info["history"][:k] - g["hist_p"][:k]) <= 1e-7 * g["hist_p"][0])
    sol, info = ctx.solve_helmholtz_cg(O.X_VELOCITY, f, np.zeros_like(f))
    assert info["iterations"] == int(g["it_h"])
    assert rel(sol, g["sol_h"]) < 1e-12
    assert rel(ctx.multigrid_preconditioner(f), g["mg"]) < 1e-9


def test_golden_particles_bitwise(gpu_ctx_factory):
    name = G.PARTICLE_CASE
    mesh, n, ctx, g = golden_case(name, gpu_ctx_factory)
    jac, tinv = G.particle_factors(mesh, n)
    ctx.setup_particle_geometry(g["points"], jac, tinv)
    ctx.set_particle_velocity(G.particle_velocity(mesh, g["points"], G.PART_T, G.PART_DT))
    state, ints = G.particle_states(mesh, g["p_state"].shape[0], 7)
    s, i, _ = ctx.integrate_particle_equations(state.copy(), ints.copy(), G.PART_T, G.PART_DT)
    done = g["p_ints"][:, 2] == 0
    assert np.sum(i[:, 0] != ints[:, 0]) > 100
    assert np.array_equal(i[:, 2] == 0, done)
    assert np.array_equal(i[done], g["p_ints"][done])
    assert np.array_equal(s[done].view(np.uint64), g["p_state"][done].view(np.uint64))


@pytest.mark.skipif(not O.reference_available(), reason="reference library not built")
def test_drop_in_setup_from_reference_arrays(gpu_ctx_factory):
    """Context set up through ssg_setup_connectivity / ssg_setup_level /
    ssg_setup_finish from the reference's own stored arrays (what a caller linking the library into the reference hands
    over) reproduces the reference's operator and Poisson solve."""
    import ssenss_b200 as S
    mk, n = G.CASES["channel433_n5"]
    mesh = mk()
    ref = O.Reference(mesh, n, dt=G.DT, visc=G.VISC, dens=G.DENS)
    ctx = S.Context(0)
    try:
        ctx.set_parameters(G.DT, G.VISC, G.DENS)
        ctx.setup_connectivity(mesh.neigh)
        for lev, m in enumerate(ref.orders):
            x, w, d, s = ref.basis(lev)         # d, s: D[i, j] (transposed from storage)
            geom = np.stack([ref.geometry(lev, a) for a in range(6)])
            interp = ref.interp(lev).T.copy() if lev > 0 else None   # [p_coarse, i_fine]
            ctx.setup_level(lev, m, d.T.copy(), s.T.copy(), w, geom, ref.geometry(lev, 6),
                            interp)
        ctx.setup_finish()
        shp = (mesh.nel, n, n, n)
        u = G.hash_field(shp, 1)
        assert np.array_equal(ctx.direct_stiffness_summation(u.copy()), ref.dss(u))
        assert rel(ctx.global_opeval(O.PRESSURE, u), ref.global_opeval(O.PRESSURE, u)) < 1e-13
        rng = np.random.default_rng(1)
        f = ref.dss(rng.standard_normal(shp))
        sol_r, hist_r = ref.solve_poisson(f, np.zeros(shp))
        sol_g, info = ctx.solve_poisson_cg(f, np.zeros(shp))
        if same_stop(info["iterations"], info["history"], hist_r):
            assert rel(sol_g, sol_r) < 1e-11
    finally:
        ctx.close()
