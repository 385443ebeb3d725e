"""GPU parity of the solve path against the CPU oracle (oracle/ssg_oracle.c),
through the C ABI.

Tolerances: integer pairing and DSS are bitwise; element operators agree to
1e-13 relative (summation order and FMA differ from the oracle); solves stop
at the reference's absolute criterion sqrt((r.r)_w) <= 1e-10 and their
solutions agree to 1e-11 relative, or to twice the oracle's own rounding
spread where the solve is not determined that closely by FP64 arithmetic
(conftest.assert_solution_close; TGV 3^3 at n = 10 is such a case: one
rounding of the oracle's dot products moves its solution by 2e-11).
"""
import numpy as np
import pytest

import oracle as O
from conftest import assert_solution_close, same_stop
from ssenss_b200.mesh import box_mesh, channel_mesh, tgv_box

pytestmark = pytest.mark.gpu

CASES = {
    "tgv3_n8": (lambda: tgv_box(3), 8),
    "tgv4_n6": (lambda: tgv_box(4), 6),
    "channel433_n7": (lambda: channel_mesh((4, 3, 3), seed=7), 7),
    "periodic233_n5": (lambda: box_mesh((2, 3, 3)), 5),
    "tgv3_n10": (lambda: tgv_box(3), 10),
}

_cache = {}


def setup_case(name, gpu_ctx_factory):
    if name not in _cache:
        mk, n = CASES[name]
        mesh = mk()
        orc = O.Oracle(mesh, n)
        ctx = gpu_ctx_factory(mesh, n)
        _cache[name] = (mesh, n, orc, ctx)
    return _cache[name]


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def weights(n):
    x = np.empty(n)
    w = np.empty(n)
    L = O.Oracle.lib()
    L.og_gll(n, x.ctypes.data_as(O._dp), w.ctypes.data_as(O._dp))
    return x, w


def smooth_field(orc, kx=1.0, ky=1.0, kz=1.0, ph=(0.3, 0.7, 1.1)):
    X, Y, Z = orc.geometry(0, 7), orc.geometry(0, 8), orc.geometry(0, 9)
    return np.cos(kx * X + ph[0]) * np.cos(ky * Y + ph[1]) * np.cos(kz * Z + ph[2])


def weak_rhs(orc, g):
    n = orc.n
    _, w = weights(n)
    rho = w[None, None, None, :] * w[None, None, :, None] * w[None, :, None, None]
    return orc.dss(rho * orc.geometry(0, 6) * g)


@pytest.mark.parametrize("name", list(CASES))
def test_level_data_matches_oracle(name, gpu_ctx_factory):
    mesh, n, orc, ctx = setup_case(name, gpu_ctx_factory)
    assert ctx.orders == orc.orders
    for L in range(orc.nlevels):
        m = orc.orders[L]
        _, w = weights(m)
        rho = w[None, None, None, :] * w[None, None, :, None] * w[None, :, None, None]
        bj = rho * orc.geometry(L, 6)
        assert rel(ctx.level_data(L, 6), bj) < 1e-15
        for a in range(6):
            g = orc.geometry(L, a) * bj
            d = ctx.level_data(L, a)
            scale = max(np.max(np.abs(orc.geometry(L, 0) * bj)), 1e-300)
            assert np.max(np.abs(d - g)) / scale < 1e-14, (L, a)
        assert np.array_equal(ctx.level_data(L, 9), orc.precon(L, 2))   # 1/multiplicity
        assert np.array_equal(ctx.level_data(L, 10), orc.precon(L, 3))  # mask
        assert rel(ctx.level_data(L, 7), orc.precon(L, 0)) < 1e-14      # Poisson diag
    assert rel(ctx.level_data(0, 8), orc.precon(0, 1)) < 1e-14          # Helmholtz diag
    assert rel(ctx.level_data(0, 11), orc.precon(0, 4)) < 1e-14         # inverse mass


@pytest.mark.parametrize("name", list(CASES))
def test_inverse_mass_matches_oracle(name, gpu_ctx_factory):
    """ssg_inverse_mass (global_inverse_mass_matrix_operator,
    src/poisson.c:77-87): u times the stored inverse assembled mass, one
    rounding per point -- bit for bit the product with the context's own
    inverse mass, and within 1e-14 of the oracle's; host and device
    operands."""
    import torch
    mesh, n, orc, ctx = setup_case(name, gpu_ctx_factory)
    rng = np.random.default_rng(4)
    u = rng.standard_normal((mesh.nel, n, n, n))
    own = u * ctx.level_data(0, 11)
    got = ctx.inverse_mass(u.copy())
    assert np.array_equal(got, own)
    assert rel(got, u * orc.precon(0, 4)) < 1e-14
    ud = torch.from_numpy(u).cuda()
    ctx.inverse_mass(ud)
    torch.cuda.synchronize()
    assert np.array_equal(ud.cpu().numpy(), own)


@pytest.mark.parametrize("name", list(CASES))
def test_dss_bitwise(name, gpu_ctx_factory):
    mesh, n, orc, ctx = setup_case(name, gpu_ctx_factory)
    rng = np.random.default_rng(1)
    u = rng.standard_normal((mesh.nel, n, n, n))
    got = ctx.direct_stiffness_summation(u.copy())
    assert np.array_equal(got, orc.dss(u))


@pytest.mark.parametrize("name", list(CASES))
@pytest.mark.parametrize("var", [O.PRESSURE, O.X_VELOCITY])
def test_operator_matches_oracle(name, var, gpu_ctx_factory):
    mesh, n, orc, ctx = setup_case(name, gpu_ctx_factory)
    rng = np.random.default_rng(2)
    p = rng.standard_normal((mesh.nel, n, n, n))
    assert rel(ctx.local_opeval(var, p), orc.local_opeval(var, p)) < 1e-13
    assert rel(ctx.global_opeval(var, p), orc.global_opeval(var, p)) < 1e-13


@pytest.mark.parametrize("name", list(CASES))
def test_dot_matches_oracle(name, gpu_ctx_factory):
    mesh, n, orc, ctx = setup_case(name, gpu_ctx_factory)
    rng = np.random.default_rng(3)
    x = rng.standard_normal((mesh.nel, n, n, n))
    y = rng.standard_normal((mesh.nel, n, n, n))
    a, b = ctx.global_dot_product(x, y), orc.dot(x, y)
    assert abs(a - b) <= 1e-12 * np.sqrt(orc.dot(x, x) * orc.dot(y, y))


@pytest.mark.parametrize("name", ["tgv3_n8", "channel433_n7", "tgv3_n10"])
def test_multigrid_preconditioner(name, gpu_ctx_factory):
    mesh, n, orc, ctx = setup_case(name, gpu_ctx_factory)
    r = weak_rhs(orc, smooth_field(orc))
    z_o = orc.mg_precon(r)
    z_g = ctx.multigrid_preconditioner(r)
    assert rel(z_g, z_o) < 1e-9


# periodic233_n5 (two elements along a periodic direction) carries the
# reference's face-pairing defect: its operator is not a consistent Laplacian
# and FCG plateaus, so it is pinned by the bitwise DSS and operator tests
# only, not by iteration counts.
@pytest.mark.parametrize("name", ["tgv3_n8", "tgv4_n6", "channel433_n7", "tgv3_n10"])
def test_poisson_solve(name, gpu_ctx_factory):
    mesh, n, orc, ctx = setup_case(name, gpu_ctx_factory)
    f = weak_rhs(orc, 3.0 * smooth_field(orc))
    u0 = np.zeros_like(f)
    u_o, h_o = orc.solve_poisson(f, u0)
    u_g, info = ctx.solve_poisson_cg(f, u0.copy())
    assert info["status"] == "SSG_OK"
    assert info["residual"] <= 1e-10
    if same_stop(info["iterations"], info["history"], h_o):
        assert_solution_close(u_g, u_o, orc, orc.solve_poisson, f)
    # residual histories: while the residual is well above the rounding floor
    # they agree to 1e-9 relative; near eps the floor itself differs between
    # any two FP64 implementations (the oracle and the reference build differ
    # there too), so the bound is 1e-9 of the first residual
    # (the inner CG solves of the V-cycle stop on the same absolute eps, so
    # once residuals near it a one-iteration shift of an inner solve moves
    # the outer history by up to ~1e-7 of the first residual)
    h_g = info["history"]
    k = min(len(h_g), len(h_o))
    h_g, h_o = h_g[:k], h_o[:k]
    assert np.all(np.abs(h_g - h_o) <= 1e-7 * h_o[0])
    lead = h_o > 1e-4 * h_o[0]
    assert np.all(np.abs(h_g - h_o)[lead] <= 1e-9 * h_o[lead])


@pytest.mark.parametrize("name", ["tgv3_n8", "channel433_n7", "tgv4_n6"])
@pytest.mark.parametrize("var", [O.X_VELOCITY, O.Z_VELOCITY])
def test_helmholtz_solve(name, var, gpu_ctx_factory):
    mesh, n, orc, ctx = setup_case(name, gpu_ctx_factory)
    f = weak_rhs(orc, smooth_field(orc))
    u0 = np.zeros_like(f)
    u_o, h_o = orc.solve_helmholtz(var, f, u0)
    u_g, info = ctx.solve_helmholtz_cg(var, f, u0.copy())
    assert info["status"] == "SSG_OK"
    assert info["iterations"] == len(h_o)
    assert rel(u_g, u_o) < 1e-12
    assert np.all(np.abs(info["history"] - h_o) <= 1e-9 * h_o[0])


@pytest.mark.parametrize("name", ["tgv3_n8", "channel433_n7"])
def test_jacobi_preconditioner_bitwise(name, gpu_ctx_factory):
    """z = r .* diag^-1: one product per point, so bitwise r times the
    context's stored diagonal inverse, and within the diagonals' own 1e-14
    (Poisson) / 1e-13 (Helmholtz) of the oracle's."""
    mesh, n, orc, ctx = setup_case(name, gpu_ctx_factory)
    rng = np.random.default_rng(17)
    r = rng.standard_normal((mesh.nel, n, n, n))
    z = ctx.jacobi_preconditioner(O.PRESSURE, r)
    assert np.array_equal(z, r * ctx.level_data(0, 7))
    assert rel(z, r * orc.precon(0, 0)) < 1e-14
    z = ctx.jacobi_preconditioner(O.Y_VELOCITY, r)
    assert np.array_equal(z, r * ctx.level_data(0, 8))
    assert rel(z, r * orc.precon(0, 1)) < 1e-13


def test_device_pointers(gpu_ctx_factory):
    """CUDA tensors are used in place (no staging)."""
    import torch
    mesh, n, orc, ctx = setup_case("tgv3_n8", gpu_ctx_factory)
    rng = np.random.default_rng(4)
    p = rng.standard_normal((mesh.nel, n, n, n))
    pd = torch.from_numpy(p).cuda()
    out = ctx.global_opeval(O.PRESSURE, pd)
    torch.cuda.synchronize()
    assert rel(out.cpu().numpy(), orc.global_opeval(O.PRESSURE, p)) < 1e-13


@pytest.mark.parametrize("name", ["tgv3_n8", "channel433_n7"])
def test_mixed_precision_solve(name, gpu_ctx_factory):
    """FP32 V-cycle inside the FP64 FCG reaches the same 1e-10 residual; the
    solution differs from the FP64 oracle only by the solver tolerance."""
    mk, n = CASES[name]
    mesh = mk()
    orc = O.Oracle(mesh, n)
    ctx = gpu_ctx_factory(mesh, n, precision="mixed")
    f = weak_rhs(orc, 3.0 * smooth_field(orc))
    u0 = np.zeros_like(f)
    u_o, h_o = orc.solve_poisson(f, u0)
    u_g, info = ctx.solve_poisson_cg(f, u0.copy())
    assert info["status"] == "SSG_OK"
    assert info["residual"] <= 1e-10
    assert info["iterations"] <= len(h_o) + 3
    assert rel(u_g, u_o) < 1e-8


@pytest.mark.parametrize("svv", [(3, 1.5), (-1, 0.3)])
def test_svv_helmholtz(svv):
    """Spectral vanishing viscosity on (ssg_set_svv before the set-up): the
    Helmholtz operator to 1e-13 and the Jacobi-CG Helmholtz solve (same
    iteration count, solution 1e-12, history 1e-9 of the first residual)
    against the oracle set up with the same svvn and svva (the oracle's SVV
    matrices are pinned to the reference's in tests/test_oracle_pins.py)."""
    import ssenss_b200 as S
    mesh, n = channel_mesh((4, 3, 3), seed=7), 8
    orc = O.Oracle(mesh, n, svv=svv)
    ctx = S.Context(0)
    try:
        ctx.set_parameters(1e-3, 1.0 / 1600.0, 1.0)
        ctx.set_svv(*svv)
        ctx.setup_mesh(mesh, n)
        rng = np.random.default_rng(41)
        u = rng.standard_normal((mesh.nel, n, n, n))
        for var in (O.X_VELOCITY, O.Y_VELOCITY):
            assert rel(ctx.global_opeval(var, u), orc.global_opeval(var, u)) < 1e-13
        f = weak_rhs(orc, smooth_field(orc))
        u0 = np.zeros_like(f)
        u_o, h_o = orc.solve_helmholtz(O.X_VELOCITY, f, u0)
        u_g, info = ctx.solve_helmholtz_cg(O.X_VELOCITY, f, u0.copy())
        assert info["status"] == "SSG_OK"
        assert info["iterations"] == len(h_o)
        assert rel(u_g, u_o) < 1e-12
        assert np.all(np.abs(info["history"] - h_o) <= 1e-9 * h_o[0])
    finally:
        ctx.close()
        orc.close()
