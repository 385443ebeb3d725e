"""GPU parity of the dealiased convection operator and the Lagrangian particle
walk against the CPU oracle (oracle/ssg_oracle.c), through the C ABI.

Convection is FP64 tensor-product arithmetic in another summation order:
1e-13 relative to the largest entry.  The particle walk is compiled without
FMA contraction and in the reference's operation order, so given the same
GLL points, factors and velocity snapshots every particle's element ids,
status, reference coordinates, velocity and time are bitwise the oracle's
(and the oracle's are bitwise the reference's for n > 5: see
tests/test_oracle_pins.py).
"""
import numpy as np
import pytest

import oracle as O
from ssenss_b200.mesh import box_mesh, channel_mesh, tgv_box

pytestmark = pytest.mark.gpu

CONV_CASES = {
    # m = 12, 15: per-element fields held in shared memory
    "tgv3_n8": (lambda: tgv_box(3), 8),
    "channel433_n7": (lambda: channel_mesh((4, 3, 3), seed=7), 7),
    "tgv3_n10": (lambda: tgv_box(3), 10),
    # m = 18: per-element fields in the global scratch region
    "tgv2_n12": (lambda: tgv_box(2), 12),
    "tgv4_n4": (lambda: tgv_box(4), 4),
}

_cache = {}


def case(name, factory, table):
    key = (name, table[name][1])
    if key not in _cache:
        mk, n = table[name]
        mesh = mk()
        _cache[key] = (mesh, n, O.Oracle(mesh, n), factory(mesh, n))
    return _cache[key]


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.mark.parametrize("name", list(CONV_CASES))
def test_convection_matches_oracle(name, gpu_ctx_factory):
    mesh, n, orc, ctx = case(name, gpu_ctx_factory, CONV_CASES)
    rng = np.random.default_rng(11)
    u = rng.standard_normal((3, mesh.nel, n, n, n))
    v = rng.standard_normal((3, mesh.nel, n, n, n))
    got = ctx.convection_operator(u, v)
    assert rel(got, orc.convection(u, v)) < 1e-13


SELF_CASES = {
    # n = 8 (m = 12): the self-convection tensor-core kernel
    "tgv3_n8": (lambda: tgv_box(3), 8),
    "channel433_n8": (lambda: channel_mesh((4, 3, 3), seed=7), 8),
}


@pytest.mark.parametrize("name", list(SELF_CASES))
def test_self_convection_matches_oracle(name, gpu_ctx_factory):
    """convection_operator(u, u), the time step's history term: at n = 8 the
    self-convection kernel, against the oracle and against the general
    kernel (a copy of u as the advected field) on the same inputs."""
    mesh, n, orc, ctx = case(name, gpu_ctx_factory, SELF_CASES)
    rng = np.random.default_rng(21)
    u = rng.standard_normal((3, mesh.nel, n, n, n))
    got = ctx.convection_operator(u, u)
    ref = orc.convection(u, u)
    assert rel(got, ref) < 1e-13
    general = ctx.convection_operator(u, u.copy())
    assert rel(general, ref) < 1e-13
    assert rel(got, general) < 1e-13
    # element ranges: elements 5 .. 5 + 7 of the mesh, fields of that range
    sub = np.ascontiguousarray(u[:, 5:12])
    part = ctx.convection_elements(5, sub, sub)
    assert rel(part, ref[:, 5:12]) < 1e-13
    one = np.ascontiguousarray(u[:, 3:4])
    assert rel(ctx.convection_elements(3, one, one), ref[:, 3:4]) < 1e-13


def test_self_convection_device_tensors_large(gpu_ctx_factory):
    """Self-convection of device tensors on a mesh with more elements than
    the persistent grid (2 blocks per SM), so blocks take several elements."""
    import torch
    mesh = tgv_box(8)
    n = 8
    orc = O.Oracle(mesh, n)
    ctx = gpu_ctx_factory(mesh, n)
    rng = np.random.default_rng(22)
    u = rng.standard_normal((3, mesh.nel, n, n, n))
    ud = torch.from_numpy(u).cuda()
    out = ctx.convection_operator(ud, ud)
    torch.cuda.synchronize()
    assert rel(out.cpu().numpy(), orc.convection(u, u)) < 1e-13


def test_convection_device_tensors(gpu_ctx_factory):
    import torch
    mesh, n, orc, ctx = case("tgv3_n8", gpu_ctx_factory, CONV_CASES)
    X = [orc.geometry(0, 7 + c) for c in range(3)]
    u = np.stack([np.sin(X[0]) * np.cos(X[1]), -np.cos(X[0]) * np.sin(X[1]), 0 * X[2]])
    ud = torch.from_numpy(u).cuda()
    out = ctx.convection_operator(ud, ud)
    torch.cuda.synchronize()
    assert rel(out.cpu().numpy(), orc.convection(u, u)) < 1e-13


def test_convection_drop_in_setup(gpu_ctx_factory):
    """ssg_setup_dealias with the caller's stored factors gives the same
    operator as the library's own dealiasing grid."""
    mesh, n, orc, ctx = case("channel433_n7", gpu_ctx_factory, CONV_CASES)
    m = (3 * n) // 2
    x, w = orc.gll(m)
    xn, _ = orc.gll(n)
    L = O.Oracle.lib()
    D = np.empty((m, m))
    L.og_deriv(m, O._d(x), O._d(D))            # D[i, j] = l_j'(x_i)
    J = np.empty((m, n))
    L.og_interp(m, O._d(x), n, O._d(xn), O._d(J))   # J[i, p] = l_p(x_i)
    tinv = np.stack([orc.conv_geometry(a) for a in range(9)])
    det = orc.conv_geometry(9)
    ctx.setup_dealias(m, D.T.copy(), w, tinv, det, J.T.copy())
    rng = np.random.default_rng(12)
    u = rng.standard_normal((3, mesh.nel, n, n, n))
    v = rng.standard_normal((3, mesh.nel, n, n, n))
    assert rel(ctx.convection_operator(u, v), orc.convection(u, v)) < 1e-13


# --------------------------------------------------------------------------
# particles
# --------------------------------------------------------------------------
PART_CASES = {
    # dt, speed: particles cross several element faces per call
    "tgv3_n8": (lambda: tgv_box(3), 8, 0.05, 20.0),
    "channel433_n7": (lambda: channel_mesh((4, 3, 3), seed=7), 7, 0.05, 20.0),
    # n <= 5: full tensor Lagrange interpolation
    "tgv3_n5": (lambda: tgv_box(3), 5, 0.05, 20.0),
    # two elements per periodic direction: the entry-face search is
    # ambiguous and many particles end with the reseed status
    "tgv2_n10": (lambda: tgv_box(2), 10, 0.05, 20.0),
    # walls on the channel's y faces: collisions reverse the normal velocity
    "walls333_n6": (lambda: box_mesh((3, 3, 3), periodic=(True, False, True)),
                    6, 0.05, 30.0),
}


def particle_inputs(orc, mesh, n, dt, speed, npart, seed):
    t = 0.1
    X = [orc.geometry(0, 7 + c) for c in range(3)]
    ur = np.empty((3, 3, mesh.nel, n, n, n))
    for lev in range(3):
        tt = t - (2 - lev) * dt
        ur[lev, 0] = 3.0 * np.sin(X[0] + tt) * np.cos(X[1])
        ur[lev, 1] = -3.0 * np.cos(X[0]) * np.sin(X[1] + 2 * tt)
        ur[lev, 2] = 2.0 * np.cos(X[2] + tt)
    rng = np.random.default_rng(seed)
    state = np.zeros((npart, 8))
    ints = np.zeros((npart, 3), np.int32)
    state[:, :3] = rng.uniform(-0.99, 0.99, (npart, 3))
    state[:, 3:6] = rng.standard_normal((npart, 3)) * speed
    state[:, 6] = t - dt
    state[:, 7] = rng.uniform(0.05, 2.0, npart)
    ints[:, 0] = rng.integers(0, mesh.nel, npart)
    ints[:, 1] = ints[:, 0]
    return t, ur, state, ints


@pytest.mark.parametrize("name", list(PART_CASES))
def test_particles_bitwise(name, gpu_ctx_factory):
    mk, n, dt, speed = PART_CASES[name]
    mesh, n, orc, ctx = case(name, gpu_ctx_factory, {name: (mk, n)})
    pts, jac, tinv = orc.particle_geometry()
    ctx.setup_particle_geometry(pts, jac, tinv)
    t, ur, state, ints = particle_inputs(orc, mesh, n, dt, speed, 2000, 5)
    orc.set_params(t, dt, 1.0 / 1600.0)
    s_o, i_o, p_o = orc.particles_advance(state, ints, ur)
    ctx.set_particle_velocity(ur)
    s_g, i_g, p_g = ctx.integrate_particle_equations(state.copy(), ints.copy(), t, dt)
    moved = int(np.sum(i_o[:, 0] != ints[:, 0]))
    assert moved > 0
    assert p_g == p_o
    assert np.array_equal(i_g, i_o)
    assert np.array_equal(s_g.view(np.uint64), s_o.view(np.uint64))


def test_particles_device_arrays(gpu_ctx_factory):
    import torch
    mk, n, dt, speed = PART_CASES["tgv3_n8"]
    mesh, n, orc, ctx = case("tgv3_n8", gpu_ctx_factory, {"tgv3_n8": (mk, n)})
    pts, jac, tinv = orc.particle_geometry()
    ctx.setup_particle_geometry(pts, jac, tinv)
    t, ur, state, ints = particle_inputs(orc, mesh, n, dt, speed, 5000, 6)
    orc.set_params(t, dt, 1.0 / 1600.0)
    s_o, i_o, p_o = orc.particles_advance(state, ints, ur)
    ctx.set_particle_velocity(torch.from_numpy(ur).cuda())
    sd = torch.from_numpy(state).cuda()
    idv = torch.from_numpy(ints).cuda()
    _, _, p_g = ctx.integrate_particle_equations(sd, idv, t, dt)
    torch.cuda.synchronize()
    assert p_g == p_o
    assert np.array_equal(idv.cpu().numpy(), i_o)
    assert np.array_equal(sd.cpu().numpy().view(np.uint64), s_o.view(np.uint64))


def test_particles_empty_and_invalid(gpu_ctx_factory):
    mk, n, dt, speed = PART_CASES["tgv3_n8"]
    mesh, n, orc, ctx = case("tgv3_n8", gpu_ctx_factory, {"tgv3_n8": (mk, n)})
    ctx.set_particle_velocity(np.zeros((3, 3, mesh.nel, n, n, n)))
    s = np.zeros((0, 8))
    i = np.zeros((0, 3), np.int32)
    _, _, passes = ctx.integrate_particle_equations(s, i, 0.1, dt)
    assert passes == 1
    # an element id outside the mesh is reported for a reseed, untouched
    s = np.zeros((2, 8))
    s[:, 7] = 1.0
    i = np.array([[mesh.nel, 0, 0], [-1, 0, 0]], np.int32)
    s_g, i_g, _ = ctx.integrate_particle_equations(s.copy(), i.copy(), 0.1, dt)
    assert list(i_g[:, 2]) == [5, 5]
    assert np.array_equal(s_g, s)
