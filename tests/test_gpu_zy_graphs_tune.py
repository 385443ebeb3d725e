"""CUDA-graph replay of the V-cycle, of the outer FCG iterations (one graph
per window state, an IF node guarded by the device stop flag) and of the
Helmholtz CG loop (a WHILE node), and the launch-shape autotuner.

The captured graphs launch the same kernels with the same arguments as the
direct path, so a solve with graphs is bitwise the solve without.  The
autotuner changes only launch shapes: element-local results and the DSS stay
bitwise, while block-partial sums of the inner products may associate
differently, so solves are compared to the oracle at the usual tolerance.
(Named to run after the other GPU tests: the tuned shapes are process-wide.)
"""
import numpy as np
import pytest

import oracle as O
from conftest import assert_solution_close, same_stop
import ssenss_b200 as S
from ssenss_b200.mesh import channel_mesh, tgv_box

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def rhs(orc, n):
    X, Y, Z = orc.geometry(0, 7), orc.geometry(0, 8), orc.geometry(0, 9)
    g = 3.0 * np.cos(X + 0.3) * np.cos(Y + 0.7) * np.cos(Z + 1.1)
    x, w = orc.gll(n)
    rho = w[None, None, None, :] * w[None, None, :, None] * w[None, :, None, None]
    return orc.dss(rho * orc.geometry(0, 6) * g)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_graph_replay_is_bitwise_direct(precision, gpu_ctx_factory):
    mesh, n = tgv_box(3), 8
    orc = O.Oracle(mesh, n)
    f = rhs(orc, n)
    ctx = gpu_ctx_factory(mesh, n, precision=precision)
    ctx.set_graphs(False)
    u_d, info_d = ctx.solve_poisson_cg(f, np.zeros_like(f))
    ctx.set_graphs(True)
    runs = [ctx.solve_poisson_cg(f, np.zeros_like(f)) for _ in range(3)]
    for u_g, info_g in runs:      # warm-up run, capture run, replay run
        assert info_g["iterations"] == info_d["iterations"]
        assert np.array_equal(u_g, u_d)
        assert np.array_equal(info_g["history"], info_d["history"])


def test_graph_launch_count_is_kept(gpu_ctx_factory):
    """Replayed graphs count the kernels they run: the direct path's, plus
    one guard kernel per enqueued FCG iteration graph (16 are enqueued for a
    solve of at most 16 iterations)."""
    mesh, n = tgv_box(3), 6
    orc = O.Oracle(mesh, n)
    f = rhs(orc, n)
    ctx = gpu_ctx_factory(mesh, n)
    ctx.set_graphs(False)
    c0 = S.kernel_launch_count()
    _, info = ctx.solve_poisson_cg(f, np.zeros_like(f))
    direct = S.kernel_launch_count() - c0
    assert info["iterations"] <= 16
    ctx.set_graphs(True)
    ctx.solve_poisson_cg(f, np.zeros_like(f))      # warm-up of the V-cycle
    ctx.solve_poisson_cg(f, np.zeros_like(f))      # capture
    c0 = S.kernel_launch_count()
    ctx.solve_poisson_cg(f, np.zeros_like(f))      # replay
    assert S.kernel_launch_count() - c0 == direct + 16


def test_helmholtz_while_graph_is_bitwise_direct(gpu_ctx_factory):
    """The Helmholtz CG's iterations after the first as one WHILE graph node:
    the same iterations, solution and residual history as direct launches,
    on capture and on replay."""
    mesh, n = channel_mesh((4, 3, 3), seed=7), 7
    orc = O.Oracle(mesh, n)
    f = rhs(orc, n)
    # lambda = (11/6) / (dt visc) = 11/6: a stiffness-dominated operator, so
    # the Jacobi CG runs many iterations
    ctx = gpu_ctx_factory(mesh, n, dt=1.0, visc=1.0)
    ctx.set_graphs(False)
    u_d, info_d = ctx.solve_helmholtz_cg(O.X_VELOCITY, f, np.zeros_like(f))
    assert info_d["iterations"] > 8
    ctx.set_graphs(True)
    for _ in range(2):                             # capture, replay
        u_g, info_g = ctx.solve_helmholtz_cg(O.X_VELOCITY, f, np.zeros_like(f))
        assert info_g["iterations"] == info_d["iterations"]
        assert np.array_equal(u_g, u_d)
        assert np.array_equal(info_g["history"], info_d["history"])


@pytest.mark.parametrize("mk,n", [(lambda: tgv_box(3), 8),
                                  (lambda: channel_mesh((4, 3, 3), seed=7), 7)])
def test_autotuned_shapes_keep_parity(mk, n, gpu_ctx_factory):
    mesh = mk()
    orc = O.Oracle(mesh, n)
    ctx = gpu_ctx_factory(mesh, n)
    shapes = ctx.autotune(reps=3)
    assert set(shapes) == set(ctx.orders)
    for n_l, sh in shapes.items():
        assert sh["ax_elements_per_block"] == 0 if n_l == 8 else \
            sh["ax_elements_per_block"] in (-1, 1, 2, 4, 8, 16, 32, 64)
        assert 4 <= sh["dss_blocks_per_sm"] <= 64
        assert 2 <= sh["vector_blocks_per_sm"] <= 64
    rng = np.random.default_rng(9)
    u = rng.standard_normal((mesh.nel, n, n, n))
    assert np.array_equal(ctx.direct_stiffness_summation(u.copy()), orc.dss(u))
    assert rel(ctx.global_opeval(O.PRESSURE, u), orc.global_opeval(O.PRESSURE, u)) < 1e-13
    f = rhs(orc, n)
    u_o, h_o = orc.solve_poisson(f, np.zeros_like(f))
    u_g, info = ctx.solve_poisson_cg(f, np.zeros_like(f))
    if same_stop(info["iterations"], info["history"], h_o):
        assert_solution_close(u_g, u_o, orc, orc.solve_poisson, f)


def test_kernel_timing_entry_points(gpu_ctx_factory):
    """ssg_time_operator / ssg_time_smoother: positive device times for the
    operator and for the three smoother kernels at every level; a level out
    of range is an argument error.  They time scratch buffers only, so the
    operator afterwards still matches the oracle."""
    mesh, n = tgv_box(3), 8
    orc = O.Oracle(mesh, n)
    ctx = gpu_ctx_factory(mesh, n)
    assert ctx.time_operator(S.PRESSURE, 5) > 0.0
    assert ctx.time_operator(S.X_VELOCITY, 5) > 0.0
    for lev in range(len(ctx.orders)):
        t = ctx.time_smoother(lev, 5)
        assert set(t) == {"operator", "dss_dot", "cg_update"}
        assert all(v > 0.0 for v in t.values())
    with pytest.raises(S.SsgError):
        ctx.time_smoother(len(ctx.orders), 5)
    rng = np.random.default_rng(3)
    u = rng.standard_normal((mesh.nel, n, n, n))
    assert rel(ctx.global_opeval(O.PRESSURE, u), orc.global_opeval(O.PRESSURE, u)) < 1e-13
