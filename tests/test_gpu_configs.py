"""Parity at the benchmark configurations' own sizes, against the reference
compiled in place (oracle/_ref), run live on the same machine.

C2  the bench's headline solve: TGV periodic 16^3 elements, N = 7 (n = 8,
    2,097,152 points), pressure Poisson right-hand side of the TGV pressure,
    FCG + p-multigrid to the absolute 1e-10, from zero -- FP64, through the
    library's own set-up (the bench's path).  The reference's residual
    history on this machine is also pinned by tests/golden/c2_tgv16_n8.json.
C3  the deformed channel at N = 9 (n = 10) on a reduced 8 x 4 x 4 mesh with
    the configuration's stretch (tanh 2.0), perturbation (0.1 of the local
    spacing) and seed; 8 seeded Fourier modes, Neumann-compatible, mean zero.
C4  20,000 particles in the 16^3 N = 7 TGV flow, 100 calls of
    integrate_particle_equations over 2 dt each (the reference's cadence) on
    frozen velocity snapshots, every particle's element id and state compared
    bit for bit after every 10th call and at the end.

Bars: iteration counts equal, or one apart only where the stop lies within a
factor 2 of eps at the deciding iteration (conftest.same_stop); residual
histories within 1e-9 of the first residual wherever both are above 1e-4 of
it (the 15-iteration inner CG solves of the V-cycle stop on the same
absolute eps, so near the end of a solve two FP64 implementations take
different inner iteration counts and their outer residuals drift apart at
that level -- measured, not assumed: the oracle against the reference shows
the same), within 1e-7 of it below; solutions 1e-11 relative to the largest
entry (conftest.assert_solution_close); mixed precision 1e-8 against the
FP64 reference solution.
"""
import json
import math
import os

import numpy as np
import pytest

import oracle as O
import ssenss_b200 as S
from conftest import EPS, assert_solution_close, check_history, history_deviation, same_stop
from ssenss_b200.mesh import channel_mesh, tgv_box

HERE = os.path.dirname(os.path.abspath(__file__))
pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not O.reference_available(), reason="reference library not built")]


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def tgv_pressure_rhs(ref, n):
    """Weak, assembled -lap p of the TGV pressure on the reference's own grid
    (what compute_pressure_rhs assembles for this p)."""
    x, w, _, _ = ref.basis(0)
    X, Y, Z = (ref.geometry(0, 7 + a) for a in range(3))
    rho = w[None, None, None, :] * w[None, None, :, None] * w[None, :, None, None]
    c2x, c2y, c2z = np.cos(2 * X), np.cos(2 * Y), np.cos(2 * Z)
    lap = (-4.0 * (c2x + c2y) * (c2z + 2.0) - 4.0 * (c2x + c2y) * c2z) / 16.0
    return ref.dss(rho * ref.geometry(0, 6) * (-lap))


def test_c2_pressure_solve_full_size():
    """C2 at its own size.  The reference's FCG is sensitive to rounding:
    its V-cycle's inner CG solves stop on the absolute eps, so a rounding
    change moves their iteration counts and the outer iterates move by more
    than rounding.  Measured here: the reference on this machine against its
    own record from the machine that wrote tests/golden/c2_tgv16_n8.json
    (OpenBLAS picks CPU-specific kernels) -- the same 11 iterations, with
    history deviations up to ~2e-4 of the first residual.  So the GPU solve
    is held to: the same stop (conftest.same_stop); its history within
    twice that measured machine-to-machine spread (or 1e-9 of the first
    residual where the spread is smaller); and its solution solving the
    reference's own discrete system to the stop criterion: the reference's
    operator gives it a residual sqrt((r.r)_w) <= 1.5 eps.  The relative
    solution difference is reported.  The spread is the larger of the two
    measured ones: the reference against its record, and the reference
    against the oracle (oracle/ssg_oracle.c, a second FP64 implementation of
    the same algorithm) on this machine."""
    mesh, n = tgv_box(16), 8
    ref = O.Reference(mesh, n)
    try:
        f = tgv_pressure_rhs(ref, n)
        u_r, h_r = ref.solve_poisson(f, np.zeros_like(f))
        ctx = S.Context(0)
        try:
            ctx.set_parameters(1e-3, 1.0 / 1600.0, 1.0)
            ctx.set_setup_options(no_dealias=True, no_particles=True)
            ctx.setup_mesh(mesh, n)
            u_g, info = ctx.solve_poisson_cg(f, np.zeros_like(f))
        finally:
            ctx.close()
        r = f - ref.global_opeval(O.PRESSURE, u_g)
        res_ref_op = float(np.sqrt(ref.dot(r, r)))
    finally:
        ref.close()
    # a second FP64 implementation of the same algorithm: the oracle
    orc = O.Oracle(mesh, n)
    try:
        _, h_o = orc.solve_poisson(f, np.zeros_like(f))
    finally:
        orc.close()
    pin = json.load(open(os.path.join(HERE, "golden", "c2_tgv16_n8.json")))
    k0 = min(len(h_r), len(h_o), len(pin["history"]))
    spread = np.maximum(history_deviation(h_r, pin["history"])[:k0],
                        history_deviation(h_r, h_o)[:k0])
    dev = history_deviation(info["history"], h_r)
    h0 = h_r[0]
    d = rel(u_g, u_r)
    print(f"C2 full size: GPU {info['iterations']} vs reference {len(h_r)} iterations "
          f"(record {pin['iterations']}); history deviation GPU-reference "
          f"{float(dev.max()) / h0:.2e} of h0, reference-record / reference-oracle spread "
          f"{float(spread.max()) / h0:.2e}; GPU solution's residual under the reference "
          f"operator {res_ref_op:.3e}; solution difference {d:.2e}")
    assert len(h_r) == pin["iterations"]
    assert info["status"] == "SSG_OK"
    same_stop(info["iterations"], info["history"], h_r)
    k = min(dev.size, spread.size)
    assert np.all(dev[:k] <= np.maximum(2.0 * spread[:k], 1e-9 * h0)), (dev / h0, spread / h0)
    assert res_ref_op <= 1.5 * EPS, res_ref_op


def channel_rhs(ref, n, seed=20241203):
    """The C3 right-hand side: 8 seeded Fourier modes, cos in x and z,
    Neumann-compatible cos(pi k (y + 1) / 2) in y, made mean-zero, weak and
    assembled (the same formula as the bench's C3 section)."""
    X, Y, Z = (ref.geometry(0, 7 + a) for a in range(3))
    x, w, _, _ = ref.basis(0)
    rho = w[None, None, None, :] * w[None, None, :, None] * w[None, :, None, None]
    bj = rho * ref.geometry(0, 6)
    rng = np.random.default_rng(seed)
    g = np.zeros_like(X)
    for _ in range(8):
        kx, kz = rng.integers(1, 4) / 2.0, rng.integers(-3, 4)
        ky = rng.integers(0, 3)
        g += rng.standard_normal() * np.cos(kx * X + kz * Z + rng.uniform(0, 6.28)) * \
            np.cos(math.pi * ky * (Y + 1) / 2)
    g -= (bj * g).sum() / bj.sum()
    return ref.dss(bj * g)


def test_c3_channel_n10_reduced():
    mesh, n = channel_mesh((8, 4, 4)), 10
    ref = O.Reference(mesh, n)
    try:
        f = channel_rhs(ref, n)
        u_r, h_r = ref.solve_poisson(f, np.zeros_like(f))
    finally:
        ref.close()
    out = {}
    for prec in ("fp64", "mixed"):
        ctx = S.Context(0)
        try:
            ctx.set_parameters(1e-3, 1.0 / 1600.0, 1.0)
            ctx.set_setup_options(no_dealias=True, no_particles=True)
            ctx.setup_mesh(mesh, n)
            ctx.set_precision(prec)
            out[prec] = ctx.solve_poisson_cg(f, np.zeros_like(f))
        finally:
            ctx.close()
    u_g, info = out["fp64"]
    assert info["status"] == "SSG_OK"
    dh = check_history(info["history"], h_r)
    d = None
    if same_stop(info["iterations"], info["history"], h_r):
        orc = O.Oracle(mesh, n)
        try:
            d = assert_solution_close(u_g, u_r, orc, orc.solve_poisson, f)
        finally:
            orc.close()
    u_m, info_m = out["mixed"]
    assert info_m["status"] == "SSG_OK" and info_m["residual"] <= EPS
    dm = rel(u_m - u_m.mean(), u_r - u_r.mean())
    assert dm < 1e-8, dm
    print(f"C3 reduced (n = 10): FP64 {info['iterations']} vs {len(h_r)} iterations, "
          f"history {dh:.2e} of h0, solution {d}; mixed {info_m['iterations']} iterations, "
          f"{dm:.2e} from the reference")


def test_c4_particle_trajectories_100_calls_bitwise():
    mesh, n = tgv_box(16), 8
    npart, calls, dt = 20000, 100, 1e-3
    ref = O.Reference(mesh, n)
    ctx = S.Context(0)
    try:
        ctx.set_parameters(dt, 1.0 / 1600.0, 1.0)
        ctx.set_setup_options(no_dealias=True)
        ctx.setup_mesh(mesh, n)
        pts, jac, tinv = ref.particle_geometry()
        ctx.setup_particle_geometry(pts, jac, tinv)
        X, Y, Z = (ref.geometry(0, 7 + a) for a in range(3))
        h = 2 * math.pi / 16
        snaps = np.stack([np.stack([np.sin(X) * np.cos(Y) * np.cos(Z),
                                    -np.cos(X) * np.sin(Y) * np.cos(Z), 0 * X]) * (2.0 / h)
                          for _ in range(3)])
        ctx.set_particle_velocity(snaps)
        rng = np.random.default_rng(7)
        state = np.zeros((npart, 8))
        ints = np.zeros((npart, 3), np.int32)
        state[:, :3] = rng.uniform(-1, 1, (npart, 3))
        state[:, 7] = np.linspace(0.1, 1.0, 10)[np.arange(npart) % 10]
        ints[:, 0] = rng.integers(0, mesh.nel, npart)
        ints[:, 1] = ints[:, 0]
        s_g, i_g = state.copy(), ints.copy()
        s_r, i_r = state.copy(), ints.copy()
        t = 0.0
        for call in range(calls):
            t += 2 * dt
            s_g, i_g, _ = ctx.integrate_particle_equations(s_g, i_g, t, dt)
            ref.set_params(t, dt, 1.0 / 1600.0)
            s_r, i_r = ref.particles_advance(s_r, i_r, snaps)
            assert not np.any(i_g[:, 2] == 5), call          # no reseed drawn
            if call % 10 == 9 or call == calls - 1:
                assert np.array_equal(i_g[:, :2], i_r[:, :2]), call
                assert np.array_equal(s_g.view(np.uint64), s_r.view(np.uint64)), call
    finally:
        ctx.close()
        ref.close()
    moved = int(np.sum(i_g[:, 0] != ints[:, 0]))
    assert moved > npart // 20
    print(f"C4: {npart} particles, {calls} calls, {moved} changed element, bitwise")


# C2's time integration: 50 steps of integrate_navier_stokes at 16^3, N = 7
# on the device, FP64 and mixed precision, against the reference's own 50
# steps recorded by tests/golden/make_golden_c2_steps.py.
C2_STEPS = 50
# FP64: every solve stops where the reference's does, or both stop inside
# the band within 2 eps of the stop (_stop_band_ok).  The fields after 1, 10
# and 50 steps, at the record's 8192 sampled points, relative to the field's
# largest magnitude: the velocity within C2_VEL_REL (measured 1e-11 after 50
# steps); the pressure within C2_P_REL: every pressure solve stops on the
# absolute eps 1e-10 (2.7e-10 of the pressure's largest magnitude 0.375),
# and where the two runs stop at different iterations inside the eps band
# their pressures are one such correction apart (measured 5e-10).
C2_STEPS = 50
C2_VEL_REL = 1e-10
C2_P_REL = 2e-9
# mixed precision: the same stop criterion, FP32 inside the V-cycle; the same
# comparison with the reference's FP64 run, within C2_MIXED_REL (measured:
# velocity 9e-12, pressure 5e-10)
C2_MIXED_REL = 1e-8


def _flow_state(ref):
    """The reference's state: velocity, convection and double-curl histories
    (three levels each, newest first) and pressure."""
    u = [np.stack([ref.get_field(c, l) for c in range(3)]) for l in range(3)]
    conv = [np.stack([ref.get_field(7 + c, l) for c in range(3)]) for l in range(3)]
    rot = [np.stack([ref.get_field(10 + c, l) for c in range(3)]) for l in range(3)]
    p = [ref.get_field(3, l) for l in range(3)]
    return u, conv, rot, p


def _stop_band_ok(hg, hr):
    """Two runs of one solve stop at the same iteration, or both reach the
    band within 2 eps of the stop at the same iteration (or one apart) and
    stop somewhere inside it.  Late in a run the pressure solve starts
    already inside that band (its extrapolated initial guess leaves a
    residual of 1-2 eps); there the V-cycle's inner solves, which stop on
    the same absolute eps, take different inner iteration counts in any two
    FP64 implementations, and the outer residual creeps down by 10-20 % an
    iteration in one run and faster in the other (measured: the reference
    2e-10 -> 9e-11 in 4 iterations where the device took 1), so the stop
    iteration inside the band is not determined by the algorithm."""
    if len(hg) == len(hr):
        return True
    kg = next(i for i, h in enumerate(hg) if h <= 2.0 * EPS)
    kr = next(i for i, h in enumerate(hr) if h <= 2.0 * EPS)
    return abs(kg - kr) <= 1


def test_c2_fifty_steps_fp64_and_mixed():
    rec = np.load(os.path.join(HERE, "golden", "c2_tgv16_n8_steps.npz"))
    mesh, n, dt, visc = tgv_box(16), 8, 1e-3, 1.0 / 1600.0
    ref = O.Reference(mesh, n, dt=dt, visc=visc, dens=1.0)
    try:
        ref.init_tgv()
        state = _flow_state(ref)
        t0 = ref.time()
    finally:
        ref.close()
    idx = rec["sample_index"]
    snaps = [int(s) for s in rec["snap_steps"]]
    umax = np.maximum(rec["snap_maxabs"][:, 0], rec["snap_maxabs"][:, 1])
    pmax = rec["snap_maxabs"][:, 3]
    ctx = S.Context(0)
    report = {}
    try:
        ctx.set_parameters(dt, visc, 1.0)
        ctx.setup_mesh(mesh, n)
        for prec in ("fp64", "mixed"):
            ctx.set_precision(prec)
            ctx.flow_set(*state, None, t0)
            du = dp = 0.0
            stops = dit = 0
            for s in range(C2_STEPS):
                got = ctx.navier_stokes_step(history=True)
                for j, g in enumerate(got):
                    assert g["residual"] <= EPS, (prec, s, j, g["residual"])
                    hr = rec["history"][s, j, :rec["iterations"][s, j]]
                    if prec == "fp64":
                        assert _stop_band_ok(g["history"], hr), (s, j, g["history"], hr)
                        stops += len(g["history"]) != len(hr)
                        dit = max(dit, abs(len(g["history"]) - len(hr)))
                if s + 1 in snaps:
                    k = snaps.index(s + 1)
                    out = ctx.flow_get()
                    assert out["t"] == pytest.approx(rec["time"][k])
                    u, p = out["u"][0], out["p"][0]
                    du = max(du, max(float(np.max(np.abs(u[c].reshape(-1)[idx] -
                                                         rec["snap_u"][k, c]))) / umax[k]
                                     for c in range(3)))
                    dp = max(dp, float(np.max(np.abs(p.reshape(-1)[idx] - rec["snap_p"][k])))
                             / pmax[k])
                    rms = np.array([np.sqrt(np.mean(u[c] * u[c])) for c in range(3)] +
                                   [np.sqrt(np.mean(p * p))])
                    drms = float(np.max(np.abs(rms - rec["snap_rms"][k]) / rec["snap_rms"][k]))
                    report[f"{prec}_rms_{s + 1}"] = drms
            report[prec] = (du, dp, stops, dit)
    finally:
        ctx.close()
    print("C2 50 steps: " + ", ".join(
        f"{p}: velocity {report[p][0]:.2e}, pressure {report[p][1]:.2e} of max "
        f"(solves stopping elsewhere inside the eps band: {report[p][2]}, by up to "
        f"{report[p][3]} iterations)" for p in ("fp64", "mixed")) +
        "; rms " + ", ".join(f"{k} {v:.1e}" for k, v in report.items() if "_rms_" in k))
    du, dp = report["fp64"][:2]
    assert du <= C2_VEL_REL and dp <= C2_P_REL, report["fp64"]
    du, dp = report["mixed"][:2]
    assert du <= C2_MIXED_REL and dp <= C2_MIXED_REL, report["mixed"]
