"""The time step's Stokes operators and the resident step on the library's
own set-up (ssg_setup_mesh), against the reference compiled in place
(oracle/_ref) on the same mesh.

The library computes its geometric factors itself; they agree with the
reference's to 1e-14, so the per-element operators (no DSS) agree to
STOKES_REL of their largest entry on random fields: the double curl chains
two derivatives of a random field through the inverse Jacobian, the
right-hand sides one derivative plus the surface terms, each within a few
hundred roundings of the largest entry.

The resident step (ssg_flow_set, ssg_navier_stokes_step, ssg_flow_get) runs
STEPS steps of C1's Taylor-Green vortex from the reference's own initial
state (velocity, pressure, convection and double-curl histories) and is
compared with the reference's integrate_navier_stokes: every solve stops
within the band the drop-in tests state, and the velocity, pressure and
histories agree to STEP_REL (each solve stops on the absolute eps 1e-10, so
the two runs are one correction of that size apart).
"""
import numpy as np
import pytest

import oracle as O
from ssenss_b200.mesh import box_mesh, channel_mesh, tgv_box

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not O.reference_available(),
                                 reason="reference library not built")]

DT, VISC = 1e-3, 1.0 / 1600.0
STOKES_REL = 1e-12
STEPS = 3
STEP_REL = 1e-9
EPS = 1e-10

CASES = {
    # periodic: no wall faces (the velocity surface terms on every face)
    "tgv3_n8": (lambda: tgv_box(3), 8),
    # walls on every side (the pressure surface terms on every face)
    "box333_n6": (lambda: box_mesh((3, 3, 3), lo=(-1.0,) * 3, hi=(1.0,) * 3,
                                   periodic=(False,) * 3), 6),
    # deformed channel: walls on two sides, curved faces
    "channel433_n7": (lambda: channel_mesh((4, 3, 3), seed=7), 7),
}


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.mark.parametrize("name", list(CASES))
def test_stokes_operators_match_reference(name, gpu_ctx_factory):
    mk, n = CASES[name]
    mesh = mk()
    ctx = gpu_ctx_factory(mesh, n, dt=DT, visc=VISC)
    ref = O.Reference(mesh, n, dt=DT, visc=VISC, dens=1.0)
    try:
        rng = np.random.default_rng(5)
        sh = (mesh.nel, n, n, n)
        u = rng.standard_normal((3,) + sh)
        g3 = rng.standard_normal((3,) + sh)
        p = rng.standard_normal(sh)
        errs = []
        for which, g in ((0, None), (1, g3), (2, p)):
            got = ctx.stokes_operator(which, u, g)
            want = ref.stokes_operator(which, u, g)
            errs.append(rel(got, want))
        print(f"{name}: double curl {errs[0]:.2e}, pressure rhs {errs[1]:.2e}, "
              f"velocity rhs {errs[2]:.2e}")
        assert max(errs) <= STOKES_REL, errs
    finally:
        ref.close()


def _state(ref):
    u = [np.stack([ref.get_field(c, l) for c in range(3)]) for l in range(3)]
    conv = [np.stack([ref.get_field(7 + c, l) for c in range(3)]) for l in range(3)]
    rot = [np.stack([ref.get_field(10 + c, l) for c in range(3)]) for l in range(3)]
    p = [ref.get_field(3, l) for l in range(3)]
    return u, conv, rot, p


def test_resident_steps_match_reference(gpu_ctx_factory):
    mesh, n = tgv_box(4), 8
    ctx = gpu_ctx_factory(mesh, n, dt=DT, visc=VISC)
    ref = O.Reference(mesh, n, dt=DT, visc=VISC, dens=1.0)
    try:
        ref.init_tgv()
        u, conv, rot, p = _state(ref)
        ctx.flow_set(u, conv, rot, p, None, ref.time())
        for s in range(STEPS):
            ref.ns_step()
            want = ref.step_log()
            got = ctx.navier_stokes_step()
            assert [k for k, _, _ in want] == [0, 1, 1, 1]
            for (kind, var, hc), g in zip(want, got):
                hg = g["history"]
                if len(hc) != len(hg):
                    k = min(len(hc), len(hg)) - 1
                    for h in (hc, hg):
                        band = h[k:max(k + 1, len(h) - 1)]
                        assert all(0.5 * EPS <= v <= 2 * EPS for v in band), (s, var, hc, hg)
        out = ctx.flow_get()
        u, conv, rot, p = _state(ref)
        assert out["t"] == pytest.approx(ref.time())
        devs = {
            "u": max(rel(out["u"][l], u[l]) for l in range(3)),
            "p": max(rel(out["p"][l], p[l]) for l in range(3)),
            "conv": max(rel(out["conv"][l], conv[l]) for l in range(3)),
            "rot": max(rel(out["rot"][l], rot[l]) for l in range(3)),
        }
        print(f"resident steps: {STEPS} steps of C1, deviations " +
              ", ".join(f"{k} {v:.2e}" for k, v in devs.items()))
        assert max(devs.values()) <= STEP_REL, devs
    finally:
        ref.close()
