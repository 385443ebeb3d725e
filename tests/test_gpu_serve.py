"""Serving loop: continuous admission of independent solves of different
meshes, orders and Helmholtz coefficients on one GPU.

Each request runs the same deterministic kernels whatever else is in flight,
so a result in the mix is bitwise the result alone (stated tolerance: 0).
Against the CPU oracle: Helmholtz (FP64 Jacobi CG) 1e-11, Poisson in mixed
precision (FP32 V-cycle inside the FP64 FCG) 1e-8, both relative to the
largest entry, with the absolute stop sqrt((r.r)_w) <= 1e-10.
"""
import numpy as np
import pytest

import oracle as O
import ssenss_b200 as S
from ssenss_b200.mesh import box_mesh, periodic_box_fourier_rhs

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


# (mesh shape, n, lambda): Poisson (lambda 0) and Helmholtz requests
MIX = [((3, 3, 3), 8, 0.0), ((4, 3, 3), 6, 12.5), ((3, 4, 5), 8, 0.0),
       ((3, 3, 3), 10, 60.0), ((5, 3, 3), 6, 0.0), ((3, 3, 4), 12, 0.0),
       ((4, 4, 4), 8, 3.0), ((3, 3, 3), 8, 0.0), ((3, 5, 3), 10, 0.0),
       ((4, 3, 3), 6, 99.0)]

_inputs = {}


def inputs(i):
    """mesh, n, lambda, right-hand side (8 seeded Fourier modes, weak and
    assembled) of request i"""
    if i not in _inputs:
        shape, n, lam = MIX[i]
        _inputs[i] = (box_mesh(shape), n, lam, periodic_box_fourier_rhs(shape, n, 100 + i))
    return _inputs[i]


def oracle_for(i):
    mesh, n, lam, f = inputs(i)
    return O.Oracle(mesh, n, dt=(11.0 / (6.0 * lam)) if lam > 0 else 1.0, visc=1.0)


def test_mix_equals_alone_and_oracle():
    alone = []
    srv = S.Server(0, hbm_budget=40e9, max_active=1)
    try:
        for i in range(len(MIX)):
            mesh, n, lam, f = inputs(i)
            rid = srv.submit(mesh, n, f, lam=lam, precision="mixed")
            u, st, info = srv.wait(rid)
            assert st == "SSG_OK", (i, st)
            alone.append(u)
    finally:
        srv.close()
    srv = S.Server(0, hbm_budget=40e9, max_active=4)
    try:
        ids = [srv.submit(*inputs(i)[:2], inputs(i)[3], lam=inputs(i)[2], precision="mixed")
               for i in range(len(MIX))]
        mixed = [srv.wait(r) for r in ids]
        st = srv.stats()
    finally:
        srv.close()
    assert st["completed"] == len(MIX)
    assert st["max_active_seen"] >= 2          # requests overlapped on the device
    for i, (u, status, info) in enumerate(mixed):
        assert status == "SSG_OK"
        assert np.array_equal(u, alone[i]), i
    # against the oracle
    for i in (0, 1, 3):
        mesh, n, lam, f = inputs(i)
        orc = oracle_for(i)
        if lam > 0:
            u_o, _ = orc.solve_helmholtz(O.X_VELOCITY, f, np.zeros_like(f))
            assert rel(alone[i], u_o) < 1e-11
        else:
            u_o, _ = orc.solve_poisson(f, np.zeros_like(f))
            assert rel(alone[i] - alone[i].mean(), u_o - u_o.mean()) < 1e-8


def test_budget_admission_and_residency():
    mesh, n, lam, f = inputs(2)
    need = S.request_bytes(n, mesh.nel, "mixed")
    srv = S.Server(0, hbm_budget=int(1.5 * need), max_active=4)
    try:
        ids = [srv.submit(mesh, n, f, precision="mixed") for _ in range(4)]
        outs = [srv.wait(r) for r in ids]
        st = srv.stats()
    finally:
        srv.close()
    assert all(o[1] == "SSG_OK" for o in outs)
    for o in outs[1:]:
        assert np.array_equal(o[0], outs[0][0])
    assert st["hbm_peak"] <= st["hbm_budget"]
    assert st["max_active_seen"] == 1          # one context fits the budget
    assert st["mesh_hits"] == 3 and st["mesh_misses"] == 1


def test_reject_cancel_deadline():
    mesh, n, lam, f = inputs(5)               # n = 12, the largest request
    small = inputs(0)
    srv = S.Server(0, hbm_budget=S.request_bytes(n, mesh.nel, "mixed") // 2, max_active=1)
    try:
        rid = srv.submit(mesh, n, f)
        _, st, _ = srv.wait(rid)
        assert st == "SSG_ERR_BUDGET"
    finally:
        srv.close()
    srv = S.Server(0, hbm_budget=40e9, max_active=1)
    try:
        first = srv.submit(mesh, n, f)
        queued = srv.submit(small[0], small[1], small[3])
        late = srv.submit(small[0], small[1], small[3], deadline_ms=1e-3)
        srv.cancel(queued)
        assert srv.wait(first)[1] == "SSG_OK"
        assert srv.wait(queued)[1] == "SSG_ERR_CANCELLED"
        assert srv.wait(late)[1] == "SSG_ERR_TIMEOUT"
        st = srv.stats()
        assert st["cancelled"] == 1 and st["completed"] == 1
    finally:
        srv.close()


def test_request_bytes_covers_the_context():
    for i in (0, 3, 5):
        mesh, n, lam, f = inputs(i)
        ctx = S.Context(0)
        try:
            ctx.set_setup_options(no_dealias=True, no_particles=True)
            ctx.setup_mesh(mesh, n)
            ctx.set_precision("mixed")
            ctx.solve_poisson_cg(f, np.zeros_like(f), history=False)
            used = ctx.memory_bytes()
        finally:
            ctx.close()
        est = S.request_bytes(n, mesh.nel, "mixed")
        assert used <= est, (i, used, est)
        assert used >= 0.7 * est, (i, used, est)


def test_failed_setup_does_not_poison_the_mesh_key():
    """A request whose mesh fails set-up (here a neighbour id out of range)
    leaves no context behind: the next request with the same mesh key sets
    the mesh up afresh and succeeds."""
    mesh, n, lam, f = inputs(0)
    bad = box_mesh((3, 3, 3))
    bad.neigh = np.array(bad.neigh, copy=True)
    bad.neigh[0, 0] = bad.nel + 5
    srv = S.Server(0, hbm_budget=40e9, max_active=2)
    try:
        key = 0x5EED
        _, st, _ = srv.wait(srv.submit(bad, n, f, key=key))
        assert st == "SSG_ERR_MESH"
        u, st, _ = srv.wait(srv.submit(mesh, n, f, key=key))
        assert st == "SSG_OK"
        stats = srv.stats()
        assert stats["resident_contexts"] == 1
    finally:
        srv.close()
    orc = oracle_for(0)
    u_o, _ = orc.solve_poisson(f, np.zeros_like(f))
    assert rel(u - u.mean(), u_o - u_o.mean()) < 1e-8


@pytest.mark.parametrize("shape,n,lam", [((2, 2, 2), 6, 0.0), ((2, 2, 3), 8, 40.0),
                                          ((2, 3, 3), 5, 0.0), ((1, 3, 3), 6, 7.5)])
def test_small_boxes_against_assembled_oracle(shape, n, lam):
    """Boxes with one or two elements along a periodic direction ("reference-
    incorrect": the reference's first-match pairing joins a face to the
    neighbour's face on the same side, so no reference run can check them).
    The serving loop pairs opposite faces; its solution is checked against
    the assembled-operator oracle with correct global numbering
    (oracle/periodic_box.py) at 1e-8 relative to the largest entry (mixed
    precision Poisson and FP64 Helmholtz, both stopped at sqrt((r.r)_w) <=
    1e-10; Poisson solutions compared with their means removed)."""
    from oracle import periodic_box as PB
    mesh = box_mesh(shape)
    f = periodic_box_fourier_rhs(shape, n, 31)
    srv = S.Server(0, hbm_budget=40e9, max_active=2)
    try:
        u, st, info = srv.wait(srv.submit(mesh, n, f, lam=lam, precision="mixed"))
    finally:
        srv.close()
    assert st == "SSG_OK", st
    u_b = PB.solve(shape, n, f, lam)
    if lam == 0:
        u, u_b = u - u.mean(), u_b - u_b.mean()
    assert rel(u, u_b) < 1e-8, (rel(u, u_b), info)


# segments of one shared-launch Helmholtz solve: (shape, lambda, eps) at n = 6
SEGMENTS = [((3, 3, 3), 3.0, 1e-10), ((4, 3, 3), 40.0, 1e-10), ((3, 4, 3), 0.7, 1e-9),
            ((3, 3, 5), 12.5, 1e-10), ((5, 3, 3), 99.0, 1e-10)]


def test_segmented_helmholtz_matches_solo():
    """ssg_solve_helmholtz_segments: five independent boxes (different
    shapes, lambdas and stops) concatenated in one context share every
    operator and DSS launch; each segment against its own solo
    ssg_solve_helmholtz_cg: the same iteration count (one apart only with
    both final residuals within a factor 2 of the segment's eps), solution
    within 1e-11 relative.  The segment's sums are grouped differently from
    the solo solve's, so rounding, not bitwise."""
    from ssenss_b200.mesh import concat_meshes
    n = 6
    meshes, fs, solo = [], [], []
    for k, (shape, lam, eps) in enumerate(SEGMENTS):
        mesh = box_mesh(shape)
        f = periodic_box_fourier_rhs(shape, n, 300 + k)
        ctx = S.Context(0)
        try:
            ctx.set_parameters(11.0 / (6.0 * lam), 1.0, 1.0)
            ctx.set_setup_options(no_dealias=True, no_particles=True, opposite_pairing=True)
            ctx.setup_mesh(mesh, n)
            u, info = ctx.solve_helmholtz_cg(S.X_VELOCITY, f, np.zeros_like(f), eps=eps,
                                             history=False)
        finally:
            ctx.close()
        meshes.append(mesh)
        fs.append(f)
        solo.append((u.copy(), info))
    big, first = concat_meshes(meshes)
    ctx = S.Context(0)
    try:
        ctx.set_setup_options(no_dealias=True, no_particles=True, opposite_pairing=True)
        ctx.setup_mesh(big, n)
        f = np.concatenate(fs)
        u, infos = ctx.solve_helmholtz_segments(S.X_VELOCITY, first, [s[1] for s in SEGMENTS],
                                                f, np.zeros_like(f), [s[2] for s in SEGMENTS])
        for k, (shape, lam, eps) in enumerate(SEGMENTS):
            us, inf = solo[k]
            ub = u[first[k]:first[k + 1]]
            ib = infos[k]
            print(f"segment {k} {shape} lambda {lam}: iterations {ib['iterations']} "
                  f"(solo {inf['iterations']}), residual {ib['residual']:.3e} "
                  f"(solo {inf['residual']:.3e}), solution {rel(ub, us):.2e}")
            assert ib["status"] == "SSG_OK" and ib["residual"] <= eps
            if ib["iterations"] != inf["iterations"]:
                assert abs(ib["iterations"] - inf["iterations"]) == 1
                assert max(ib["residual"], inf["residual"]) <= 2 * eps
            assert rel(ub, us) < 1e-11
            assert ib["initial_residual"] == pytest.approx(inf["initial_residual"], rel=1e-12)
        # a segment table that splits a mesh (an element neighbouring
        # another segment) is refused
        bad = np.array([0, 10, big.nel], dtype=np.int32)
        with pytest.raises(S.SsgError):
            ctx.solve_helmholtz_segments(S.X_VELOCITY, bad, [1.0, 2.0], f, np.zeros_like(f),
                                         [1e-10, 1e-10])
    finally:
        ctx.close()


def test_shared_launch_batches_match_solo():
    """ssg_server_set_batching: a burst of small Helmholtz requests of one
    order (different boxes and lambdas) behind a one-slot server runs in
    shared-launch batches; every request against the same request solved
    alone by a server without batching: status OK, solution within 1e-11
    relative (the batch groups each segment's sums differently)."""
    n = 6
    shapes = [(3, 3, 3), (4, 3, 3), (3, 4, 3), (3, 3, 4)]
    reqs = [(shapes[k % 4], 0.5 + 9.5 * k) for k in range(10)]
    fs = [periodic_box_fourier_rhs(sh, n, 500 + k) for k, (sh, _) in enumerate(reqs)]

    def run(batching):
        srv = S.Server(0, hbm_budget=20e9, max_active=1)
        try:
            if batching:
                srv.set_batching(8, 1 << 20)
            ids = [srv.submit(box_mesh(sh), n, fs[k], lam=lam, eps=1e-10, precision="fp64")
                   for k, (sh, lam) in enumerate(reqs)]
            out = [srv.wait(r) for r in ids]
            return out, srv.stats()
        finally:
            srv.close()

    solo, st0 = run(False)
    batched, st1 = run(True)
    assert st0["batches"] == 0
    print(f"shared launches: {st1['batches']} batches holding {st1['batched_requests']} of "
          f"{len(reqs)} requests")
    assert st1["batches"] >= 1 and st1["batched_requests"] >= 2
    assert st1["completed"] == len(reqs)
    for k in range(len(reqs)):
        (ua, sa, ia), (ub, sb, ib) = solo[k], batched[k]
        assert sa == "SSG_OK" and sb == "SSG_OK", (k, sa, sb)
        assert ib["residual"] <= 1e-10
        assert rel(ub, ua) < 1e-11, k
