#!/usr/bin/env python
"""Benchmark of the SSENSS per-timestep solve path on B200.

Workload (one "step"): the pressure Poisson solve of the Taylor-Green vortex
on the triply periodic [0, 2 pi]^3 box of 16 x 16 x 16 hexahedra at N = 7
(n = 8 GLL points per direction, 2,097,152 local points): flexible CG with
the p-multigrid preconditioner (solve_poisson_cg, src/solver.c:159-173) to
the reference's absolute criterion sqrt((r.r)_w) <= 1e-10, from a zero
initial guess, right-hand side the weak form of -lap p for the TGV pressure
p = (cos 2x + cos 2y)(cos 2z + 2)/16, assembled by DSS.  Synthetic data: the
mesh and fields are generated, not read.

Metric: GDOF/s per PCG iteration = unique DOFs x outer iterations / time,
plus solves/s; FP64 (the plain form, `value`) and the mixed-precision form
(FP32 storage in the V-cycle) side by side.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

N > 1 runs independent replicas, one per GPU (the solve does not shard at
this tier); value = DOF-iterations of all ranks / max-over-ranks time.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
os.environ.setdefault("OPENBLAS_NUM_THREADS", "1")

METRIC = ("GDOF/s per PCG iter & solves/s: mixed vs FP64 GPU at 1e-10 resid; "
          "p99 latency")
UNIT = "GDOF/s"
NE, NORD = 16, 8          # 16^3 elements, n = N + 1 = 8
EPS = 1e-10
# dominant kernel: the level-0 element operator (Laplacian), bytes per local
# point: read u (8) + six G*rho*J factors (48) + write (8)
OP_BYTES_PER_POINT = 64
# DRAM bytes per launch of that kernel (dram__bytes_read.sum +
# dram__bytes_write.sum) from the ncu capture of the same workload
# summarised in profiles/k_ax8_dmma_tgv16_n8.md
OP_TRAFFIC_BYTES = 117918464 + 7999744


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--ne", type=int, default=NE)
    ap.add_argument("--n", type=int, default=NORD)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extra", action="store_true",
                    help="skip the channel (C3), particle (C4) and convection sections")
    ap.add_argument("--no-tune", action="store_true",
                    help="keep the default launch shapes (skip ssg_autotune)")
    ap.add_argument("--no-graphs", action="store_true",
                    help="launch the V-cycle kernels directly (no CUDA graph)")
    ap.add_argument("--serve-requests", type=int, default=300,
                    help="requests of the serving stream (the full stream is 2000)")
    ap.add_argument("--serve-rate", type=float, default=15.0,
                    help="Poisson arrival rate of the serving stream (requests/s; "
                         "15/s is the rate the service target is stated at)")
    ap.add_argument("--serve-slots", type=int, default=8,
                    help="requests in flight at once in the serving loop")
    ap.add_argument("--serve-open-only", action="store_true",
                    help="serving: only the open-loop runs (served and plain), no "
                         "closed-loop throughput runs")
    ap.add_argument("--no-time", action="store_true",
                    help="conv section: the launches only, no timing loop")
    ap.add_argument("--sections", default="all",
                    choices=["all", "fp64", "mixed", "op", "conv", "serve", "extra", "channel",
                             "particles", "step"],
                    help="fp64: only the FP64 solves; op / conv: only the operator / "
                         "convection launches (for profiler captures)")
    return ap.parse_args()


def tgv_rhs_strong(X, Y, Z):
    """-lap p for p = (cos 2x + cos 2y)(cos 2z + 2)/16."""
    import numpy as np
    c2x, c2y, c2z = np.cos(2 * X), np.cos(2 * Y), np.cos(2 * Z)
    lap = (-4.0 * (c2x + c2y) * (c2z + 2.0) - 4.0 * (c2x + c2y) * c2z) / 16.0
    return -lap


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class Clocks:
    """nvidia-smi clock / throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.fh, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.fh.close()
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                 "sw_power_cap"]
        for line in open(self.path):
            p = [x.strip() for x in line.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = max(mx, float(p[2]))
            except ValueError:
                continue
            for nm, v in zip(names, p[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl" if args.impl == "ours" else "gloo",
                                timeout=datetime.timedelta(seconds=600))
        pg = dist
    return world, rank, local, pg


def max_over_ranks(pg, v, device=None):
    if pg is None:
        return v
    import torch
    t = torch.tensor([v], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(pg, v, device=None):
    if pg is None:
        return v
    import torch
    t = torch.tensor([v], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=pg.ReduceOp.SUM)
    return float(t.item())


# ---------------------------------------------------------------------------
# CPU reference (the reference sources compiled in place, oracle/_ref)
# ---------------------------------------------------------------------------
def reference_sample(mesh, n, f, max_iter):
    """Time the reference's FCG + p-MG (flexible_conjugate_gradient,
    src/solver.c:83-157) on this workload, 1 core, for at most max_iter outer
    iterations; returns (seconds, iterations run)."""
    import numpy as np
    import oracle
    ref = oracle.Reference(mesh, n)
    f = np.ascontiguousarray(f)
    u = np.zeros_like(f)
    t0 = time.perf_counter()
    ref.lib().ssgref_fcg_mg(oracle._d(f), oracle._d(u), EPS, max_iter)
    dt = time.perf_counter() - t0
    # iterations actually run: rerun is too costly; the cap is reached unless
    # the residual fell below eps first, which the oracle's count tells
    ref.close()
    return dt, max_iter


def reference_step_sample(steps=2):
    """The reference's integrate_navier_stokes (src/navier_stokes.c:224-235)
    on C1 (TGV 4^3, n = 8, dt 1e-3, Re 1600) from its initial state, 1 core:
    seconds per step over `steps` steps after one untimed step."""
    import oracle
    from ssenss_b200.mesh import tgv_box
    ref = oracle.Reference(tgv_box(4), 8, dt=1e-3, visc=1.0 / 1600.0, dens=1.0)
    ref.init_tgv()
    ref.ns_step()
    t0 = time.perf_counter()
    for _ in range(steps):
        ref.ns_step()
    dt = (time.perf_counter() - t0) / steps
    ref.close()
    return dt


# resident memory of one reference process at the 16^3, n = 8 workload
# (measured: 4.1 GB peak), used to bound how many run at once
REF_PROC_BYTES = 4.6e9


# at most this many reference processes at once: each sets up its own 4 GB
# copy of the workload (page-fault heavy), which bounds the arm's wall time
REF_PROC_MAX = 64


def reference_processes():
    """Independent reference processes the host can run at once: one per
    core, bounded by 60 % of the available memory and by REF_PROC_MAX."""
    try:
        import psutil
        avail = psutil.virtual_memory().available
    except Exception:
        avail = 16e9
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    return max(1, min(int(cores or 1), int(0.6 * avail / REF_PROC_BYTES), REF_PROC_MAX))


def _reference_worker(ne, n, iters, warmup, steps, barrier, out):
    """One reference process (1 thread): set up the TGV pressure solve, wait
    for the others, then time warmup + steps solves of `iters` FCG + p-MG
    iterations each from a zero guess."""
    os.environ["OPENBLAS_NUM_THREADS"] = "1"
    sys.path.insert(0, ROOT)
    import numpy as np
    import oracle
    from ssenss_b200.mesh import tgv_box
    mesh = tgv_box(ne)
    ref = oracle.Reference(mesh, n)
    x, w, _, _ = ref.basis(0)
    X, Y, Z = (ref.geometry(0, 7 + a) for a in range(3))
    rho = w[None, None, None, :] * w[None, None, :, None] * w[None, :, None, None]
    f = ref.dss(rho * ref.geometry(0, 6) * tgv_rhs_strong(X, Y, Z))
    barrier.wait()
    times = []
    for s in range(warmup + steps):
        u = np.zeros_like(f)
        t0 = time.perf_counter()
        ref.lib().ssgref_fcg_mg(oracle._d(f), oracle._d(u), EPS, iters)
        dt = time.perf_counter() - t0
        if s >= warmup:
            times.append(dt)
    ref.close()
    out.put(times)


def run_reference(args):
    world, rank, local, pg = dist_setup(args)
    if rank != 0:
        if pg is not None:
            pg.destroy_process_group()
        return 0
    import multiprocessing as mp
    import oracle
    from ssenss_b200.mesh import tgv_box
    if not oracle.reference_available():
        print(json.dumps({"impl": "reference",
                          "unavailable": "oracle/_ref/libssenss_ref.so not built "
                                         "(the reference sources were absent at build)"}))
        return 0
    n = args.n
    udofs = tgv_box(args.ne).unique_nodes(n)
    iters_per_step = 1
    procs = reference_processes()
    ctx = mp.get_context("spawn")
    barrier = ctx.Barrier(procs)
    q = ctx.Queue()
    ps = [ctx.Process(target=_reference_worker,
                      args=(args.ne, n, iters_per_step, args.warmup, args.steps, barrier, q))
          for _ in range(procs)]
    for p in ps:
        p.start()
    res = [q.get() for _ in ps]
    for p in ps:
        p.join()
    # the processes ran side by side: whole-host throughput is the sum of
    # their rates; a step lasts as long as the slowest process's
    value = sum(udofs * iters_per_step * len(t) / sum(t) for t in res) / 1e9
    ms_step = max(1e3 * sum(t) / len(t) for t in res)
    sample = (f"{procs} independent reference processes x 1 thread side by side (one per "
              f"host core, bounded by memory and by {REF_PROC_MAX}), each timing {iters_per_step} FCG+p-MG "
              f"iteration of the {args.ne}^3 N={n-1} TGV pressure solve from zero per step "
              f"(the first outer iteration, the costliest of the 11 of a full solve); "
              f"reference sources compiled in place, OPENBLAS_NUM_THREADS=1")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_step, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": (f"TGV {args.ne}^3 hex N={n-1} (n={n}) pressure Poisson, "
                                f"FCG+p-MG to sqrt((r.r)_w)<=1e-10 from zero"),
                   "elements": args.ne ** 3, "n": n, "unique_dofs": udofs,
                   "parallelism": f"{procs} host processes (rank 0 host)"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": procs, "kind": "reference",
                         "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------------------
# serving stream (periodic boxes of E elements, orders N in {5,7,9,11})
# ---------------------------------------------------------------------------
def near_cube_shapes(lo=2, hi=16):
    """Element counts a*b*c with lo <= a <= b <= c <= a + 1 (near-cubes)."""
    out = {}
    for a in range(lo, hi + 1):
        for b in (a, a + 1):
            for c in (b, b + 1):
                if c <= a + 1:
                    out.setdefault(a * b * c, (a, b, c))
    return sorted(out.items())


def serve_stream(nreq, rate, seed=2024):
    """Requests (arrival s, shape, n, lambda, rhs seed): E log-uniform in
    [8, 4096], rounded (in log E) to the nearest product a b c of three
    integers with a <= b <= c <= a + 1 -- 8, 12, 18, 27, 36, ... -- so that
    the boxes keep their elements near cubic; counts below 27 have two
    elements along a periodic direction and are solved with the opposite
    face pairing (the reference's first match pairs them wrongly), n uniform
    in {6, 8, 10, 12}, Poisson (lambda = 0) or Helmholtz with lambda uniform
    in (0, 100] with probability 1/2 each, Poisson arrivals."""
    import numpy as np
    rng = np.random.default_rng(seed)
    shapes = near_cube_shapes()
    counts = np.array([e for e, _ in shapes], dtype=float)
    t = 0.0
    out = []
    for i in range(nreq):
        t += rng.exponential(1.0 / rate)
        e = math.exp(rng.uniform(math.log(8.0), math.log(4096.0)))
        shape = shapes[int(np.argmin(np.abs(np.log(counts) - math.log(e))))][1]
        n = int(rng.choice([6, 8, 10, 12]))
        lam = 0.0 if rng.uniform() < 0.5 else float(rng.uniform(1e-9, 100.0))
        out.append((t, shape, n, lam, int(rng.integers(1 << 31))))
    return out


def run_serving(args, device):
    """Open-loop serving stream through ssg_server (mixed precision, up to
    --serve-slots in flight, 150 GB budget) beside the plain FP64
    one-at-a-time path on the same stream; closed-loop throughput of both."""
    import numpy as np
    import ssenss_b200 as S
    from ssenss_b200.mesh import box_mesh, periodic_box_fourier_rhs
    stream = serve_stream(args.serve_requests, args.serve_rate)
    meshes, keys, rhs = {}, {}, []
    for (_, shape, n, lam, sd) in stream:
        if shape not in meshes:
            meshes[shape] = box_mesh(shape)
        if (shape, n) not in keys:
            keys[(shape, n)] = S.mesh_key(meshes[shape], n)
        rhs.append(periodic_box_fourier_rhs(shape, n, sd))

    def run(slots, precision, open_loop):
        srv = S.Server(device, hbm_budget=150e9, max_active=slots)
        ids = []
        t0 = time.perf_counter()
        for i, (ta, shape, n, lam, _) in enumerate(stream):
            if open_loop:
                dt = ta - (time.perf_counter() - t0)
                if dt > 0:
                    time.sleep(dt)
            ids.append(srv.submit(meshes[shape], n, rhs[i], lam=lam, eps=EPS,
                                  precision=precision, key=keys[(shape, n)]))
        outs = [srv.wait(r) for r in ids]
        wall = time.perf_counter() - t0
        st = srv.stats()
        srv.close()
        bad = [o[1] for o in outs if o[1] != "SSG_OK"]
        return outs, st, wall, bad

    # warm-up: module loading and first-use attributes outside the runs
    wsrv = S.Server(device, hbm_budget=150e9, max_active=args.serve_slots)
    wid = [wsrv.submit(meshes[shape], n, rhs[i], lam=lam, eps=EPS, precision=p,
                       key=keys[(shape, n)])
           for i, (_, shape, n, lam, _) in enumerate(stream[:16]) for p in ("mixed", "fp64")]
    for r in wid:
        wsrv.wait(r)
    wsrv.close()
    served, st_s, wall_s, bad_s = run(args.serve_slots, "mixed", True)
    plain, st_p, wall_p, bad_p = run(1, "fp64", True)
    closed = None
    if not args.serve_open_only:
        _, st_sc, wall_sc, _ = run(args.serve_slots, "mixed", False)
        _, st_pc, wall_pc, _ = run(1, "fp64", False)
        closed = {"served_mixed": st_sc["completed"] / wall_sc,
                  "plain_fp64_one_at_a_time": st_pc["completed"] / wall_pc}
    diff = 0.0
    for (u_s, st1, _), (u_p, st2, _), (_, _, _, lam, _) in zip(served, plain, stream):
        if u_s is None or u_p is None or st1 != "SSG_OK" or st2 != "SSG_OK":
            continue
        a, b = (u_s - u_s.mean(), u_p - u_p.mean()) if lam == 0 else (u_s, u_p)
        diff = max(diff, float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)))
    npois = sum(1 for r in stream if r[3] == 0.0)

    def pick(st, wall):
        return {"p50_ms": st["p50_ms"], "p99_ms": st["p99_ms"], "mean_ms": st["mean_ms"],
                "max_ms": st["max_ms"], "queue_p99_ms": st["queue_p99_ms"],
                "solves_per_s": st["completed"] / wall, "completed": st["completed"],
                "hbm_peak_gb": st["hbm_peak"] / 1e9, "mesh_hits": st["mesh_hits"],
                "mesh_misses": st["mesh_misses"], "evictions": st["evictions"],
                "max_in_flight": st["max_active_seen"]}

    burst = None if args.serve_open_only else run_burst(device)
    return {
        "shared_launch_burst": burst,
        "workload": (f"{len(stream)} requests ({npois} Poisson FCG+p-MG, "
                     f"{len(stream) - npois} Helmholtz CG-Jacobi), periodic boxes E "
                     f"log-uniform in [8, 4096] rounded to near-cubes a*b*c from 2*2*2 "
                     f"(E < 27 included), n in {{6,8,10,12}}, Poisson arrivals "
                     f"{args.serve_rate}/s, stop sqrt((r.r)_w) <= {EPS}, HBM budget 150 GB"),
        "served_mixed": pick(st_s, wall_s),
        "plain_fp64_one_at_a_time": pick(st_p, wall_p),
        "closed_loop_solves_per_s": closed,
        "failed": len(bad_s) + len(bad_p),
        "failed_statuses": sorted(set(bad_s + bad_p)),
        "max_rel_diff_mixed_vs_fp64": diff,
        "slots": args.serve_slots,
    }


def run_burst(device, nreq=64, n=8):
    """A burst of small Helmholtz requests of one order (periodic boxes of 8 to
    64 elements, n = 8, lambda in (0, 100]) submitted at once: one slot
    without batching, eight slots without batching (overlap on streams), and
    one slot with shared-launch batches of up to 16 requests
    (ssg_server_set_batching).  The burst runs once to warm the resident
    contexts, then three timed passes; the median pass is reported."""
    import numpy as np
    import ssenss_b200 as S
    from ssenss_b200.mesh import box_mesh, periodic_box_fourier_rhs
    rng = np.random.default_rng(17)
    shapes = [(2, 2, 2), (2, 2, 3), (3, 3, 3), (2, 4, 4), (4, 4, 4), (3, 3, 2)]
    reqs = []
    for k in range(nreq):
        sh = shapes[int(rng.integers(len(shapes)))]
        reqs.append((sh, float(rng.uniform(0.5, 100.0)), periodic_box_fourier_rhs(sh, n, 900 + k)))
    meshes = {sh: box_mesh(sh) for sh in shapes}

    def once(slots, batch):
        srv = S.Server(device, hbm_budget=40e9, max_active=slots)
        if batch:
            srv.set_batching(16, 1 << 16)
        out, walls = None, []
        for rep in range(4):
            t0 = time.perf_counter()
            ids = [srv.submit(meshes[sh], n, f, lam=lam, eps=EPS, precision="fp64")
                   for sh, lam, f in reqs]
            out = [srv.wait(r) for r in ids]
            if rep > 0:
                walls.append(time.perf_counter() - t0)
        st = srv.stats()
        srv.close()
        wall = statistics.median(walls)
        return out, {"solves_per_s": nreq / wall, "wall_ms": 1e3 * wall,
                     "wall_ms_passes": [1e3 * w for w in walls],
                     "p50_ms": st["p50_ms"], "p99_ms": st["p99_ms"],
                     "batches": st["batches"], "batched_requests": st["batched_requests"],
                     "failed": sum(1 for o in out if o[1] != "SSG_OK")}

    ref, one = once(1, False)
    _, eight = once(8, False)
    bat, batched = once(1, True)
    diff = max(float(np.abs(a[0] - b[0]).max() / max(np.abs(a[0]).max(), 1e-300))
               for a, b in zip(bat, ref))
    return {"workload": f"{nreq} Helmholtz requests at once, n = {n}, periodic boxes of 8 to "
                        f"64 elements, lambda in (0, 100], stop {EPS} absolute, FP64",
            "one_slot": one, "eight_slots": eight, "one_slot_shared_launches": batched,
            "max_rel_diff_batched_vs_one_slot": diff}


# ---------------------------------------------------------------------------
# other configurations: channel Poisson (C3), particles (C4), convection
# ---------------------------------------------------------------------------
def cuda_timed(lib_stream, fn, k, w=1):
    """Device time (ms) of k calls of fn on the library's stream."""
    import torch
    for _ in range(w):
        fn()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(lib_stream)
    out = [fn() for _ in range(k)]
    e1.record(lib_stream)
    e1.synchronize()
    return e0.elapsed_time(e1), out


def run_channel(args, device):
    """C3: deformed channel 32 x 16 x 16, N = 9 (n = 10, 8.2M local points),
    Poisson solve of 8 seeded Fourier modes (Neumann-compatible in y, mean
    zero), FP64 vs mixed, autotuned shapes, graph-captured V-cycle."""
    import numpy as np
    import torch
    import ssenss_b200 as S
    from ssenss_b200.mesh import channel_mesh
    mesh = channel_mesh((32, 16, 16))
    n = 10
    ctx = S.Context(device)
    ctx.set_setup_options(no_dealias=True, no_particles=True)
    t0 = time.perf_counter()
    ctx.setup_mesh(mesh, n)
    setup_s = time.perf_counter() - t0
    tuned = ctx.autotune()
    X, Y, Z = (ctx.level_data(0, 12 + a) for a in range(3))
    rng = np.random.default_rng(20241203)
    g = np.zeros_like(X)
    for _ in range(8):
        kx, kz = rng.integers(1, 4) / 2.0, rng.integers(-3, 4)
        ky = rng.integers(0, 3)
        g += rng.standard_normal() * np.cos(kx * X + kz * Z + rng.uniform(0, 6.28)) * \
            np.cos(math.pi * ky * (Y + 1) / 2)
    bj = ctx.level_data(0, 6)
    g -= (bj * g).sum() / bj.sum()
    f = torch.from_numpy(ctx.direct_stiffness_summation(np.ascontiguousarray(bj * g))).cuda(device)
    u = torch.zeros_like(f)
    lib_stream = torch.cuda.ExternalStream(ctx.stream, device=torch.device("cuda", device))
    udofs = mesh.unique_nodes(n)
    out = {"workload": "channel 32x16x16 tanh(2.0) y-stretch, perturb 0.1, N=9 (n=10), "
                       "8 Fourier modes, Poisson FCG+p-MG to 1e-10 abs",
           "local_points": mesh.nel * n ** 3, "unique_dofs": udofs,
           "host_setup_s": setup_s,
           "launch_shapes": {str(k): v for k, v in tuned.items()}}
    # the level-0 operator at n = 10 (the solve's dominant kernel at this
    # order): 64 B per local point (u, six metric terms, out), timed alone
    # on the library's stream (ssg_time_operator, 50 launches, best of 3)
    peak, peak_kind = peaks()
    op_us = ctx.time_operator(S.PRESSURE, 50)
    op_alg = 64 * mesh.nel * n ** 3
    out["operator_n10"] = {"us_per_launch": op_us, "bytes_per_launch": op_alg,
                           "achieved_gbs": op_alg / (op_us * 1e-6) / 1e9,
                           "frac": op_alg / (op_us * 1e-6) / 1e9 / peak,
                           "peak_gbs": peak, "peak_source": peak_kind,
                           "operator_shape": S.tuning(n)["ax_elements_per_block"]}
    sols = {}
    for prec in ("fp64", "mixed"):
        ctx.set_precision(prec)

        def solve():
            with torch.cuda.stream(lib_stream):
                u.zero_()
            return ctx.solve_poisson_cg(f, u, eps=EPS, history=False)[1]

        ms, infos = cuda_timed(lib_stream, solve, 3, 2)
        it = sum(i["iterations"] for i in infos) / 3
        sols[prec] = u.cpu().numpy().copy()
        out[prec] = {"ms_per_solve": ms / 3, "iterations": it,
                     "gdof_per_s": udofs * it / (ms / 3 * 1e-3) / 1e9,
                     "solves_per_s": 3 / (ms * 1e-3),
                     "residual": infos[-1]["residual"]}
    d64 = sols["fp64"] - sols["fp64"].mean()
    d32 = sols["mixed"] - sols["mixed"].mean()
    out["mixed"]["max_rel_diff_vs_fp64"] = float(np.abs(d32 - d64).max() / np.abs(d64).max())
    out["mixed"]["speedup_solves_vs_fp64"] = out["mixed"]["solves_per_s"] / \
        out["fp64"]["solves_per_s"]
    ctx.close()
    return out


def run_particles(args, ctx, mesh, n, device, nsteps=100, npart=1_000_000):
    """C4: 1M particles in the 16^3 N=7 TGV flow: nsteps calls of
    integrate_particle_equations, each advancing 2 dt (the reference's
    cadence, flow dt = 1e-3), on frozen velocity snapshots (the reference
    computes ur once, src/main.c:84) of the TGV field in reference
    components; particles start at rest, tau in {0.1, ..., 1.0}.  The walk
    runs on the library's own GLL points and level-0 factors (built by
    ssg_setup_mesh); element ids and states are checked bit for bit against
    the reference in tests/test_gpu_configs.py.  Algorithmic bytes: the
    particle state read and written once per call, 2 x (8 x 8 + 3 x 4) B."""
    import numpy as np
    import torch
    X, Y, Z = (ctx.level_data(0, 12 + a) for a in range(3))
    dt = 1e-3
    h = 2 * math.pi / args.ne          # element width: ur = u / (h / 2)
    snaps = np.stack([np.stack([np.sin(X) * np.cos(Y) * np.cos(Z),
                                -np.cos(X) * np.sin(Y) * np.cos(Z), 0 * X]) * (2.0 / h)
                      for _ in range(3)])
    ctx.set_particle_velocity(torch.from_numpy(snaps).cuda(device))
    rng = np.random.default_rng(7)
    state = np.zeros((npart, 8))
    ints = np.zeros((npart, 3), np.int32)
    state[:, :3] = rng.uniform(-1, 1, (npart, 3))
    state[:, 7] = np.linspace(0.1, 1.0, 10)[np.arange(npart) % 10]
    ints[:, 0] = rng.integers(0, mesh.nel, npart)
    ints[:, 1] = ints[:, 0]
    sd = torch.from_numpy(state).cuda(device)
    idv = torch.from_numpy(ints).cuda(device)
    lib_stream = torch.cuda.ExternalStream(ctx.stream, device=torch.device("cuda", device))
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    t, total_ms, passes = 0.0, 0.0, []
    for step in range(nsteps):
        t += 2 * dt
        e0.record(lib_stream)
        _, _, p = ctx.integrate_particle_equations(sd, idv, t, dt)
        e1.record(lib_stream)
        e1.synchronize()
        total_ms += e0.elapsed_time(e1)
        passes.append(p)
    final = idv.cpu().numpy()
    moved = int((final[:, 0] != ints[:, 0]).sum())
    ms = total_ms / nsteps
    peak, _ = peaks()
    state_bytes = 2 * (8 * 8 + 3 * 4) * npart
    return {"workload": f"{npart} particles in TGV {args.ne}^3 N={n-1}, {nsteps} calls of "
                        "integrate_particle_equations, each over 2 dt (dt = 1e-3), "
                        "library's own particle geometry",
            "ms_per_call": ms,
            "particle_steps_per_s": npart * nsteps / (total_ms * 1e-3),
            "state_bytes_per_call": state_bytes,
            "state_gbs": state_bytes / (ms * 1e-3) / 1e9,
            "state_frac_of_hbm": state_bytes / (ms * 1e-3) / 1e9 / peak,
            "max_passes": max(passes), "changed_element": moved,
            "reseeded": int((final[:, 2] == 5).sum())}


def run_convection(args, ctx, mesh, n, device, calls=25):
    """Dealiased convection over all elements at the time step's two forms:
    the velocity advecting itself (the history term, 1 call per step,
    src/navier_stokes.c:79-83) and a field advected by another (the RK4
    stages of the convection sub-steps, 24 calls per step,
    src/time.c:114-116).  ms_per_step_25_calls = 1 self + 24 general."""
    import numpy as np
    import torch
    X, Y, Z = (ctx.level_data(0, 12 + a) for a in range(3))
    u = torch.from_numpy(np.stack([np.sin(X) * np.cos(Y) * np.cos(Z),
                                   -np.cos(X) * np.sin(Y) * np.cos(Z), 0 * X])).cuda(device)
    out = torch.empty_like(u)
    lib_stream = torch.cuda.ExternalStream(ctx.stream, device=torch.device("cuda", device))
    # the velocity advecting itself (u == v)
    ms, _ = cuda_timed(lib_stream, lambda: ctx.convection_operator(u, u, out), calls, 2)
    # a field advected by another (an RK4 stage: v = a perturbed copy of u)
    v = u * 0.9 + 0.01
    ms_gen, _ = cuda_timed(lib_stream, lambda: ctx.convection_operator(u, v, out), calls, 2)
    # a step's convection sub-steps on the device: the three
    # integrate_convection_rk4 calls of lagrangian_convection_integration
    # (24 general-form convections, DSS and inverse mass per stage)
    ctx.set_velocity_history(u, u * 0.99, u * 0.98, 0.05, 1e-3)
    ut = u.clone()
    tt = [0.05 - 2e-3, 0.05 - 1e-3, 0.05, 0.05 + 1e-3]

    def substeps():
        for a, b, beta in ((0, 1, 1.0 / 3.0), (1, 2, -1.5), (2, 3, 3.0)):
            ctx.integrate_convection_rk4(ut, tt[a], tt[b], 5e-4, beta)
    ms_sub, _ = cuda_timed(lib_stream, substeps, 5, 1)
    npts = mesh.nel * n ** 3
    m = (3 * n) // 2
    # u in and udv out at n points (u == v); the nine stored weights
    # W[a][b] = rho J tinv[a][b] / 2 at the m points
    wbytes = 9 * 8 * mesh.nel * m ** 3
    alg = (3 * 8 + 3 * 8) * npts + wbytes
    alg_gen = (6 * 8 + 3 * 8) * npts + wbytes
    return {"workload": f"TGV {args.ne}^3 N={n-1}, m={m} dealiasing grid, {calls} calls each "
                        "of convection_operator(u, u) and convection_operator(u, v)",
            "ms_per_step_25_calls": (ms + 24 * ms_gen) / calls,
            "self_u_eq_v": {"ms_per_call": ms / calls,
                            "achieved_gbs": alg / (ms / calls * 1e-3) / 1e9,
                            "algorithmic_bytes_per_call": alg},
            "general_u_ne_v": {"ms_per_call": ms_gen / calls,
                               "achieved_gbs": alg_gen / (ms_gen / calls * 1e-3) / 1e9,
                               "algorithmic_bytes_per_call": alg_gen},
            "substeps_ms_per_step": ms_sub / 5}


def tgv_initial_state(ctx, device):
    """The reference's Taylor-Green initial state (src/poisson.c:245-273 with
    the TGV functions, pressure at three levels) built by the library on its
    own grid: the velocity at three levels, the convection and double-curl
    histories of the two older levels (zero at the oldest), the TGV
    pressure."""
    import numpy as np
    import torch
    dev = torch.device("cuda", device)
    X, Y, Z = (ctx.level_data(0, 12 + a) for a in range(3))
    u = torch.from_numpy(np.stack([np.sin(X) * np.cos(Y) * np.cos(Z),
                                   -np.cos(X) * np.sin(Y) * np.cos(Z), 0 * X])).to(dev)
    conv = ctx.convection_operator(u, u, torch.empty_like(u))
    rot = ctx.stokes_operator(0, u, None, torch.empty_like(u))
    p = torch.from_numpy((np.cos(2 * X) + np.cos(2 * Y)) * (np.cos(2 * Z) + 2.0) / 16.0).to(dev)
    zero = torch.zeros_like(u)
    return [u, u.clone(), u.clone()], [conv, conv.clone(), zero], [rot, rot.clone(), zero.clone()], \
        [p, p.clone(), p.clone()]


def run_timestep(args, ctx, mesh, n, device, steps=50, warmup=3, c1=True):
    """C2's time integration: `steps` steps of the reference's
    integrate_navier_stokes (src/navier_stokes.c:224-235) on the device
    (ssg_navier_stokes_step) from the reference's Taylor-Green initial state,
    FP64 and then mixed precision, device time per step; the velocity and
    pressure after the last step against the reference's own run of the
    same steps (tests/golden/c2_tgv16_n8_steps.npz, written by the reference
    compiled in place: a seeded sample of 8192 points and the whole-field
    rms), as L2 errors over the sample relative to its norm and as max
    errors relative to the field's largest magnitude.  `warmup` untimed steps
    from the same state first (graph captures of the solves), then the state
    is set again."""
    import numpy as np
    import torch
    dev = torch.device("cuda", device)
    dt = 1e-3
    rec = None
    path = os.path.join(ROOT, "tests", "golden", "c2_tgv16_n8_steps.npz")
    if steps == 50 and os.path.exists(path):
        rec = np.load(path)
    lib_stream = torch.cuda.ExternalStream(ctx.stream, device=dev)
    state = tgv_initial_state(ctx, device)
    npts = mesh.nel * n ** 3
    out = {"workload": f"TGV {args.ne}^3 N={n-1}: {steps} steps of integrate_navier_stokes on "
                       f"the device, dt {dt}, Re 1600, from the reference's initial state",
           "points": npts, "steps_timed": steps}
    for prec in ("fp64", "mixed"):
        ctx.set_precision(prec)
        if warmup > 0:
            ctx.flow_set(*state, None, 0.0)
            for _ in range(warmup):
                ctx.navier_stokes_step(history=False)
        ctx.flow_set(*state, None, 0.0)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(lib_stream)
        iters = []
        for _ in range(steps):
            last = ctx.navier_stokes_step(history=False)
            iters.append([g["iterations"] for g in last])
        e1.record(lib_stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1) / steps
        r = {"ms_per_step": ms, "steps_per_s": 1e3 / ms,
             "solve_iterations_total": [int(x) for x in np.sum(iters, axis=0)],
             "iterations_last_step": {"pressure": iters[-1][0], "u": iters[-1][1],
                                      "v": iters[-1][2], "w": iters[-1][3]}}
        if rec is not None:
            f = ctx.flow_get()
            idx = rec["sample_index"]
            ug = np.stack([f["u"][0][c].reshape(-1)[idx] for c in range(3)])
            pg = f["p"][0].reshape(-1)[idx]
            ur, pr = rec["snap_u"][-1], rec["snap_p"][-1]
            umax = max(rec["snap_maxabs"][-1, 0], rec["snap_maxabs"][-1, 1])
            r["vs_reference"] = {
                "velocity_l2_rel": float(np.linalg.norm(ug - ur) / np.linalg.norm(ur)),
                "pressure_l2_rel": float(np.linalg.norm(pg - pr) / np.linalg.norm(pr)),
                "velocity_max_rel": float(np.max(np.abs(ug - ur)) / umax),
                "pressure_max_rel": float(np.max(np.abs(pg - pr)) / rec["snap_maxabs"][-1, 3]),
                "reference_iterations_total": [int(x) for x in rec["iterations"].sum(axis=0)],
                "sample": f"{idx.size} seeded points of {npts}, after step {steps}"}
        out[prec] = r
    ctx.set_precision("fp64")
    out["ms_per_step"] = out["fp64"]["ms_per_step"]
    out["mixed_speedup_steps_vs_fp64"] = out["fp64"]["ms_per_step"] / out["mixed"]["ms_per_step"]
    if rec is not None:
        out["reference_cpu_s_per_step"] = float(rec["cpu_s_per_step"])
    if c1:
        # the same at C1 (TGV 4^3, n = 8), the size the reference's own step
        # is timed at in the CPU baseline
        import ssenss_b200 as S
        from ssenss_b200.mesh import tgv_box
        small = S.Context(device)
        try:
            small.set_parameters(dt, 1.0 / 1600.0, 1.0)
            small.setup_mesh(tgv_box(4), n)
            sub = run_timestep(args, small, tgv_box(4), n, device, steps=20, warmup=warmup,
                               c1=False)
            out["c1"] = {"ms_per_step": sub["fp64"]["ms_per_step"],
                         "mixed_ms_per_step": sub["mixed"]["ms_per_step"],
                         "points": sub["points"], "steps": 20}
        finally:
            small.close()
    return out


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
def run_ours(args):
    world, rank, local, pg = dist_setup(args)
    import numpy as np
    import torch
    import ssenss_b200 as S
    from ssenss_b200.mesh import tgv_box

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    mesh = tgv_box(args.ne)
    n = args.n
    ctx = S.Context(local)
    ctx.set_parameters(1e-3, 1.0 / 1600.0, 1.0)
    ctx.setup_mesh(mesh, n)
    ctx.set_graphs(not args.no_graphs)
    tuned = None if args.no_tune else ctx.autotune()
    npts = mesh.nel * n ** 3
    udofs = mesh.unique_nodes(n)
    X, Y, Z = (ctx.level_data(0, 12 + a) for a in range(3))
    bj = ctx.level_data(0, 6)
    f_host = ctx.direct_stiffness_summation(np.ascontiguousarray(bj * tgv_rhs_strong(X, Y, Z)))
    lib_stream = torch.cuda.ExternalStream(ctx.stream, device=dev)
    f = torch.from_numpy(f_host).to(dev)
    u = torch.zeros_like(f)
    torch.cuda.synchronize()

    def barrier():
        torch.cuda.synchronize()
        if pg is not None:
            pg.barrier()
        torch.cuda.synchronize()

    def timed(fn, k, w):
        for _ in range(w):
            fn()
        barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(lib_stream)
        out = [fn() for _ in range(k)]
        e1.record(lib_stream)
        e1.synchronize()
        barrier()
        return e0.elapsed_time(e1), out

    def solve_dev():
        with torch.cuda.stream(lib_stream):
            u.zero_()
        _, info = ctx.solve_poisson_cg(f, u, eps=EPS, history=False)
        return info

    if args.sections == "serve":
        out = run_serving(args, local)
        if rank == 0:
            print(json.dumps({"metric": METRIC, "sections": "serve", "serving": out}))
        ctx.close()
        if pg is not None:
            pg.destroy_process_group()
        return 0

    if args.sections == "particles":
        res = run_particles(args, ctx, mesh, n, local, nsteps=max(1, args.steps))
        if rank == 0:
            print(json.dumps({"metric": METRIC, "sections": "particles", "particles": res}))
        ctx.close()
        return 0

    if args.sections == "channel":
        ctx.close()
        res = run_channel(args, local)
        if rank == 0:
            print(json.dumps({"metric": METRIC, "sections": "channel", "channel": res}))
        return 0

    if args.sections == "extra":
        res = {"convection": run_convection(args, ctx, mesh, n, local),
               "particles": run_particles(args, ctx, mesh, n, local),
               "channel": run_channel(args, local)}
        if rank == 0:
            print(json.dumps({"metric": METRIC, "sections": "extra", **res}))
        ctx.close()
        return 0

    if args.sections == "step":
        res = run_timestep(args, ctx, mesh, n, local,
                           steps=max(1, args.steps) if args.no_time else 50,
                           warmup=max(1, args.warmup), c1=not args.no_time)
        if rank == 0 and not args.no_time:
            print(json.dumps({"metric": METRIC, "sections": "step", "timestep": res}))
        ctx.close()
        return 0

    if args.sections == "conv":
        X3 = np.stack([np.sin(X) * np.cos(Y) * np.cos(Z), -np.cos(X) * np.sin(Y) * np.cos(Z),
                       0 * X])
        uc = torch.from_numpy(X3).to(dev)
        vc = uc * 0.9 + 0.01
        oc = torch.empty_like(uc)
        for _ in range(args.warmup + args.steps):
            ctx.convection_operator(uc, uc, oc)
            ctx.convection_operator(uc, vc, oc)
        torch.cuda.synchronize()
        if rank == 0 and not args.no_time:
            print(json.dumps({"metric": METRIC, "sections": "conv",
                              "convection": run_convection(args, ctx, mesh, n, local)}))
        ctx.close()
        return 0

    if args.sections == "op":
        p = torch.randn(mesh.nel, n, n, n, dtype=torch.float64, device=dev)
        ap = torch.empty_like(p)
        for _ in range(args.warmup + args.steps):
            ctx.local_opeval(S.PRESSURE, p, ap)
            ctx.global_opeval(S.PRESSURE, p, ap)
        torch.cuda.synchronize()
        ctx.close()
        return 0

    if args.sections == "mixed":
        ctx.set_precision("mixed")
        for _ in range(args.warmup):
            solve_dev()
        ms, infos = timed(solve_dev, args.steps, 0)
        if rank == 0:
            print(json.dumps({"metric": METRIC, "sections": "mixed",
                              "ms_per_step": ms / args.steps,
                              "iterations_per_solve":
                                  sum(i["iterations"] for i in infos) / args.steps}))
        ctx.close()
        return 0

    # ---- FP64 (plain form): device-resident timed region -------------------
    ctx.set_precision("fp64")
    clk = Clocks(local)
    for _ in range(args.warmup):
        solve_dev()
    barrier()
    lc0 = ctx.lib.ssg_kernel_launch_count()
    clk.start()
    ms64, infos = timed(solve_dev, args.steps, 0)
    clocks = clk.stop()
    launches = ctx.lib.ssg_kernel_launch_count() - lc0
    u64 = u.cpu().numpy().copy()
    it64 = sum(i["iterations"] for i in infos)
    fnorm = math.sqrt(ctx.global_dot_product(f_host, f_host))
    resid64 = infos[-1]["residual"]
    ms64 = max_over_ranks(pg, ms64, dev)
    dof_it = sum_over_ranks(pg, float(udofs) * it64, dev)
    value = dof_it / (ms64 * 1e-3) / 1e9
    solves_s = sum_over_ranks(pg, float(args.steps), dev) / (ms64 * 1e-3)
    if args.sections == "fp64":
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": value, "unit": UNIT,
                              "ms_per_step": ms64 / args.steps, "sections": "fp64",
                              "iterations_per_solve": it64 / args.steps,
                              "gpu_launches": int(launches)}))
        ctx.close()
        if pg is not None:
            pg.destroy_process_group()
        return 0

    # ---- mixed precision ----------------------------------------------------
    ctx.set_precision("mixed")
    for _ in range(args.warmup):
        solve_dev()
    ms32, infos32 = timed(solve_dev, args.steps, 0)
    u32 = u.cpu().numpy().copy()
    it32 = sum(i["iterations"] for i in infos32)
    ms32 = max_over_ranks(pg, ms32, dev)
    value32 = sum_over_ranks(pg, float(udofs) * it32, dev) / (ms32 * 1e-3) / 1e9
    solves32 = sum_over_ranks(pg, float(args.steps), dev) / (ms32 * 1e-3)
    d64 = u64 - u64.mean()
    d32 = u32 - u32.mean()
    err32 = float(np.abs(d32 - d64).max() / np.abs(d64).max())
    ctx.set_precision("fp64")

    # ---- e2e: public API with pinned host buffers, copies in the region -----
    fh = torch.from_numpy(f_host).pin_memory()
    uh = torch.zeros_like(fh).pin_memory()

    def solve_host():
        uh.zero_()
        _, info = ctx.solve_poisson_cg(fh, uh, eps=EPS, history=False)
        return info

    # two untimed solves: the first runs directly, the second captures the FCG
    # iteration graphs for these host-staged operands
    ms_e2e, infos_e = timed(solve_host, max(3, args.steps // 2), 2)
    ke = max(3, args.steps // 2)
    ms_e2e = max_over_ranks(pg, ms_e2e, dev)
    e2e = sum_over_ranks(pg, float(udofs) * sum(i["iterations"] for i in infos_e), dev) / \
        (ms_e2e * 1e-3) / 1e9

    # ---- roofline of the dominant kernel: level-0 element operator ----------
    # 50 launches back to back on the library's stream between CUDA events
    # (ssg_time_operator), best of three
    op_ms = ctx.time_operator(S.PRESSURE, 50) * 1e-3
    op_ms_h = ctx.time_operator(S.X_VELOCITY, 50) * 1e-3
    alg = OP_BYTES_PER_POINT * npts
    peak, peak_kind = peaks()
    achieved = alg / (op_ms * 1e-3) / 1e9
    # the three kernels of a smoother CG iteration at every level, each timed
    # alone; algorithmic bytes per point: DSS + dot 24 (in, y, out), CG update
    # 65 (x, p, r, ap, dinv, multiplicity in; x, r, z out)
    smoother = {}
    for lev, m in enumerate(ctx.orders):
        t = ctx.time_smoother(lev, 50)
        pts = mesh.nel * m ** 3
        smoother[str(m)] = {
            "us_per_launch": t,
            "dss_dot_frac": 24 * pts / (t["dss_dot"] * 1e-6) / 1e9 / peak,
            "cg_update_frac": 65 * pts / (t["cg_update"] * 1e-6) / 1e9 / peak}

    # ---- Helmholtz (velocity) solve, reported beside -------------------------
    fvel = torch.from_numpy(ctx.direct_stiffness_summation(
        np.ascontiguousarray(bj * np.sin(X) * np.cos(Y) * np.cos(Z)))).to(dev)
    uvel = torch.zeros_like(fvel)

    def helm():
        with torch.cuda.stream(lib_stream):
            uvel.zero_()
        _, info = ctx.solve_helmholtz_cg(S.X_VELOCITY, fvel, uvel, eps=EPS, history=False)
        return info

    hms, hinfo = timed(helm, 5, 1)

    serving = run_serving(args, local) if args.serve_requests > 0 else None
    extra = {}
    if not args.no_extra:
        extra["convection"] = run_convection(args, ctx, mesh, n, local)
        extra["timestep"] = run_timestep(args, ctx, mesh, n, local)
        extra["particles"] = run_particles(args, ctx, mesh, n, local)
        extra["channel"] = run_channel(args, local)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            import oracle
            if oracle.reference_available():
                secs, its = reference_sample(mesh, n, f_host, int(round(it64 / args.steps)))
                cpu = {"value": udofs * its / secs / 1e9, "unit": UNIT, "cores": 1,
                       "kind": "reference",
                       "sample": (f"{its} FCG+p-MG iterations of the same solve "
                                  f"(reference sources compiled in place, 1 thread): "
                                  f"{secs:.1f} s")}
        except Exception as ex:  # reported, never fatal
            cpu = {"value": None, "unit": UNIT, "cores": 1, "kind": "reference",
                   "sample": f"failed: {ex}"}
        if cpu is not None and not args.no_extra:
            try:
                cpu["timestep_c1"] = {
                    "ms_per_step": 1e3 * reference_step_sample(),
                    "sample": ("integrate_navier_stokes on C1 (TGV 4^3, n = 8), 2 steps after "
                               "one untimed step, reference compiled in place, 1 thread")}
            except Exception as ex:  # reported, never fatal
                cpu["timestep_c1"] = {"ms_per_step": None, "sample": f"failed: {ex}"}

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms64 / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {
            "workload": (f"TGV {args.ne}^3 hex N={n-1} (n={n}) pressure Poisson, "
                         f"FCG+p-MG to sqrt((r.r)_w)<=1e-10 from zero"),
            "elements": mesh.nel, "n": n, "mg_orders": ctx.orders,
            "unique_dofs": udofs, "local_points": npts,
            "parallelism": f"replicas x{world}",
            "launch_shapes": ({str(k): v for k, v in tuned.items()} if tuned
                              else "default (autotuner off)"),
            "cuda_graphs": "V-cycle captured" if not args.no_graphs else "off",
            "l2": "inputs larger than L2 (level-0 factors 100 MB + FCG vectors 420 MB)",
        },
        "iterations_per_solve": it64 / args.steps,
        "solves_per_s": solves_s,
        "residual": {"absolute": resid64, "relative": resid64 / fnorm,
                     "stop": "absolute sqrt((r.r)_w) <= 1e-10 (the reference's criterion, "
                             "src/navier_stokes.c:94-99); relative = absolute / sqrt((f.f)_w)"},
        "mixed": {"value": value32, "unit": UNIT, "solves_per_s": solves32,
                  "iterations_per_solve": it32 / args.steps,
                  "ms_per_step": ms32 / args.steps,
                  "speedup_solves_vs_fp64": solves32 / solves_s,
                  "max_rel_diff_vs_fp64": err32,
                  "residual": {"absolute": infos32[-1]["residual"],
                               "relative": infos32[-1]["residual"] / fnorm}},
        "helmholtz": {"ms_per_solve": hms / 5,
                      "iterations": hinfo[0]["iterations"]},
        "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": 2 * 8 * npts,
                "d2h_bytes_per_step": 8 * npts, "ms_per_step": ms_e2e / ke},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak,
                     "traffic": OP_TRAFFIC_BYTES if (n == 8 and args.ne == NE) else None,
                     "kernel": ("k_ax8_dmma<double> (level-0 Laplacian, FP64 DMMA)"
                                if n == 8 else f"k_ax<{n},double> (level-0 Laplacian)"),
                     "us_per_launch": op_ms * 1e3,
                     "bytes_per_point": OP_BYTES_PER_POINT,
                     "helmholtz": {"us_per_launch": op_ms_h * 1e3,
                                   "achieved": 72 * npts / (op_ms_h * 1e-3) / 1e9,
                                   "frac": 72 * npts / (op_ms_h * 1e-3) / 1e9 / peak},
                     "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)"},
        "smoother_kernels": smoother,
        "serving": serving,
        "channel_c3": extra.get("channel"),
        "particles_c4": extra.get("particles"),
        "convection": extra.get("convection"),
        "timestep": extra.get("timestep"),
        "cpu_baseline": cpu,
        "gpu_launches": int(launches),
        "clocks": clocks,
    }
    ctx.close()
    if rank == 0:
        print(json.dumps(line))
    if pg is not None:
        pg.destroy_process_group()
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
