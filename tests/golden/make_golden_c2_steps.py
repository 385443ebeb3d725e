"""Pin the reference's own C2 time integration: 50 steps of
integrate_navier_stokes (src/navier_stokes.c:224-235) on the Taylor-Green
vortex, periodic 16^3 elements, N = 7 (n = 8, 2,097,152 points), dt = 1e-3,
Re = 1600, from the reference's initial state (src/poisson.c:245-273:
velocity at three levels, convection and double-curl histories; the TGV
pressure at three levels), computed by the reference compiled in place
(oracle/_ref/libssenss_ref.so, one thread).  Written to
tests/golden/c2_tgv16_n8_steps.npz:

  iterations   (50, 4)    each step's solves (pressure, then u, v, w)
  history      (50, 4, H) their residual histories, NaN-padded
  sample_index (S,)       a seeded sample of flat point indices into
                          (nel, n, n, n), S = 8192
  snap_steps   (3,)       the steps after which the fields were recorded
  snap_u       (3, 3, S)  velocity components at the sample
  snap_p       (3, S)     pressure at the sample
  snap_rms     (3, 4)     root mean square over all points of u, v, w, p
  snap_maxabs  (3, 4)     largest magnitude over all points of u, v, w, p
  time         (3,)       solver time after those steps
  cpu_s_per_step ()       the reference's wall time per step on the
                          machine that wrote the file

The whole fields are 67 MB a level; the sample and the whole-field norms
stand in for them.  tests/test_gpu_configs.py runs the same 50 steps on the
device from the same initial state (FP64 and mixed precision) and compares
them with this record; bench.py reports the same deviations.

Usage (about 40 minutes of one core, where the reference sources were
present at build):
    OPENBLAS_NUM_THREADS=1 python tests/golden/make_golden_c2_steps.py
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle as O  # noqa: E402
from ssenss_b200.mesh import tgv_box  # noqa: E402

STEPS = 50
SNAPS = (1, 10, 50)
SAMPLE = 8192
HMAX = 64


def main():
    mesh, n = tgv_box(16), 8
    npts = mesh.nel * n ** 3
    idx = np.sort(np.random.default_rng(20261204).choice(npts, SAMPLE, replace=False))
    iters = np.zeros((STEPS, 4), np.int32)
    hist = np.full((STEPS, 4, HMAX), np.nan)
    snap_u = np.zeros((len(SNAPS), 3, SAMPLE))
    snap_p = np.zeros((len(SNAPS), SAMPLE))
    rms = np.zeros((len(SNAPS), 4))
    maxabs = np.zeros((len(SNAPS), 4))
    times = np.zeros(len(SNAPS))
    ref = O.Reference(mesh, n, dt=1e-3, visc=1.0 / 1600.0, dens=1.0)
    try:
        ref.init_tgv()
        t0 = time.time()
        for s in range(STEPS):
            ref.ns_step()
            log = ref.step_log()
            assert [k for k, _, _ in log] == [0, 1, 1, 1], log
            for j, (_, _, h) in enumerate(log):
                iters[s, j] = len(h)
                hist[s, j, :min(len(h), HMAX)] = h[:HMAX]
            if s + 1 in SNAPS:
                k = SNAPS.index(s + 1)
                fields = [ref.get_field(c, 0) for c in range(4)]
                for c in range(4):
                    flat = fields[c].reshape(-1)
                    if c < 3:
                        snap_u[k, c] = flat[idx]
                    else:
                        snap_p[k] = flat[idx]
                    rms[k, c] = np.sqrt(np.mean(flat * flat))
                    maxabs[k, c] = np.max(np.abs(flat))
                times[k] = ref.time()
            print(s + 1, iters[s].tolist(), f"{time.time() - t0:.0f} s", flush=True)
        per_step = (time.time() - t0) / STEPS
    finally:
        ref.close()
    np.savez(os.path.join(HERE, "c2_tgv16_n8_steps.npz"), iterations=iters, history=hist,
             sample_index=idx, snap_steps=np.array(SNAPS), snap_u=snap_u, snap_p=snap_p,
             snap_rms=rms, snap_maxabs=maxabs, time=times, cpu_s_per_step=per_step)


if __name__ == "__main__":
    main()
