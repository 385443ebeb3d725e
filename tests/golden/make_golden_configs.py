"""Pin the reference's own C2 solve: the residual history of the full-size
TGV pressure solve (16^3 elements, N = 7, FCG + p-multigrid to the absolute
1e-10 from zero) computed by the reference compiled in place
(oracle/_ref/libssenss_ref.so, OPENBLAS_NUM_THREADS=1), written to
tests/golden/c2_tgv16_n8.json.  tests/test_gpu_configs.py reruns the
reference live and checks it against this record before it compares the GPU
solve with that live run.

Usage (about a minute, where the reference sources were present at build):
    OPENBLAS_NUM_THREADS=1 python tests/golden/make_golden_configs.py
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

import oracle as O  # noqa: E402
from ssenss_b200.mesh import tgv_box  # noqa: E402
from test_gpu_configs import tgv_pressure_rhs  # noqa: E402


def main():
    mesh, n = tgv_box(16), 8
    ref = O.Reference(mesh, n)
    try:
        f = tgv_pressure_rhs(ref, n)
        u, hist = ref.solve_poisson(f, np.zeros_like(f))
    finally:
        ref.close()
    rec = {"workload": "TGV periodic 16^3 elements, N = 7 (n = 8), pressure Poisson "
                       "of the TGV pressure, FCG + p-MG to sqrt((r.r)_w) <= 1e-10 from zero",
           "iterations": int(len(hist)), "history": [float(h) for h in hist],
           "solution_max_abs": float(np.max(np.abs(u))),
           "solution_mean": float(np.mean(u))}
    with open(os.path.join(HERE, "c2_tgv16_n8.json"), "w") as fh:
        json.dump(rec, fh, indent=1)
    print(rec["iterations"], rec["history"][-1])


if __name__ == "__main__":
    main()
