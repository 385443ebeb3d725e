import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def gpu_ctx_factory():
    """Build ssenss_b200 contexts on cuda:0 (GPU tests only)."""
    import ssenss_b200 as S

    made = []

    def make(mesh, n, dt=1e-3, visc=1.0 / 1600.0, precision="fp64"):
        ctx = S.Context(0)
        ctx.set_parameters(dt, visc, 1.0)
        ctx.set_precision(precision)
        ctx.setup_mesh(mesh, n)
        made.append(ctx)
        return ctx

    yield make
    for c in made:
        c.close()


EPS = 1e-10


SOLVE_REL = 1e-11


def assert_solution_close(u_g, u_o, orc, solve, f):
    """GPU solution u_g against the oracle's u_o = solve(f, 0): within 1e-11
    relative (max |du| / max |u|), or, where the solve itself is not
    determined that closely by FP64 arithmetic, within twice the oracle's
    own rounding spread (Oracle.rounding_spread: the same oracle solve with
    its dot products perturbed by one rounding).  Both tolerances stated
    here; the spread is only measured when the plain bound is missed."""
    d = float(np.max(np.abs(u_g - u_o)) / max(np.max(np.abs(u_o)), 1e-300))
    if d < SOLVE_REL:
        return d
    spread = orc.rounding_spread(solve, f)
    assert d < 2.0 * spread, (d, spread)
    return d


def same_stop(it_g, h_g, h_o):
    """True when both runs stop at the same iteration.  Otherwise they may
    differ by one iteration only where the residual crosses the absolute
    stop 1e-10 within a factor 2 at the deciding iteration: near eps the
    V-cycle's inner CG solves, which stop on the same absolute eps, take
    different numbers of steps in any two FP64 implementations (the
    reference and the oracle already differ by 20 % in the residual there),
    and the outer history follows.  The caller then skips the 1e-11
    solution comparison (the two iterates are one correction apart)."""
    it_o = len(h_o)
    if it_g == it_o:
        return True
    assert abs(it_g - it_o) == 1, (it_g, it_o)
    k = min(it_g, it_o) - 1   # the iteration after which one run stopped
    for h in (h_g[k], h_o[k]):
        assert 0.5 * EPS <= h <= 2 * EPS, (it_g, it_o, h_g[k], h_o[k])
    return False


def history_deviation(h_g, h_o):
    """|h_g - h_o| over the common iterations of two residual histories."""
    k = min(len(h_g), len(h_o))
    return np.abs(np.asarray(h_g[:k], dtype=float) - np.asarray(h_o[:k], dtype=float))


def check_history(h_g, h_o, floor=0.0):
    """Residual histories of two runs of the same solve, over the common
    iterations: within 1e-9 of the first residual wherever the residual is
    above 1e-4 of it, within 1e-7 of it below.  Near the stop the residual
    is set by the rounding of the V-cycle's inner CG solves, which stop on
    the same absolute eps and so take different inner iteration counts in
    any two FP64 implementations (the oracle and the reference differ there
    by up to 20 % of the residual itself); both bounds are stated here.
    floor: an absolute deviation always accepted (the rounding level of the
    problem's data, stated by the caller).  Returns the largest deviation
    relative to the first residual."""
    d = history_deviation(h_g, h_o)
    if d.size == 0:
        return 0.0
    h_o = np.asarray(h_o[:d.size], dtype=float)
    h0 = h_o[0]
    hi = h_o > 1e-4 * h0
    assert np.all(d[hi] <= np.maximum(1e-9 * h0, floor)), d / h0
    assert np.all(d <= np.maximum(1e-7 * h0, floor)), d / h0
    return float(np.max(d) / h0)
