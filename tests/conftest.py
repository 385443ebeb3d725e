import os
import sys

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
