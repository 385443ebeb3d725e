"""The allocation-free weighted inner product (ssg_weighted_dot_noalloc).

It serves callers that cannot let the library call cudaMalloc -- a process
that gives all device memory to its own pool under a fixed budget.  The
entry point keeps its partial sums in one fixed device array shared by all
calls, so this file is collected last and the check runs twice in a row:
the second call must not be disturbed by what the first left in the array.
Results are compared, through the C ABI, with ssg_global_dot_product under
the dot-product tolerance of the other parity tests, and at a size of many
hundred blocks with an exactly rounded sum of the same products on the host.
"""
import ctypes as C
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _dev(t):
    return C.c_void_p(t.data_ptr())


def test_noalloc_dot_matches_context_dot():
    import torch

    import ssenss_b200 as S
    from ssenss_b200.mesh import tgv_box

    lib = S._lib.load()
    mesh, n = tgv_box(3), 8
    ctx = S.Context(0)
    ctx.setup_mesh(mesh, n)
    w_host = ctx.level_data(0, 9)                      # 1 / multiplicity
    w = torch.from_numpy(w_host).cuda()
    result = torch.zeros(1, dtype=torch.float64, device="cuda")
    rng = np.random.default_rng(11)
    for call in range(2):
        x_host = rng.standard_normal(w_host.shape)
        y_host = rng.standard_normal(w_host.shape)
        x = torch.from_numpy(x_host).cuda()
        y = torch.from_numpy(y_host).cuda()
        torch.cuda.synchronize()
        st = lib.ssg_weighted_dot_noalloc(_dev(x), _dev(y), _dev(w), x.numel(),
                                          _dev(result), None)
        assert st == 0, st
        torch.cuda.synchronize()
        got = float(result.item())
        want = ctx.global_dot_product(x_host, y_host)
        scale = np.sqrt(ctx.global_dot_product(x_host, x_host) *
                        ctx.global_dot_product(y_host, y_host))
        assert abs(got - want) <= 1e-12 * scale, (call, got, want)
    ctx.close()


def test_noalloc_dot_many_blocks_matches_exact_sum():
    """2,000,000 points (977 partial sums, so the final kernel's strided loop
    over the partials runs) against math.fsum of the products (x*w)*y."""
    import torch

    import ssenss_b200 as S

    lib = S._lib.load()
    rng = np.random.default_rng(12)
    npts = 2_000_000
    w_host = 1.0 / rng.choice([1.0, 2.0, 4.0, 8.0], npts)
    result = torch.zeros(1, dtype=torch.float64, device="cuda")
    for call in range(2):
        x_host = rng.standard_normal(npts)
        y_host = rng.standard_normal(npts)
        x, y, w = (torch.from_numpy(a).cuda() for a in (x_host, y_host, w_host))
        torch.cuda.synchronize()
        assert lib.ssg_weighted_dot_noalloc(_dev(x), _dev(y), _dev(w), npts, _dev(result),
                                            None) == 0
        torch.cuda.synchronize()
        want = math.fsum((x_host * w_host) * y_host)
        scale = np.linalg.norm(x_host) * np.linalg.norm(y_host)
        assert abs(float(result.item()) - want) <= 1e-12 * scale, (call, result.item(), want)


def test_noalloc_rejects_bad_arguments():
    import torch

    import ssenss_b200 as S

    lib = S._lib.load()
    a = torch.ones(16, dtype=torch.float64, device="cuda")
    r = torch.zeros(1, dtype=torch.float64, device="cuda")
    too_many = 65536 * 2048 + 1
    assert lib.ssg_weighted_dot_noalloc(_dev(a), _dev(a), _dev(a), too_many, _dev(r),
                                        None) == 1
    h = np.ones(16)
    hp = C.c_void_p(h.ctypes.data)
    assert lib.ssg_weighted_dot_noalloc(hp, _dev(a), _dev(a), 16, _dev(r), None) == 1
    assert lib.ssg_weighted_dot_noalloc(_dev(a), _dev(a), _dev(a), 16, _dev(r), None) == 0
    torch.cuda.synchronize()
    assert float(r.item()) == 16.0
