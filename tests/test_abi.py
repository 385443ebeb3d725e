"""The C-ABI library loads and exports every entry point include/ssenss_b200.h
declares (no GPU needed)."""
import ctypes
import os
import re

import pytest

from conftest import ROOT


def header_symbols():
    src = open(os.path.join(ROOT, "include", "ssenss_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(ssg_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_entry_points():
    syms = header_symbols()
    for s in ("ssg_global_opeval", "ssg_solve_poisson_cg", "ssg_solve_helmholtz_cg",
              "ssg_direct_stiffness_summation", "ssg_convection_operator",
              "ssg_integrate_particle_equations"):
        assert s in syms


def test_library_exports_every_declared_symbol():
    from ssenss_b200 import _lib
    lib = ctypes.CDLL(_lib.LIB_PATH)
    missing = [s for s in header_symbols() if not hasattr(lib, s)]
    assert not missing, missing
    bound = {name for name, _, _ in _lib.SIGNATURES}
    assert set(header_symbols()) <= bound


def test_status_strings():
    from ssenss_b200 import _lib
    lib = _lib.load()
    for s in range(11):
        assert lib.ssg_status_string(s)


def test_no_device_fails_cleanly():
    """Without a usable GPU the library refuses (no CPU fallback)."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    import ssenss_b200 as S
    with pytest.raises(S.SsgError) as ei:
        S.Context(0)
    assert ei.value.status == 2


def test_request_bytes_estimate_is_monotone():
    """The serving loop's admission estimate (host only, no GPU)."""
    import ssenss_b200 as S
    assert S.request_bytes(8, 0) == 0
    assert S.request_bytes(13, 27) == 0
    prev = 0
    for nel in (8, 27, 512, 4096):
        b = S.request_bytes(8, nel, "fp64")
        assert b > prev
        prev = b
        assert S.request_bytes(8, nel, "mixed") > b
    for n in (6, 8, 10, 12):
        assert S.request_bytes(n, 64) < S.request_bytes(n + 1 if n < 12 else 12, 64) or n == 12
    # at least the level-0 operator factors and the 24 FCG vectors
    assert S.request_bytes(8, 4096, "fp64") > 4096 * 512 * (48 + 24 * 8)


def test_gll_matches_the_oracle():
    """ssg_gll (host only): the library's GLL points and weights against the
    oracle's restatement of src/basis.c, every order the library builds."""
    import numpy as np
    import oracle as O
    from ssenss_b200 import _lib
    lib = _lib.load()
    for n in range(2, 19):
        x, w = np.empty(n), np.empty(n)
        assert lib.ssg_gll(n, x.ctypes.data_as(_lib._dp), w.ctypes.data_as(_lib._dp)) == 0
        xo, wo = O.Oracle.gll(n)
        assert np.max(np.abs(x - xo)) <= 4e-16 and np.max(np.abs(w - wo)) <= 4e-16, n
        assert x[0] == -1.0 and x[-1] == 1.0
        assert abs(w.sum() - 2.0) < 1e-14
    x, w = np.empty(1), np.empty(1)
    assert lib.ssg_gll(1, x.ctypes.data_as(_lib._dp), w.ctypes.data_as(_lib._dp)) == 1


def test_default_launch_shapes():
    """ssg_tuning (host only) before any autotuning: the FP64 tensor-core
    operator at n = 8 (0), the line-form operator elsewhere (-1), positive
    grid shapes, orders out of range rejected."""
    import ssenss_b200 as S
    t8 = S.tuning(8)
    assert t8["ax_elements_per_block"] == 0
    for n in (2, 4, 6, 10, 12):
        t = S.tuning(n)
        assert t["ax_elements_per_block"] == -1
        assert t["dss_blocks_per_sm"] >= 1 and t["vector_blocks_per_sm"] >= 1
    for bad in (1, 19):
        with pytest.raises(S.SsgError):
            S.tuning(bad)
