"""ctypes binding of libssenss_b200.so (the C ABI of include/ssenss_b200.h).

The shared library is built in place by ssenss_b200/csrc/Makefile.  There is
no fallback: importing a compute entry point without the library raises.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libssenss_b200.so")

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


class SolveInfo(C.Structure):
    _fields_ = [
        ("iterations", C.c_int),
        ("residual", C.c_double),
        ("initial_residual", C.c_double),
        ("solve_ms", C.c_double),
        ("history", _dp),
        ("history_cap", C.c_int),
        ("history_len", C.c_int),
    ]


class Request(C.Structure):
    _fields_ = [
        ("nel", C.c_int),
        ("vertices", _dp),
        ("neigh", _ip),
        ("mesh_key", C.c_ulonglong),
        ("n", C.c_int),
        ("lam", C.c_double),
        ("eps", C.c_double),
        ("relative", C.c_int),
        ("precision", C.c_int),
        ("max_iter", C.c_int),
        ("deadline_ms", C.c_double),
    ]


class FlowFields(C.Structure):
    """ssg_flow_fields: history levels newest first; u, conv, rot and f
    three fields each, p one."""
    _fields_ = [
        ("u", C.c_void_p * 3),
        ("conv", C.c_void_p * 3),
        ("rot", C.c_void_p * 3),
        ("p", C.c_void_p * 3),
        ("f", C.c_void_p),
    ]


class ServerStats(C.Structure):
    _fields_ = [
        ("submitted", C.c_ulonglong), ("completed", C.c_ulonglong),
        ("failed", C.c_ulonglong), ("cancelled", C.c_ulonglong),
        ("rejected", C.c_ulonglong),
        ("p50_ms", C.c_double), ("p99_ms", C.c_double), ("mean_ms", C.c_double),
        ("max_ms", C.c_double), ("queue_p50_ms", C.c_double), ("queue_p99_ms", C.c_double),
        ("solves_per_s", C.c_double),
        ("hbm_in_use", C.c_size_t), ("hbm_peak", C.c_size_t), ("hbm_budget", C.c_size_t),
        ("mesh_hits", C.c_ulonglong), ("mesh_misses", C.c_ulonglong),
        ("evictions", C.c_ulonglong),
        ("max_active_seen", C.c_int), ("resident_contexts", C.c_int),
        ("batches", C.c_ulonglong), ("batched_requests", C.c_ulonglong),
    ]


# (name, restype, argtypes) of every symbol include/ssenss_b200.h declares
SIGNATURES = [
    ("ssg_create", C.c_int, [C.c_int, C.POINTER(C.c_void_p)]),
    ("ssg_create_on_stream", C.c_int, [C.c_int, C.c_void_p, C.POINTER(C.c_void_p)]),
    ("ssg_destroy", None, [C.c_void_p]),
    ("ssg_status_string", C.c_char_p, [C.c_int]),
    ("ssg_last_error", C.c_char_p, [C.c_void_p]),
    ("ssg_stream", C.c_void_p, [C.c_void_p]),
    ("ssg_set_parameters", C.c_int, [C.c_void_p, C.c_double, C.c_double, C.c_double]),
    ("ssg_set_precision", C.c_int, [C.c_void_p, C.c_int]),
    ("ssg_set_graphs", C.c_int, [C.c_void_p, C.c_int]),
    ("ssg_setup_mesh", C.c_int, [C.c_void_p, C.c_int, C.c_int, _dp, _ip]),
    ("ssg_setup_connectivity", C.c_int, [C.c_void_p, C.c_int, _ip]),
    ("ssg_setup_level", C.c_int, [C.c_void_p, C.c_int, C.c_int, _dp, _dp, _dp, _dp,
                                  _dp, _dp]),
    ("ssg_setup_finish", C.c_int, [C.c_void_p]),
    ("ssg_setup_dealias", C.c_int, [C.c_void_p, C.c_int, _dp, _dp, _dp, _dp, _dp]),
    ("ssg_setup_particle_geometry", C.c_int, [C.c_void_p, _dp, _dp, _dp]),
    ("ssg_mesh_info", C.c_int, [C.c_void_p, _ip, _ip, _ip, _ip]),
    ("ssg_level_data", C.c_int, [C.c_void_p, C.c_int, C.c_int, _dp]),
    ("ssg_global_opeval", C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]),
    ("ssg_local_opeval", C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]),
    ("ssg_direct_stiffness_summation", C.c_int, [C.c_void_p, C.c_void_p]),
    ("ssg_global_dot_product", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, _dp]),
    ("ssg_weighted_dot_noalloc", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t,
                                           C.c_void_p, C.c_void_p]),
    ("ssg_inverse_mass", C.c_int, [C.c_void_p, C.c_void_p]),
    ("ssg_solve_poisson_cg", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_double,
                                       C.c_int, C.POINTER(SolveInfo)]),
    ("ssg_solve_helmholtz_cg", C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p,
                                         C.c_double, C.c_int, C.POINTER(SolveInfo)]),
    ("ssg_conjugate_gradient", C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p,
                                         C.c_double, C.c_int, C.POINTER(SolveInfo)]),
    ("ssg_solve_helmholtz_segments", C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_void_p,
                                               C.c_void_p, C.c_void_p, C.c_void_p,
                                               C.c_void_p, C.c_int, C.POINTER(SolveInfo)]),
    ("ssg_jacobi_preconditioner", C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]),
    ("ssg_multigrid_preconditioner", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p,
                                               C.c_double]),
    ("ssg_convection_operator", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p,
                                          C.c_void_p]),
    ("ssg_convection_elements", C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_void_p,
                                          C.c_void_p, C.c_void_p]),
    ("ssg_kernel_launch_count", C.c_ulonglong, []),
    ("ssg_autotune", C.c_int, [C.c_void_p, C.c_int]),
    ("ssg_set_setup_options", C.c_int, [C.c_void_p, C.c_uint]),
    ("ssg_set_svv", C.c_int, [C.c_void_p, C.c_int, C.c_double]),
    ("ssg_set_velocity_history", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                           C.c_double, C.c_double]),
    ("ssg_integrate_convection_rk4", C.c_int, [C.c_void_p, C.c_void_p, C.c_double, C.c_double,
                                               C.c_double, C.c_double]),
    ("ssg_flow_set", C.c_int, [C.c_void_p, C.POINTER(FlowFields), C.c_double]),
    ("ssg_flow_get", C.c_int, [C.c_void_p, C.POINTER(FlowFields), _dp]),
    ("ssg_navier_stokes_step", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                         C.POINTER(SolveInfo)]),
    ("ssg_stokes_operator", C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p,
                                      C.c_void_p]),
    ("ssg_memory_info", C.c_int, [C.c_void_p, C.POINTER(C.c_size_t)]),
    ("ssg_request_bytes", C.c_size_t, [C.c_int, C.c_int, C.c_int]),
    ("ssg_gll", C.c_int, [C.c_int, _dp, _dp]),
    ("ssg_server_create", C.c_int, [C.c_int, C.c_size_t, C.c_int, C.POINTER(C.c_void_p)]),
    ("ssg_server_submit", C.c_int, [C.c_void_p, C.POINTER(Request), _dp, _dp,
                                    C.POINTER(C.c_ulonglong)]),
    ("ssg_server_wait", C.c_int, [C.c_void_p, C.c_ulonglong, C.c_double,
                                  C.POINTER(C.c_int), C.POINTER(SolveInfo)]),
    ("ssg_server_cancel", C.c_int, [C.c_void_p, C.c_ulonglong]),
    ("ssg_server_drain", C.c_int, [C.c_void_p, C.c_double]),
    ("ssg_server_get_stats", C.c_int, [C.c_void_p, C.POINTER(ServerStats)]),
    ("ssg_server_set_batching", C.c_int, [C.c_void_p, C.c_int, C.c_size_t]),
    ("ssg_server_destroy", None, [C.c_void_p]),
    ("ssg_tuning", C.c_int, [C.c_int, _ip, _ip, _ip]),
    ("ssg_time_operator", C.c_int, [C.c_void_p, C.c_int, C.c_int, _dp]),
    ("ssg_time_smoother", C.c_int, [C.c_void_p, C.c_int, C.c_int, _dp]),
    ("ssg_set_particle_velocity", C.c_int, [C.c_void_p, C.c_void_p]),
    ("ssg_integrate_particle_equations", C.c_int, [C.c_void_p, C.c_size_t, C.c_void_p,
                                                   C.c_void_p, C.c_double, C.c_double,
                                                   _ip]),
]

_LIB = None


def load():
    """Load libssenss_b200.so; raises when it has not been built."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `make -C ssenss_b200/csrc` "
                "(there is no CPU fallback)")
        lib = C.CDLL(LIB_PATH)
        for name, res, args in SIGNATURES:
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = lib
    return _LIB
