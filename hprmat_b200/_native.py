"""ctypes binding of ``libhprmat_b200.so`` (the C ABI of include/hprmat_b200.h).

The library is loaded from ``hprmat_b200/lib/`` inside the package.  There is no
fallback: if the library is missing or cannot be loaded, every entry point raises.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libhprmat_b200.so")

OK = 0
ERR_ARG = -1
ERR_CUDA = -2
ERR_OOM = -3
ERR_TIMEOUT = -4
ERR_UNSUPPORTED = -5
ERR_NODEVICE = -6
SINGULAR = 1
PIVOT_GROWTH = 2
NOT_CONVERGED = 99

# HPRMAT_B200_ABI_VERSION of include/hprmat_b200.h: the struct mirrors below follow it
ABI_VERSION = 101

PREC_FP64 = 0
PREC_MIXED = 1
SOLVER_B200 = 7

# Every symbol include/hprmat_b200.h declares.
EXPORTED = (
    "hprmat_b200_default_opts", "hprmat_b200_create", "hprmat_b200_destroy", "hprmat_b200_set_opts",
    "hprmat_b200_set_stream", "hprmat_b200_rmat_ini", "hprmat_b200_rmatrix", "hprmat_b200_rmatrix_device",
    "hprmat_b200_solve_linear", "hprmat_b200_solve_linear_device", "hprmat_b200_solve_rmatrix",
    "gpu_b200_solve_mixed_", "gpu_b200_solve_double_", "gpu_b200_finalize_", "hprmat_b200_status_string",
    "hprmat_b200_last_error", "hprmat_b200_version", "hprmat_b200_boundary",
    "hprmat_b200_solve_linear_noalloc", "hprmat_b200_rmatrix_scan", "hprmat_b200_scan_autotune",
    "hprmat_b200_scan_tune_get", "hprmat_b200_scan_tune_set", "hprmat_b200_rmatrix_scan_shifted",
    "hprmat_b200_rmatrix_adjoint", "hprmat_b200_rmatrix_wf", "hprmat_b200_rmatrix_wf_device",
    "hprmat_b200_wf_print", "hprmat_b200_rmatrix_full", "hprmat_b200_rmatrix_x", "hprmat_b200_adjoint_from_x",
    "hprmat_b200_rmatrix_x_device", "hprmat_b200_adjoint_from_x_device",
    # include/hprmat_b200_dev.h
    "hprmat_b200_dev_tc_update", "hprmat_b200_dev_split_planes", "hprmat_b200_dev_set_profile",
    "hprmat_b200_dev_counters", "hprmat_b200_dev_wave_trace", "hprmat_b200_dev_wave_trace_read",
    "hprmat_b200_dev_panel_trace_read", "hprmat_b200_dev_set_tuning", "hprmat_b200_dev_mesh",
    "hprmat_b200_dev_factorizations", "hprmat_b200_dev_wait_probe", "hprmat_b200_dev_binary_version",
    "hprmat_b200_dev_zgemm", "hprmat_b200_dev_hessenberg", "hprmat_b200_dev_hess_timings",
)


class Opts(ctypes.Structure):
    _fields_ = [("precision", ctypes.c_int), ("max_refine", ctypes.c_int), ("tol", ctypes.c_double),
                ("surface_tol", ctypes.c_double), ("panel_nb", ctypes.c_int), ("reuse_factors", ctypes.c_int),
                ("estimate_condition", ctypes.c_int), ("growth_error", ctypes.c_int),
                ("reserved", ctypes.c_int * 1)]


class Stats(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int), ("info", ctypes.c_int), ("refine_steps", ctypes.c_int), ("inner_iterations", ctypes.c_int),
                ("nb", ctypes.c_int), ("n", ctypes.c_int), ("nrhs", ctypes.c_int),
                ("rel_residual", ctypes.c_double), ("surface_change", ctypes.c_double),
                ("residual_floor", ctypes.c_double), ("floor_history", ctypes.c_double * 9),
                ("residual_history", ctypes.c_double * 9),
                ("ms_assemble", ctypes.c_double), ("ms_factor", ctypes.c_double), ("ms_solve", ctypes.c_double),
                ("ms_refine", ctypes.c_double), ("ms_umatrix", ctypes.c_double), ("ms_total", ctypes.c_double),
                ("factorizations", ctypes.c_int), ("fp64_fallback", ctypes.c_int), ("pivot_growth", ctypes.c_double),
                ("cond_estimate", ctypes.c_double), ("ms_condest", ctypes.c_double)]

    def as_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_ if k not in ("residual_history", "floor_history")}
        d["floor_history"] = [self.floor_history[i] for i in range(9) if self.floor_history[i] != 0.0]
        d["residual_history"] = [self.residual_history[i] for i in range(9) if self.residual_history[i] != 0.0]
        return d


class ScanBlock(ctypes.Structure):
    """hprmat_b200_scan_block (include/hprmat_b200.h)."""
    _fields_ = [("nch", ctypes.c_int), ("lval", ctypes.POINTER(ctypes.c_int)), ("cpot", ctypes.POINTER(ctypes.c_double)),
                ("ncp1", ctypes.c_int), ("nenergies", ctypes.c_int), ("qk", ctypes.POINTER(ctypes.c_double)),
                ("eta", ctypes.POINTER(ctypes.c_double)), ("cu", ctypes.POINTER(ctypes.c_double)),
                ("nopen", ctypes.POINTER(ctypes.c_int)), ("status", ctypes.POINTER(ctypes.c_int))]


class HprmatError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"hprmat_b200 status {status}: {message}")
        self.status = status


_lib = None


def load():
    """Load the CUDA library (once).  Raises if it is absent or unloadable."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing; build it with `python -m hprmat_b200.build`")
    lib = ctypes.CDLL(LIB_PATH)
    P, I, D = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
    IP, DP = ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double)
    SP = ctypes.POINTER(Stats)
    sig = {
        "hprmat_b200_default_opts": (None, [ctypes.POINTER(Opts)]),
        "hprmat_b200_create": (I, [I, ctypes.POINTER(Opts), ctypes.POINTER(P)]),
        "hprmat_b200_destroy": (I, [P]),
        "hprmat_b200_set_opts": (I, [P, ctypes.POINTER(Opts)]),
        "hprmat_b200_set_stream": (I, [P, P]),
        "hprmat_b200_rmat_ini": (I, [P, I, I, D, DP]),
        "hprmat_b200_rmatrix": (I, [P, I, IP, DP, DP, D, I, I, DP, I, I, DP, IP, SP]),
        "hprmat_b200_rmatrix_device": (I, [P, I, IP, DP, DP, D, I, I, P, I, I, P, IP, SP]),
        "hprmat_b200_rmatrix_scan": (I, [P, I, ctypes.POINTER(ScanBlock), D, I, I, DP]),
        "hprmat_b200_scan_autotune": (I, [P, I, ctypes.POINTER(ScanBlock), D, I, I, DP]),
        "hprmat_b200_rmatrix_scan_shifted": (I, [P, I, ctypes.POINTER(ScanBlock), D, I, DP]),
        "hprmat_b200_scan_tune_get": (I, [P, IP, DP, I]),
        "hprmat_b200_scan_tune_set": (I, [P, IP, I]),
        "hprmat_b200_rmatrix_adjoint": (I, [P, I, IP, DP, DP, D, I, I, DP, I, I, DP, DP, IP, DP, SP]),
        "hprmat_b200_rmatrix_wf": (I, [P, I, IP, DP, DP, D, I, I, DP, I, I, DP, IP, I, IP, DP, I, I, SP]),
        "hprmat_b200_rmatrix_wf_device": (I, [P, I, IP, DP, DP, D, I, I, P, I, I, P, IP, I, IP, P, I, I, SP]),
        "hprmat_b200_wf_print": (I, [I, IP, DP, DP, D, I, I, DP, I, I, DP, I, I, DP, I, I, I, D, DP]),
        "hprmat_b200_rmatrix_x": (I, [P, I, IP, DP, DP, D, I, DP, I, I, DP, IP, P, ctypes.c_long, SP]),
        "hprmat_b200_adjoint_from_x": (I, [P, I, IP, DP, DP, D, I, DP, I, I, DP, P, ctypes.c_long, DP, DP]),
        "hprmat_b200_rmatrix_x_device": (I, [P, I, IP, DP, DP, D, I, P, I, I, P, IP, P, ctypes.c_long, SP]),
        "hprmat_b200_adjoint_from_x_device": (I, [P, I, IP, DP, DP, D, I, P, I, I, DP, P, ctypes.c_long, DP, P]),
        "hprmat_b200_rmatrix_full": (I, [P, I, IP, DP, DP, D, I, I, DP, I, I, DP, IP, I, DP, I, I, I, IP, I, DP,
                                         SP]),
        "hprmat_b200_solve_linear": (I, [P, DP, DP, I, I, SP]),
        "hprmat_b200_solve_linear_device": (I, [P, P, P, I, I, SP]),
        "hprmat_b200_solve_rmatrix": (I, [P, DP, DP, I, I, D, DP, SP]),
        "gpu_b200_solve_mixed_": (I, [DP, DP, IP, IP, IP, DP, IP]),
        "gpu_b200_solve_double_": (I, [DP, DP, IP, IP, IP]),
        "gpu_b200_finalize_": (I, []),
        "hprmat_b200_status_string": (ctypes.c_char_p, [I]),
        "hprmat_b200_last_error": (ctypes.c_char_p, []),
        "hprmat_b200_version": (I, []),
        "hprmat_b200_boundary": (I, [I, IP, DP, DP, D, DP, DP, DP, DP, IP]),
        "hprmat_b200_solve_linear_noalloc": (I, [P, P, I, I, P, IP]),
        "hprmat_b200_dev_tc_update": (I, [P, P, P, ctypes.c_long, I, P, ctypes.c_long, I, I, I]),
        "hprmat_b200_dev_split_planes": (I, [P, P, I, I, P, ctypes.c_long]),
        "hprmat_b200_dev_set_profile": (I, [P, I]),
        "hprmat_b200_dev_counters": (I, [P, ctypes.POINTER(ctypes.c_ulonglong), DP, DP, IP, I]),
        "hprmat_b200_dev_wave_trace": (I, [P, I]),
        "hprmat_b200_dev_wave_trace_read": (I, [P, ctypes.POINTER(ctypes.c_longlong), I, IP]),
        "hprmat_b200_dev_panel_trace_read": (I, [P, ctypes.POINTER(ctypes.c_longlong), I, IP]),
        "hprmat_b200_dev_set_tuning": (I, [P, ctypes.c_char_p, I]),
        "hprmat_b200_dev_mesh": (I, [I, I, D, DP, DP, DP, DP, DP]),
        "hprmat_b200_dev_factorizations": (ctypes.c_longlong, [P, I]),
        "hprmat_b200_dev_wait_probe": (I, [P, I]),
        "hprmat_b200_dev_binary_version": (I, []),
        "hprmat_b200_dev_zgemm": (I, [P, P, ctypes.c_long, P, ctypes.c_long, P, ctypes.c_long, I, I, I]),
        "hprmat_b200_dev_hessenberg": (I, [P, P, ctypes.c_long, I, P]),
        "hprmat_b200_dev_hess_timings": (I, [P, DP, IP, I]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    got = lib.hprmat_b200_version()
    if got != ABI_VERSION:
        raise ImportError(f"{LIB_PATH} has ABI version {got}, these bindings expect {ABI_VERSION}; rebuild it with "
                          "`python -m hprmat_b200.build`")
    _lib = lib
    return lib


def check(status: int, allow=(OK,)):
    if status in allow:
        return status
    lib = load()
    msg = lib.hprmat_b200_last_error().decode(errors="replace")
    raise HprmatError(status, f"{lib.hprmat_b200_status_string(status).decode()}: {msg}")
