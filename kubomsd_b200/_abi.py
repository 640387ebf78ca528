"""ctypes binding of libkmsd_b200.so (declared in include/kmsd.h).

The library is loaded from the package's `_lib/` directory; a missing library
is an error (there is no CPU fallback): `require_library()` raises
BackendUnavailable with the build command.
"""
from __future__ import annotations

import ctypes as C
import os
import re
from pathlib import Path

from .errors import BackendUnavailable

LIB_PATH = Path(os.environ.get("KUBOMSD_B200_LIB", Path(__file__).resolve().parent / "_lib" / "libkmsd_b200.so"))
HEADER = Path(__file__).resolve().parent.parent / "include" / "kmsd.h"

KMSD_OK, KMSD_EINVAL, KMSD_ERUNTIME, KMSD_EMETRIC, KMSD_ECUDA = 0, 1, 2, 3, 4
KMSD_FP64, KMSD_MIXED = 0, 1
KMSD_MOMENTS_DIRECT, KMSD_MOMENTS_DOUBLING = 0, 1
KMSD_FORM_ELL, KMSD_FORM_BSR4 = 1, 2


class SolveReport(C.Structure):
    _fields_ = [("converged", C.POINTER(C.c_uint8)), ("breakdown", C.POINTER(C.c_uint8)),
                ("iterations", C.POINTER(C.c_int64)), ("true_residual", C.POINTER(C.c_double)),
                ("relative_residual", C.POINTER(C.c_double))]


class MetricStats(C.Structure):
    _fields_ = [("calls", C.c_int64), ("max_iterations_sum", C.c_int64), ("seconds", C.c_double),
                ("max_relative_residual", C.c_double), ("true_residual_refreshes", C.c_int64),
                ("true_residual_checks", C.c_int64), ("residual_restarts", C.c_int64),
                ("refinement_steps", C.c_int64)]


P = C.c_void_p
I64 = C.c_int64
D = C.c_double
PD = C.POINTER(C.c_double)
PI64 = C.POINTER(C.c_int64)

SIGNATURES = {
    "kmsd_last_error": (C.c_char_p, []),
    "kmsd_build_info": (C.c_char_p, []),
    "kmsd_device": (C.c_int, [C.POINTER(C.c_int)]),
    "kmsd_kernel_launches": (I64, []),
    "kmsd_csr_create": (C.c_int, [I64, PI64, PI64, PD, PD, C.POINTER(P)]),
    "kmsd_csr_destroy": (None, [P]),
    "kmsd_csr_rows": (I64, [P]),
    "kmsd_csr_nnz": (I64, [P]),
    "kmsd_csr_forms": (C.c_int, [P]),
    "kmsd_csr_matmul": (C.c_int, [P, P, P, I64, P]),
    "kmsd_metric_create": (C.c_int, [P, PD, I64, PI64, PI64, PD, PD, C.POINTER(P)]),
    "kmsd_metric_destroy": (None, [P]),
    "kmsd_metric_set_residual_policy": (C.c_int, [P, C.c_int, C.c_int, D]),
    "kmsd_metric_set_segments": (C.c_int, [P, I64, PI64]),
    "kmsd_metric_set_storage": (C.c_int, [P, C.c_int]),
    "kmsd_metric_solve": (C.c_int, [P, P, P, I64, D, D, C.c_int, C.POINTER(SolveReport), P]),
    "kmsd_metric_sample": (C.c_int, [P, P, P, I64, PD, I64, D, D, P]),
    "kmsd_metric_stats_get": (C.c_int, [P, C.POINTER(MetricStats)]),
    "kmsd_metric_is_identity": (C.c_int, [P]),
    "kmsd_engine_create": (C.c_int, [P, P, C.POINTER(C.c_int), C.POINTER(P), D, D, C.c_int, D, C.c_int,
                                     C.POINTER(P)]),
    "kmsd_engine_destroy": (None, [P]),
    "kmsd_engine_h_action": (C.c_int, [P, P, P, I64, P]),
    "kmsd_engine_v_cov": (C.c_int, [P, PD, P, P, I64, D, D, C.c_int, P]),
    "kmsd_engine_series": (C.c_int, [P, P, P, I64, PD, I64, D, D, PD, I64, P]),
    "kmsd_engine_chain": (C.c_int, [P, P, P, I64, I64, D, D, P]),
    "kmsd_engine_chain_correlate": (C.c_int, [P, P, P, I64, I64, I64, D, D, P, P]),
    "kmsd_engine_lanczos": (C.c_int, [P, P, I64, PD, PD, P]),
    "kmsd_vac_nodes": (C.c_int, [P, I64, I64, I64, I64, P, P, I64, P, I64, P, I64, P, P]),
    "kmsd_random_phases": (C.c_int, [I64, I64, P, P, P]),
    "kmsd_project_moments": (C.c_int, [P, I64, I64, P, I64, P, P]),
    "kmsd_bootstrap_ratio": (C.c_int, [P, P, I64, I64, I64, P, I64, P, P, P]),
    "kmsd_engine_moments": (C.c_int, [P, P, PD, I64, I64, D, D, C.c_int, P]),
    "kmsd_engine_moments_noalloc": (C.c_int, [P, P, PD, I64, I64, D, D, C.c_int, P]),
    "kmsd_engine_counters": (C.c_int, [P, PI64, PI64]),
    "kmsd_engine_failure_report": (C.c_int, [P, C.POINTER(SolveReport), I64, PI64]),
    "kmsd_engine_inner": (C.c_int, [P, P, P, P, I64, P]),
    "kmsd_column_dot": (C.c_int, [P, P, I64, I64, P, P]),
    "kmsd_batch_create": (C.c_int, [I64, C.POINTER(P), C.c_int, I64, C.POINTER(P)]),
    "kmsd_batch_attach_metric": (C.c_int, [P, P, P, D, D, C.c_int]),
    "kmsd_batch_destroy": (None, [P]),
    "kmsd_batch_rows": (C.c_int, [P, PI64]),
    "kmsd_batch_moments": (C.c_int, [P, P, PD, I64, I64, PD, PD, C.c_int, C.c_int, P]),
    "kmsd_batch_set_tile_rows": (C.c_int, [P, I64]),
    "kmsd_batch_tune": (C.c_int, [P, P, PD, I64, I64, PD, PD, C.c_int, PI64, P]),
}


def header_functions(path: Path = HEADER) -> list[str]:
    """Names of every function declared in include/kmsd.h."""
    text = path.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(kmsd_[a-z0-9_]+)\s*\(", text)))


_lib = None


def load(path: Path = LIB_PATH):
    """Load the shared library and attach the prototypes (no GPU needed)."""
    global _lib
    if _lib is not None and path == LIB_PATH:
        return _lib
    if not path.exists():
        raise BackendUnavailable(
            "B200 stochastic backend requires building its CUDA library: python -m kubomsd_b200.build "
            "(requires nvcc for sm_100a)")
    lib = C.CDLL(str(path))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path == LIB_PATH:
        _lib = lib
    return lib


def require_library():
    return load()


def last_error(lib) -> str:
    msg = lib.kmsd_last_error()
    return msg.decode() if msg else ""
