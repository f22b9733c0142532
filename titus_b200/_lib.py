"""ctypes binding of libtitus.so (the C ABI declared in include/titus.h).

The shared library is built in-tree (``titus_b200/libtitus.so``) by
``titus_b200.build``. Loading fails loudly if it is missing: the package has
no CPU fallback for the energy loop.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libtitus.so")

TITUS_OK, TITUS_ERR_ARG, TITUS_ERR_CUDA, TITUS_ERR_DEVICE, TITUS_ERR_LIMIT = 0, 1, 2, 3, 4
TITUS_DLR_FIXED = 0
TITUS_PARALLEL_ADAPTIVE = 1
TITUS_BUG_ADAPTIVE = 2
TITUS_DLR_HIGH_ORDER = 3
TITUS_PN_FULL = 4
TITUS_PARALLEL_REJECTION = 5
TITUS_PRECISION_FP64 = 0
TITUS_PRECISION_MIXED = 1
# exclusive device timers (titus_profile order); "other" is time outside every named phase
PROFILE_NAMES = ["barrier", "reduce", "jacobi", "cholesky", "completion", "rows_stream", "rows_scatter", "rf_passes",
                 "small", "other", "prologue"]
# event counters titus_profile appends after the timers
PROFILE_COUNTERS = ["svd_sweeps", "svd_calls", "eig_calls", "eig_sweeps", "chol_calls", "rf_slow", "rf_fast",
                    "barriers"]

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)


class Problem(C.Structure):
    _fields_ = [
        ("nx", C.c_int32), ("ny", C.c_int32), ("npn", C.c_int32), ("n_moments", C.c_int32),
        ("n_ordinates", C.c_int32), ("n_energies", C.c_int32), ("r", C.c_int32),
        ("dx", C.c_double), ("dy", C.c_double), ("theta", C.c_double), ("theta_index", C.c_double),
        ("c_eta", C.c_double),
        ("density", _dp), ("e_trafo", _dp), ("stopping", _dp), ("bc_energy", _dp), ("sigma", _dp),
        ("bc_space", _dp), ("bc_angle", _dp), ("omega", _dp), ("m_reduced", _dp),
        ("op_rowptr", _ip * 4), ("op_col", _ip * 4), ("op_val", _dp * 4),
        ("x_completion", _ip), ("n_x_completion", C.c_int32),
        ("w_completion", _ip), ("n_w_completion", C.c_int32),
        ("sweep_restore", _ip), ("n_sweep_restore", C.c_int32),
        ("stopping_mid", _dp),
    ]


class Problem3D(C.Structure):
    _fields_ = [("nz", C.c_int32), ("dz", C.c_double), ("op_rowptr", _ip * 2), ("op_col", _ip * 2),
                ("op_val", _dp * 2)]


class Options(C.Structure):
    _fields_ = [("team_ctas", C.c_int32), ("max_steps", C.c_int32), ("rank_tol", C.c_double),
                ("profile", C.c_int32), ("precision", C.c_int32)]


class Result(C.Structure):
    _fields_ = [
        ("dose", _dp), ("X", _dp), ("S", _dp), ("W", _dp), ("psi", _dp),
        ("r_cap", C.c_int32), ("rank", C.c_int32), ("steps_done", C.c_int32),
        ("rank_history", _ip), ("eta_history", _dp), ("bound_history", _dp), ("time_history", _dp),
    ]


class Spot(C.Structure):
    _fields_ = [("n_energies", C.c_int32), ("d_e", C.c_double), ("stopping", _dp), ("bc_energy", _dp),
                ("sigma", _dp), ("bc_space", _dp)]


# (name, restype, argtypes) for every symbol include/titus.h declares
SIGNATURES = [
    ("titus_create", C.c_int, [C.POINTER(Problem), C.POINTER(C.c_void_p)]),
    ("titus_create_3d", C.c_int, [C.POINTER(Problem), C.POINTER(Problem3D), C.POINTER(C.c_void_p)]),
    ("titus_solve", C.c_int, [C.c_void_p, C.c_int32, C.POINTER(Options), C.POINTER(Result)]),
    ("titus_solve_device", C.c_int, [C.c_void_p, C.c_int32, C.POINTER(Options), C.c_void_p]),
    ("titus_fetch", C.c_int, [C.c_void_p, C.POINTER(Result)]),
    ("titus_solve_problem", C.c_int, [C.POINTER(Problem), C.c_int32, C.POINTER(Options), C.POINTER(Result)]),
    ("titus_set_state", C.c_int, [C.c_void_p, C.c_int32, _dp, _dp, _dp, _dp, _dp, C.c_int32]),
    ("titus_solve_from", C.c_int, [C.c_void_p, C.c_int32, C.POINTER(Options), C.c_int32, C.POINTER(Result)]),
    ("titus_resume_point", C.c_int, [C.c_void_p, _ip, _dp]),
    ("titus_solve_batched", C.c_int, [C.c_void_p, C.c_int32, C.POINTER(Options), C.c_int32, C.POINTER(Spot), _dp,
                                      _ip, _ip]),
    ("titus_batch_upload", C.c_int, [C.c_void_p, C.c_int32, C.POINTER(Spot), C.POINTER(C.c_void_p)]),
    ("titus_batch_solve_device", C.c_int, [C.c_void_p, C.c_int32, C.POINTER(Options), C.c_void_p]),
    ("titus_batch_fetch", C.c_int, [C.c_void_p, _dp, _ip, _ip]),
    ("titus_batch_rank_sums", C.c_int, [C.c_void_p, _ip]),
    ("titus_batch_destroy", None, [C.c_void_p]),
    ("titus_destroy", None, [C.c_void_p]),
    ("titus_last_error", C.c_int, [C.c_char_p, C.c_size_t]),
    ("titus_profile", C.c_int, [C.c_void_p, _dp, C.c_int32]),
    ("titus_solve_noalloc", C.c_int, [C.POINTER(Problem), C.POINTER(Options), _dp, _dp, _dp, _dp, _dp, _ip,
                                      C.c_void_p, C.c_char_p, C.c_size_t]),
    ("titus_limited_flux", C.c_int, [C.c_int32, C.c_int32, C.c_int32, C.c_double, C.c_double, C.c_void_p,
                                     C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    ("titus_pn_full_solve_device", C.c_int, [C.c_void_p, C.POINTER(Options), C.c_void_p]),
    ("titus_pn_full_fetch", C.c_int, [C.c_void_p, _dp, _dp, _dp]),
    ("titus_pn_full_solve", C.c_int, [C.c_void_p, C.POINTER(Options), _dp, _dp, _dp]),
    ("titus_dose_adjoint", C.c_int, [C.c_void_p, C.c_int32, C.POINTER(Options), _dp, _dp, _dp, C.c_int32, _dp, _dp,
                                     _dp, _dp]),
    ("titus_debug_barrier_fault", C.c_int, [C.c_void_p, C.c_int32, C.c_int64]),
    ("titus_debug_fail_alloc", C.c_int, [C.c_int32]),
    ("titus_debug_tc_gram", C.c_int, [_dp, C.c_int32, C.c_int32, C.c_int32, _dp]),
    ("titus_max_rank", C.c_int, []),
    ("titus_max_ordinates", C.c_int, []),
    ("titus_version", C.c_char_p, []),
]

_lib = None


class TitusError(RuntimeError):
    pass


def load(path: str | None = None):
    """Load libtitus.so once; raise if it is not built."""
    global _lib
    if _lib is not None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise TitusError(f"libtitus.so not found at {p}; run titus_b200.build.build() (nvcc, sm_100a)")
    lib = C.CDLL(p)
    for name, res, args in SIGNATURES:
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def last_error() -> str:
    buf = C.create_string_buffer(1024)
    load().titus_last_error(buf, len(buf))
    return buf.value.decode()


def check(rc: int, what: str):
    if rc != 0:
        raise TitusError(f"{what} failed (status {rc}): {last_error()}")


def as_dp(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_dp)


def as_ip(a: np.ndarray):
    assert a.dtype == np.int32 and a.flags.c_contiguous
    return a.ctypes.data_as(_ip)
