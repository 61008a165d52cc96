"""ctypes binding of the C ABI in include/tpm.h (libtigerpm_b200.so).

The shared library is built in-tree by tigerpm_b200/build.py.  Loading fails
loudly when it is missing: there is no Python or CPU fallback for any entry
point.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libtigerpm_b200.so")

TPM_OK = 0
TPM_ERR_INVALID = -1
TPM_ERR_NOMEM = -2
TPM_ERR_CUDA = -3
TPM_ERR_CUFFT = -4
TPM_ERR_STATE = -5
TPM_ERR_RUNG = -6
TPM_ERR_CAPACITY = -7
TPM_ERR_BUDGET = -8
TPM_ERR_TIMEOUT = -9
TPM_ERR_NOEXT = -10
TPM_EWALD_NOALLOC_MAX_SINKS = 4096

GRAVITY_LONG_PM = 0
GRAVITY_LONG_PME = 1
ASSIGN = {"cloud4": 0, "cic": 1, "tsc": 2}
SORT = {"parity": 0, "fast": 1}
FFT = {"auto": 0, "cufft": 1, "block": 2}


class Options(C.Structure):
    """struct tpm_options: the reference's struct options (tigerpm/options.hpp:6-27)
    followed by this library's extensions."""
    _fields_ = [
        ("four_dim", C.c_int), ("chain_dim", C.c_int), ("parts_dim", C.c_int),
        ("parts_o_four", C.c_int), ("parts_o_chain", C.c_int), ("four_o_chain", C.c_int),
        ("eta", C.c_double), ("sigma8", C.c_double), ("code_to_cm", C.c_double),
        ("hubble", C.c_double), ("GM", C.c_double), ("hsoft", C.c_double),
        ("box_size", C.c_double), ("rs", C.c_double), ("omega_m", C.c_double),
        ("z0", C.c_double),
        ("rcut_over_rs", C.c_double), ("assign", C.c_int), ("deconv_order", C.c_int),
        ("sort_mode", C.c_int), ("kahan", C.c_int), ("deterministic_deposit", C.c_int),
        ("fft", C.c_int), ("seed", C.c_uint64), ("fft_group", C.c_int), ("kick_grid", C.c_int),
    ]


class StageTimes(C.Structure):
    _fields_ = [(n, C.c_float) for n in ("sort_ms", "deposit_ms", "fft_forward_ms", "green_ms",
                                         "fft_inverse_ms", "kick_ms", "drift_ms", "ewald_ms",
                                         "interp_ms")]


class HostParticles(C.Structure):
    """struct tpm_host_particles: host array addresses of one particle set."""
    _fields_ = [(n, C.c_void_p) for n in ("x", "y", "z", "vx", "vy", "vz", "rung")]


class KickShape(C.Structure):
    """struct tpm_kick_shape."""
    _fields_ = [("warps", C.c_int), ("stage", C.c_int), ("npass", C.c_int), ("tuned", C.c_int), ("ms", C.c_float)]


class BatchTimes(C.Structure):
    """struct tpm_batch_times."""
    _fields_ = [(n, C.c_float) for n in ("long_range_ms", "queue_ms", "interp_ms", "kick_ms")]


class ServeResult(C.Structure):
    """struct tpm_serve_result."""
    _fields_ = [("status", C.c_int), ("box", C.c_int), ("latency_ms", C.c_double), ("queue_ms", C.c_double),
                ("device_ms", C.c_float), ("particles", C.c_int64)]


class ServeStats(C.Structure):
    """struct tpm_serve_stats_t."""
    _fields_ = [("budget_bytes", C.c_int64), ("resident_bytes", C.c_int64), ("inflight_peak_bytes", C.c_int64),
                ("max_working_set_bytes", C.c_int64), ("boxes", C.c_int), ("max_concurrent_steps", C.c_int),
                ("steps_done", C.c_int64), ("particles_done", C.c_int64), ("launches", C.c_int64)]


class Substep(C.Structure):
    """struct tpm_substep."""
    _fields_ = [("tick", C.c_int64), ("ticks_per_step", C.c_int64), ("max_rung", C.c_int), ("min_rung", C.c_int),
                ("drift_dt", C.c_double), ("done", C.c_int)]


class Diag(C.Structure):
    """struct tpm_diag."""
    _fields_ = [("kinetic", C.c_double), ("potential", C.c_double), ("momentum", C.c_double * 3),
                ("n", C.c_int64)]


class ICParams(C.Structure):
    """struct tpm_ic_params."""
    _fields_ = [("n_side", C.c_int), ("seed", C.c_uint64), ("npower", C.c_int), ("power_k", C.c_void_p),
                ("power_p", C.c_void_p), ("index", C.c_double), ("kcut_over_nyq", C.c_double),
                ("rms_disp", C.c_double)]


BATCH_RESTORE = 1
BATCH_GRAPH = 2


class DeviceArrays(C.Structure):
    _fields_ = [("x", C.c_void_p), ("y", C.c_void_p), ("z", C.c_void_p), ("vx", C.c_void_p),
                ("vy", C.c_void_p), ("vz", C.c_void_p), ("rung", C.c_void_p), ("gx", C.c_void_p),
                ("gy", C.c_void_p), ("gz", C.c_void_p), ("pot", C.c_void_p),
                ("cell_begin", C.c_void_p), ("phi", C.c_void_p), ("n", C.c_int64)]


# (name, restype, argtypes) of every exported function in include/tpm.h
_P = C.c_void_p
_I = C.c_int
_I64 = C.c_int64
_D = C.c_double
SIGNATURES = [
    ("tpm_error_string", C.c_char_p, [_I]),
    ("tpm_last_error_message", C.c_char_p, []),
    ("tpm_options_init", _I, [C.POINTER(Options), _I, _I, _I]),
    ("tpm_options_parse", _I, [C.POINTER(Options), _I, C.POINTER(C.c_char_p)]),
    ("tpm_ctx_create", _I, [C.POINTER(Options), _I64, C.POINTER(_P)]),
    ("tpm_ctx_destroy", _I, [_P]),
    ("tpm_ctx_options", _I, [_P, C.POINTER(Options)]),
    ("tpm_ctx_device_bytes", _I, [_P, C.POINTER(_I64)]),
    ("tpm_plan_device_bytes", _I, [C.POINTER(Options), _I64, C.POINTER(_I64)]),
    ("tpm_set_particles", _I, [_P, _I64, _P, _P, _P, _P, _P, _P, _P]),
    ("tpm_set_particles_device", _I, [_P, _I64, _P, _P, _P, _P, _P, _P, _P]),
    ("tpm_get_particles", _I, [_P, _P, _P, _P, _P, _P, _P, _P]),
    ("tpm_get_forces", _I, [_P, _P, _P, _P, _P]),
    ("tpm_get_device_arrays", _I, [_P, C.POINTER(DeviceArrays)]),
    ("tpm_num_particles", _I, [_P, C.POINTER(_I64)]),
    ("tpm_chainmesh_create", _I, [_P]),
    ("tpm_chainmesh_get", _I, [_P, _P, _P, _P]),
    ("tpm_chainmesh_offsets", _I, [_P, _P]),
    ("tpm_chainmesh_interior_box", _I, [_P, _P]),
    ("tpm_gravity_long_compute", _I, [_P, _I]),
    ("tpm_gravity_long_get_phi", _I, [_P, _P, _P]),
    ("tpm_gravity_long_set_phi", _I, [_P, _P]),
    ("tpm_gravity_long_get_phi_box", _I, [_P, _P]),
    ("tpm_gravity_long_force_at", _I, [_P, _I64, _P, _P, _P]),
    ("tpm_kick_pme", _I, [_P, _P, _I, _D, _D, _I]),
    ("tpm_drift", _I, [_P, _D]),
    ("tpm_gravity_short_ewald", _I, [_P, _I64, _P, _P, _P, _I, _P, _P, _P, _P]),
    ("tpm_ewald_fp64", _I, [_P, _I64, _P, _I, _P, _P, _P, _P]),
    ("tpm_ewald_fp64_noalloc", _I, [_P, _P, _P, _I64, _P, _P, _P, _I64, _D, _P, _P, _P, _P, _P]),
    ("tpm_get_stage_times", _I, [_P, C.POINTER(StageTimes)]),
    ("tpm_reset_stage_times", _I, [_P]),
    ("tpm_get_launch_count", _I, [_P, C.POINTER(_I64)]),
    ("tpm_synchronize", _I, [_P]),
    ("tpm_ctx_stream", _I, [_P, C.POINTER(_P)]),
    ("tpm_pme_step", _I, [_P, _I, _D, _D, _I]),
    ("tpm_pme_steps_host", _I, [_P, _I64, _I64, _P, _P, _I, _D, _D, _I]),
    ("tpm_check_errors", _I, [_P]),
    ("tpm_batch_create", _I, [_I, C.POINTER(Options), C.POINTER(_I64), C.POINTER(_P)]),
    ("tpm_batch_destroy", _I, [_P]),
    ("tpm_batch_size", _I, [_P, C.POINTER(_I), C.POINTER(_I64)]),
    ("tpm_batch_box", _I, [_P, _I, C.POINTER(_P)]),
    ("tpm_batch_set_input", _I, [_P, _I, _I64, _P, _P, _P, _P, _P, _P, _P]),
    ("tpm_batch_step", _I, [_P, _I, _I, _D, _D, _I]),
    ("tpm_batch_steps_sequential", _I, [_P, _I, _I, _D, _D, _I]),
    ("tpm_batch_synchronize", _I, [_P]),
    ("tpm_batch_stream", _I, [_P, C.POINTER(_P)]),
    ("tpm_batch_launch_count", _I, [_P, C.POINTER(_I64)]),
    ("tpm_batch_phase_times", _I, [_P, C.POINTER(BatchTimes)]),
    ("tpm_batch_get_shape", _I, [_P, C.POINTER(KickShape)]),
    ("tpm_batch_set_shape", _I, [_P, C.POINTER(KickShape)]),
    ("tpm_batch_autotune", _I, [_P, _I, _I, C.POINTER(KickShape)]),
    ("tpm_integrate_begin", _I, [_P, _D, _D, _I]),
    ("tpm_integrate_substep", _I, [_P, C.POINTER(Substep)]),
    ("tpm_integrate", _I, [_P, _D, _D, _I, _I, _P, _I, C.POINTER(_I)]),
    ("tpm_diagnostics", _I, [_P, C.POINTER(Diag)]),
    ("tpm_ic_zeldovich", _I, [_P, C.POINTER(ICParams), C.POINTER(_D)]),
    ("tpm_ic_power", _I, [_P, _P, _I, _D, _D, _I, _P, _P]),
    ("tpm_growth_factor", _I, [_D, _D, C.POINTER(_D)]),
    ("tpm_serve_create", _I, [_I64, _I, C.POINTER(_P)]),
    ("tpm_serve_destroy", _I, [_P]),
    ("tpm_serve_add_box", _I, [_P, C.POINTER(Options), _I64, _P, _P, _P, _P, _P, _P, _P, C.POINTER(_I)]),
    ("tpm_serve_add_box_ic", _I, [_P, C.POINTER(Options), C.POINTER(ICParams), C.POINTER(_I)]),
    ("tpm_serve_submit", _I, [_P, _I, _D, _I, _D, _D, _I, C.POINTER(_I)]),
    ("tpm_serve_wait", _I, [_P, _I, C.POINTER(ServeResult)]),
    ("tpm_serve_drain", _I, [_P]),
    ("tpm_serve_replay", _I, [_P, _I, _P, _P, _D, _I, _D, _D, _I, _P]),
    ("tpm_serve_box", _I, [_P, _I, C.POINTER(_P)]),
    ("tpm_serve_stats", _I, [_P, C.POINTER(ServeStats)]),
    ("tpm_count_pairs", _I, [_P, _I, C.POINTER(_I64), C.POINTER(_I64)]),
    ("tpm_fp32_peak_probe", _I, [C.POINTER(_D)]),
]

_LIB = None


class TPMError(RuntimeError):
    def __init__(self, status: int, where: str, msg: str):
        super().__init__(f"{where}: {msg} (status {status})")
        self.status = status


def load():
    """Load libtigerpm_b200.so; raises if it has not been built."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: run tigerpm_b200/build.py (nvcc, sm_100a)")
    lib = C.CDLL(LIB_PATH)
    for name, res, args in SIGNATURES:
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _LIB = lib
    return lib


def check(status: int, where: str) -> int:
    if status != TPM_OK:
        lib = load()
        msg = lib.tpm_last_error_message().decode()
        raise TPMError(status, where, msg)
    return status
