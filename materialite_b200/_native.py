"""ctypes binding of libssfft (the C ABI declared in include/ssfft.h).

The library is built in-tree by ``materialite_b200/csrc/build.py``.  There is no CPU
fallback: if the shared library is missing or no CUDA device is present, every solver
entry point raises.
"""

import ctypes
import os

import numpy as np

_LIB_NAME = "libssfft.so"
_lib = None

SSFFT_FP64 = 0
SSFFT_MIXED = 1

HARDENING_IDS = {
    "perfect_plasticity": 0,
    "linear": 1,
    "voce": 2,
    "armstrong_frederick": 3,
}

FIELD_IDS = {
    "stress": 0,
    "strain": 1,
    "slip_resistances": 2,
    "plastic_strains": 3,
    "slip_system_shear_strains": 4,
    "residual": 5,
    "yield_stresses": 6,
    "eq_plastic_strains": 7,
}

EXPORTED_SYMBOLS = [
    "ssfft_last_error", "ssfft_create", "ssfft_destroy", "ssfft_estimate_bytes",
    "ssfft_set_phase_elastic", "ssfft_set_phase_evp", "ssfft_set_phase_j2",
    "ssfft_set_microstructure", "ssfft_voronoi",
    "ssfft_reset", "ssfft_step", "ssfft_commit", "ssfft_scale_fluctuation",
    "ssfft_get_field", "ssfft_num_slip", "ssfft_apply_projection",
    "ssfft_apply_projection_device", "ssfft_stats", "ssfft_timer", "ssfft_profile_krylov",
    "ssfft_apply_projection_noalloc", "ssfft_solve_constant_rates", "ssfft_set_options",
    "ssfft_server_create", "ssfft_server_submit", "ssfft_server_poll", "ssfft_server_pending",
    "ssfft_server_clock", "ssfft_server_destroy", "ssfft_server_launches",
]


class SsfftConfig(ctypes.Structure):
    _fields_ = [
        ("n", ctypes.c_int32 * 3),
        ("precision", ctypes.c_int32),
        ("device", ctypes.c_int32),
        ("max_newton_iterations", ctypes.c_int32),
        ("max_krylov_iterations", ctypes.c_int64),
        ("global_tolerance", ctypes.c_double),
        ("strain_correction_tolerance", ctypes.c_double),
        ("linear_solver_tolerance", ctypes.c_double),
        ("stress_mask", ctypes.c_double * 6),
        ("krylov_floor", ctypes.c_double),
        ("krylov_forcing", ctypes.c_double),
    ]


class SsfftStepIn(ctypes.Structure):
    _fields_ = [
        ("strain_increment", ctypes.c_double * 6),
        ("stress_increment", ctypes.c_double * 6),
        ("mean_applied_stress", ctypes.c_double * 6),
        ("dt", ctypes.c_double),
        ("summed_von_mises_stress", ctypes.c_double),
        ("time_step_id", ctypes.c_int32),
        ("reset_fluctuation", ctypes.c_int32),
    ]


class SsfftRateSchedule(ctypes.Structure):
    _fields_ = [
        ("strain_rate", ctypes.c_double * 6),
        ("stress_rate", ctypes.c_double * 6),
        ("start_time", ctypes.c_double),
        ("end_time", ctypes.c_double),
        ("initial_time_increment", ctypes.c_double),
        ("max_time_increment", ctypes.c_double),
        ("min_time_increment", ctypes.c_double),
    ]


class SsfftSolveOut(ctypes.Structure):
    _fields_ = [
        ("status", ctypes.c_int32),
        ("steps", ctypes.c_int32),
        ("cutbacks", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
        ("newton_iterations", ctypes.c_int64),
        ("krylov_iterations", ctypes.c_int64),
        ("device_seconds", ctypes.c_double),
        ("mean_stress", ctypes.c_double * 6),
        ("mean_strain", ctypes.c_double * 6),
        ("kernel_launches", ctypes.c_int64),
    ]


class SsfftStepOut(ctypes.Structure):
    _fields_ = [
        ("converged", ctypes.c_int32),
        ("constitutive_failed", ctypes.c_int32),
        ("newton_iterations", ctypes.c_int32),
        ("max_constitutive_iterations", ctypes.c_int32),
        ("krylov_iterations", ctypes.c_int64),
        ("linear_solves", ctypes.c_int32),
        ("status", ctypes.c_int32),
        ("equilibrium_error", ctypes.c_double),
        ("scaled_strain_error", ctypes.c_double),
        ("mean_von_mises_stress", ctypes.c_double),
        ("mean_stress", ctypes.c_double * 6),
        ("mean_strain", ctypes.c_double * 6),
    ]


def library_path():
    return os.path.join(os.path.dirname(os.path.abspath(__file__)), _LIB_NAME)


def load_library():
    """Load (once) and return the ctypes handle of libssfft; raises if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    path = library_path()
    if not os.path.isfile(path):
        raise RuntimeError(
            f"{path} is missing: build it with `python -m materialite_b200.csrc.build` "
            "(there is no CPU fallback for the SmallStrainFFT solve)")
    lib = ctypes.CDLL(path)
    P = ctypes.c_void_p
    dp = ctypes.POINTER(ctypes.c_double)
    ip = ctypes.POINTER(ctypes.c_int32)
    lib.ssfft_last_error.restype = ctypes.c_char_p
    lib.ssfft_last_error.argtypes = []
    lib.ssfft_create.argtypes = [ctypes.POINTER(SsfftConfig), ctypes.POINTER(P)]
    lib.ssfft_destroy.argtypes = [P]
    lib.ssfft_estimate_bytes.argtypes = [ctypes.POINTER(SsfftConfig), ctypes.c_int, ctypes.c_int,
                                         ctypes.POINTER(ctypes.c_size_t)]
    lib.ssfft_set_phase_elastic.argtypes = [P, ctypes.c_int, dp]
    lib.ssfft_set_phase_evp.argtypes = [P, ctypes.c_int, dp, ctypes.c_int, dp, ctypes.c_double,
                                        ctypes.c_double, ctypes.c_double, ctypes.c_int, dp,
                                        ctypes.c_int, ctypes.c_double]
    lib.ssfft_set_phase_j2.argtypes = [P, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                       ctypes.c_double, ctypes.c_int, dp, ctypes.c_int]
    lib.ssfft_set_microstructure.argtypes = [P, ctypes.c_int, dp, ip, ip]
    lib.ssfft_voronoi.argtypes = [ip, dp, dp, dp, dp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                  ip]
    lib.ssfft_reset.argtypes = [P]
    lib.ssfft_step.argtypes = [P, ctypes.POINTER(SsfftStepIn), ctypes.POINTER(SsfftStepOut)]
    lib.ssfft_commit.argtypes = [P, ctypes.c_double]
    lib.ssfft_scale_fluctuation.argtypes = [P, ctypes.c_double]
    lib.ssfft_get_field.argtypes = [P, ctypes.c_int, dp, ctypes.c_int]
    lib.ssfft_num_slip.argtypes = [P]
    lib.ssfft_apply_projection.argtypes = [P, dp, dp]
    lib.ssfft_apply_projection_device.argtypes = [P, P, P]
    lib.ssfft_stats.argtypes = [P, dp, ctypes.POINTER(ctypes.c_int64)]
    lib.ssfft_timer.argtypes = [P, ctypes.c_int, dp]
    lib.ssfft_profile_krylov.argtypes = [P, ctypes.c_int, dp]
    lib.ssfft_apply_projection_noalloc.argtypes = [ip, dp, P, P, P]
    lib.ssfft_solve_constant_rates.argtypes = [P, ctypes.POINTER(SsfftRateSchedule),
                                               ctypes.POINTER(SsfftSolveOut)]
    lib.ssfft_set_options.argtypes = [P, ctypes.POINTER(SsfftConfig)]
    for name in EXPORTED_SYMBOLS:
        if name not in ("ssfft_last_error", "ssfft_server_clock") and not name.startswith("ssfft_server"):
            getattr(lib, name).restype = ctypes.c_int
    _lib = lib
    return lib


class SsfftError(RuntimeError):
    def __init__(self, code, message):
        super().__init__(f"libssfft error {code}: {message}")
        self.code = code


def check(rc):
    if rc != 0:
        msg = load_library().ssfft_last_error().decode(errors="replace")
        raise SsfftError(rc, msg)


def as_double_ptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def as_int_ptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))


def c_doubles(values, n):
    arr = (ctypes.c_double * n)()
    vals = np.asarray(values, dtype=np.float64).ravel()
    for i in range(min(n, vals.size)):
        arr[i] = float(vals[i])
    return arr
