"""ctypes binding of libsimulato_cuda.so (include/simulato_cuda.h).

The library is built in-tree by `simulatokit_b200.build`. Loading fails loudly: there is no CPU fallback anywhere in
this package, so a missing library or a missing sm_100 device raises `CudaUnavailable` at the first call.
"""

from __future__ import annotations

import ctypes as C
import os
import threading

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsimulato_cuda.so")

SIMK_OK, SIMK_ERR_INVALID, SIMK_ERR_CUDA, SIMK_ERR_UNAVAILABLE, SIMK_ERR_MEMORY, SIMK_ERR_TIMEOUT = range(6)
FORM_PLAIN, FORM_FUSED, FORM_BF16X3 = 0, 1, 2
OPT_FORM, OPT_BATCH, OPT_BATCH_BYTES, OPT_GRAPHS, OPT_TIMING, OPT_COL_TILE, OPT_TMA = 0, 1, 2, 3, 4, 5, 6
OPT_GRAPHS_CACHED = 7
OPT_AUTOTUNE, OPT_TUNED_COL_TILE, OPT_TUNED_TMA, OPT_TUNED_BATCH = 8, 9, 10, 11
OPT_TCGEN05, OPT_EPILOGUE_DETECT, OPT_POISSON_STREAM, OPT_COMPOSITE = 12, 13, 14, 15
OPT_TABLE_LAUNCHES, OPT_TABLE_KERNELS, OPT_TABLE_SHAPES, OPT_TUNED_ENGINE = 16, 17, 18, 19
OPT_PAIRED = 20
PI_EXACT, PI_ABTEM_FLOAT32 = 0, 1
DET_ANNULAR, DET_PIXELATED, DET_COM, DET_SEGMENTED, DET_BINNED = 0, 1, 2, 3, 4
MAXANGLE_CUTOFF, MAXANGLE_VALID, MAXANGLE_FULL = 0, 1, 2
UNITS_MRAD, UNITS_INV_ANGSTROM = 0, 1

EXPORTED = [
    "simk_cuda_available", "simk_last_error", "simk_context_create", "simk_context_destroy",
    "simk_context_set_stream", "simk_context_set_option", "simk_context_get_option", "simk_context_synchronize",
    "simk_context_launch_count", "simk_context_kernel_time", "simk_potential_from_atoms", "simk_potential_from_values", "simk_potential_destroy",
    "simk_potential_slice_count", "simk_potential_read_slices", "simk_potential_read_transmission", "simk_run",
    "simk_run_batch", "simk_probe_spectrum", "simk_build_probes", "simk_detector_shape", "simk_scan",
    "simk_scan_device", "simk_fft2", "simk_probe_spectrum_noalloc", "simk_finite_profile",
    "simk_potential_from_atoms_finite", "simk_surrogate_train", "simk_surrogate_destroy", "simk_surrogate_info",
    "simk_surrogate_evaluate", "simk_surrogate_parameters", "simk_surrogate_gradients", "simk_job_table_run",
    "simk_scan_waves", "simk_ctf_kernel", "simk_apply_ctf", "simk_gaussian_source_size",
    "simk_gaussian_source_size_device", "simk_poisson_noise", "simk_poisson_noise_device", "simk_integrate_gradient",
    "simk_integrate_gradient_device", "simk_potential_tile", "simk_potential_project", "simk_potential_grid",
]
SURROGATE_PARAMS = 11249


class SimulatoError(Exception):
    """A refused argument or a failed device call (SimulatoError, Sources/SimulatoCore/SimulatoError.swift:7-57)."""

    def __init__(self, status: int, message: str):
        super().__init__(message)
        self.status = status


class CudaUnavailable(SimulatoError):
    """No library or no sm_100 device: the `.metalUnavailable` analogue."""


class CudaFailure(SimulatoError):
    """A CUDA error: the `.metalFailure(String)` analogue."""


class InvalidArgument(SimulatoError, ValueError):
    """A refused argument."""


class Grid_t(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("extent_x", C.c_double), ("extent_y", C.c_double)]


class Probe_t(C.Structure):
    _fields_ = [("energy", C.c_double), ("semiangle_mrad", C.c_double), ("soft", C.c_int32), ("reserved", C.c_int32),
                ("aberrations", C.c_double * 25), ("tilt_x", C.c_double), ("tilt_y", C.c_double)]


class Detector_t(C.Structure):
    _fields_ = [("kind", C.c_int32), ("max_angle", C.c_int32), ("units", C.c_int32), ("has_outer", C.c_int32),
                ("nr", C.c_int32), ("nphi", C.c_int32), ("inner", C.c_double), ("outer", C.c_double),
                ("rotation", C.c_double)]


class Ctf_t(C.Structure):
    _fields_ = [("aberrations", C.c_double * 25), ("semiangle_mrad", C.c_double), ("soft", C.c_int32),
                ("reserved", C.c_int32), ("focal_spread", C.c_double), ("angular_spread", C.c_double)]


JOB_PLANE_WAVE, JOB_PROBE = 0, 1


class Job_t(C.Structure):
    _fields_ = [("potential", C.c_void_p), ("energy", C.c_double), ("incident", C.c_int32), ("reserved", C.c_int32),
                ("probe", Probe_t), ("x", C.c_double), ("y", C.c_double), ("intensity", C.POINTER(C.c_double))]


_lib = None
_lock = threading.Lock()

P = C.c_void_p
PD = C.POINTER(C.c_double)
PI32 = C.POINTER(C.c_int32)


def _signatures(lib):
    i32, i64, d = C.c_int32, C.c_int64, C.c_double
    sig = {
        "simk_cuda_available": [PI32],
        "simk_context_create": [i32, C.POINTER(P)],
        "simk_context_destroy": [P],
        "simk_context_set_stream": [P, P],
        "simk_context_set_option": [P, i32, i64],
        "simk_context_get_option": [P, i32, C.POINTER(i64)],
        "simk_context_synchronize": [P],
        "simk_context_launch_count": [P, C.POINTER(i64), i32],
        "simk_context_kernel_time": [P, C.c_char_p, PD, C.POINTER(i64), PD, i32],
        "simk_potential_from_atoms": [P, C.POINTER(Grid_t), i32, PD, i32, i32, PI32, PD, PI32, C.POINTER(P)],
        "simk_potential_from_values": [P, C.POINTER(Grid_t), i32, PD, PD, C.POINTER(P)],
        "simk_potential_destroy": [P],
        "simk_potential_slice_count": [P, PI32],
        "simk_potential_read_slices": [P, P, PD],
        "simk_potential_read_transmission": [P, P, d, i32, PD, PD],
        "simk_run": [P, P, d, d, d, PD, PD, i32, PI32, PD, PD],
        "simk_run_batch": [P, P, d, d, d, i32, PD, PD, PD, PD],
        "simk_probe_spectrum": [P, C.POINTER(Grid_t), C.POINTER(Probe_t), PD, PD],
        "simk_build_probes": [P, C.POINTER(Grid_t), C.POINTER(Probe_t), i32, PD, PD, PD],
        "simk_detector_shape": [C.POINTER(Grid_t), d, C.POINTER(Detector_t), PI32, PI32],
        "simk_scan": [P, C.POINTER(Probe_t), i32, C.POINTER(P), i32, PD, i32, C.POINTER(Detector_t), C.POINTER(PD)],
        "simk_scan_device": [P, C.POINTER(Probe_t), i32, C.POINTER(P), i32, P, i32, C.POINTER(Detector_t),
                             C.POINTER(P)],
        "simk_fft2": [P, i32, i32, i32, i32, i32, PD, PD, PD, PD],
        "simk_probe_spectrum_noalloc": [C.POINTER(Grid_t), C.POINTER(Probe_t), P, P],
        "simk_finite_profile": [P, i32, PI32, PD, PD, PD, PD],
        "simk_potential_from_atoms_finite": [P, C.POINTER(Grid_t), i32, PD, i32, PI32, PD, P, d, PI32, PD,
                                             C.POINTER(P)],
        "simk_surrogate_train": [P, i32, PI32, i64, i32, i32, d, C.c_uint64, d, d, C.POINTER(P)],
        "simk_surrogate_destroy": [P],
        "simk_surrogate_info": [P, PD],
        "simk_surrogate_evaluate": [P, P, i32, PI32, PD, PD, PD, PD],
        "simk_surrogate_parameters": [P, P, C.POINTER(C.c_float), C.POINTER(C.c_float), PD],
        "simk_surrogate_gradients": [P, P, i32, PI32, PD, PD, PD, PD, C.POINTER(C.c_float), PD],
        "simk_job_table_run": [P, i32, C.POINTER(Job_t), PD],
        "simk_scan_waves": [P, C.POINTER(Probe_t), P, i32, PD, i32, i32, PD, PD],
        "simk_ctf_kernel": [P, C.POINTER(Grid_t), d, C.POINTER(Ctf_t), PD, PD],
        "simk_apply_ctf": [P, C.POINTER(Grid_t), d, C.POINTER(Ctf_t), i32, PD, PD, PD, PD, PD],
        "simk_gaussian_source_size": [P, i32, i32, i64, d, d, d, d, PD, PD],
        "simk_gaussian_source_size_device": [P, i32, i32, i64, d, d, d, d, P, P],
        "simk_poisson_noise": [P, i64, PD, d, i32, C.c_uint64, PD],
        "simk_poisson_noise_device": [P, i64, P, d, i32, C.c_uint64, P],
        "simk_integrate_gradient": [P, i32, i32, d, d, PD, PD, i64, PD],
        "simk_integrate_gradient_device": [P, i32, i32, d, d, P, P, i64, P],
        "simk_potential_tile": [P, P, i32, i32, i32, C.POINTER(P)],
        "simk_potential_project": [P, P, PD],
        "simk_potential_grid": [P, C.POINTER(Grid_t)],
    }
    for name, args in sig.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = C.c_int
    lib.simk_last_error.argtypes = []
    lib.simk_last_error.restype = C.c_char_p


def lib():
    """The loaded library; raises CudaUnavailable when it is not built."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise CudaUnavailable(SIMK_ERR_UNAVAILABLE,
                                      f"{LIB_PATH} is not built: run `python -m simulatokit_b200.build`")
            h = C.CDLL(LIB_PATH)
            _signatures(h)
            _lib = h
        return _lib


def check(status: int):
    if status == SIMK_OK:
        return
    msg = lib().simk_last_error().decode(errors="replace")
    if status == SIMK_ERR_UNAVAILABLE:
        raise CudaUnavailable(status, msg)
    if status == SIMK_ERR_INVALID:
        raise InvalidArgument(status, msg)
    raise CudaFailure(status, msg)


def dptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(PD)


def iptr(a: np.ndarray):
    assert a.dtype == np.int32 and a.flags.c_contiguous
    return a.ctypes.data_as(PI32)
