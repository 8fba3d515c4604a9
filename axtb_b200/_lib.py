"""ctypes binding of ``libaxtb_gpu.so`` (include/axtb_gpu.h, include/axtb_gpu_debug.h).

The library is built in-tree (``python -m axtb_b200.build`` or ``__graft_entry__.build()``) for
sm_100a. There is no CPU implementation behind this package: loading fails with an error
when the library is missing, and every call needs a CUDA device.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libaxtb_gpu.so"

AXTB_OK = 0
AXTB_ERR_INPUT = 1
AXTB_ERR_UNSUPPORTED_ELEMENT = 2
AXTB_ERR_SCF_NOT_CONVERGED = 3
AXTB_ERR_NUMERICAL = 4
AXTB_ERR_DEVICE = 5

DBG = {"cn": 0, "overlap": 1, "h0": 2, "dipole": 3, "quadrupole": 4, "density": 5, "fock": 6, "emo": 7,
       "focc": 8, "wdensity": 9, "eeq": 10, "linv": 11, "eigen_cycles": 12,
       "status_bits": 13}


class AxtbOptions(C.Structure):
    _fields_ = [("accuracy", C.c_double), ("etemp", C.c_double), ("max_iter", C.c_int32), ("damping", C.c_double),
                ("guess", C.c_int32), ("precision", C.c_int32), ("device", C.c_int32), ("mixer", C.c_int32),
                ("conventions", C.c_int32), ("solvation", C.c_int32), ("solvent", C.c_char_p),
                ("solvation_state", C.c_int32), ("dispersion", C.c_int32),
                ("band_max_nao", C.c_int32), ("grid_min_nao", C.c_int32)]


class AxtbResult(C.Structure):
    _fields_ = [("energy", C.c_double), ("gradient", C.POINTER(C.c_double)), ("charges", C.POINTER(C.c_double)),
                ("dipole", C.POINTER(C.c_double)), ("qsh", C.POINTER(C.c_double)), ("dpat", C.POINTER(C.c_double)),
                ("qpat", C.POINTER(C.c_double)), ("terms", C.c_double * 8), ("iterations", C.c_int32),
                ("converged", C.c_int32), ("status", C.c_int32), ("energy_change", C.c_double),
                ("residual", C.c_double), ("mixer_used", C.c_int32), ("solvation", C.c_double),
                ("emo", C.POINTER(C.c_double)), ("focc", C.POINTER(C.c_double)), ("focc_alpha", C.POINTER(C.c_double)),
                ("fermi_levels", C.c_double * 2), ("electronic_temperature", C.c_double), ("nao", C.c_int32),
                ("warm_start", C.c_int32), ("fallback_iterations", C.c_int32), ("timings", C.c_double * 4)]


class AxtbMol(C.Structure):
    _fields_ = [("nat", C.c_int32), ("numbers", C.POINTER(C.c_int32)), ("positions", C.POINTER(C.c_double)),
                ("charge", C.c_double), ("uhf", C.c_int32)]


# every entry point of include/axtb_gpu.h and include/axtb_gpu_debug.h: (restype, argtypes)
PD = C.POINTER(C.c_double)
PI32 = C.POINTER(C.c_int32)
SIGNATURES = {
    "axtb_gpu_default_options": (None, [C.POINTER(AxtbOptions)]),
    "axtb_gpu_basis_size": (C.c_int, [PI32, C.c_int32, PI32, PI32]),
    "axtb_gpu_create": (C.c_int, [PI32, C.c_int32, C.c_double, C.c_int32, C.POINTER(AxtbOptions), C.POINTER(C.c_void_p)]),
    "axtb_gpu_singlepoint": (C.c_int, [C.c_void_p, PD, C.c_int32, C.POINTER(AxtbResult)]),
    "axtb_gpu_destroy": (None, [C.c_void_p]),
    "axtb_gpu_last_error": (C.c_int, [C.c_void_p, C.c_char_p, C.c_size_t]),
    "axtb_gpu_batch": (C.c_int, [C.POINTER(AxtbMol), C.c_int32, C.POINTER(AxtbOptions), C.c_int32,
                                 C.POINTER(AxtbResult), PI32]),
    "axtb_gpu_batch_create": (C.c_int, [C.POINTER(AxtbMol), C.c_int32, C.POINTER(AxtbOptions), C.POINTER(C.c_void_p)]),
    "axtb_gpu_batch_run": (C.c_int, [C.c_void_p, PD, C.c_int32, C.POINTER(AxtbResult), PI32]),
    "axtb_gpu_batch_run_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, PI32]),
    "axtb_gpu_batch_stream": (C.c_void_p, [C.c_void_p]),
    "axtb_gpu_batch_launches": (C.c_int64, [C.c_void_p]),
    "axtb_gpu_batch_destroy": (None, [C.c_void_p]),
    "axtb_gpu_density_static": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32, C.c_double, C.c_double, C.c_double,
                                          C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "axtb_gpu_batch_debug": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, PD]),
    "axtb_gpu_batch_set_profiling": (C.c_int, [C.c_void_p, C.c_int32]),
    "axtb_gpu_batch_set_restart": (C.c_int, [C.c_void_p, C.c_int32]),
    "axtb_gpu_batch_profile": (C.c_int, [C.c_void_p, C.c_char_p, C.c_size_t]),
    "axtb_gpu_get_moments": (C.c_int, [C.c_void_p, PD, PD, PD]),
    "axtb_gpu_set_moments": (C.c_int, [C.c_void_p, PD, PD, PD, C.c_int32]),
    "axtb_gpu_batch_get_moments": (C.c_int, [C.c_void_p, C.c_int32, PD, PD, PD]),
    "axtb_gpu_batch_set_moments": (C.c_int, [C.c_void_p, C.c_int32, PD, PD, PD]),
}

_lib = None


def load() -> C.CDLL:
    """The engine library; raises when it was not built (there is no fallback)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m axtb_b200.build` "
                               "(the GFN2-xTB engine has no CPU path)")
        lib = C.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args
        _lib = lib
    return _lib


def last_error(handle=None) -> str:
    buf = C.create_string_buffer(512)
    load().axtb_gpu_last_error(handle, buf, 512)
    return buf.value.decode(errors="replace")


def default_options(**kw) -> AxtbOptions:
    o = AxtbOptions()
    load().axtb_gpu_default_options(C.byref(o))
    for k, v in kw.items():
        if v is not None:
            setattr(o, k, v)
    return o
