"""ctypes mirror of include/amoeba_gpu.h and the loader of libamoeba_gpu.so.

The structures here must match the C header field for field; tests check the
exported symbols against the header's declarations.  The library is built
in-tree (polmdqc_b200/_lib/libamoeba_gpu.so) by polmdqc_b200.build; a missing
library is an error, never a silent fallback.
"""
from __future__ import annotations

import ctypes as C
import os
import re

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB_PATH = os.path.join(HERE, "_lib", "libamoeba_gpu.so")
HEADER = os.path.join(ROOT, "include", "amoeba_gpu.h")

AMG_OK = 0
STATUS = {0: "OK", 1: "BAD_ARG", 2: "UNSUPPORTED", 3: "NO_CONVERGE", 4: "NAN",
          5: "CUDA_ERROR", 6: "NO_DEVICE", 7: "OUT_OF_RANGE"}

FRAME_NONE, FRAME_ZTHENX, FRAME_ZONLY, FRAME_BISECTOR, FRAME_ZBISECT, FRAME_THREEFOLD = range(6)
PREC_FP64, PREC_MIXED = 0, 1
POL_NONE, POL_MUTUAL, POL_DIRECT, POL_OPT = 0, 1, 2, 3
CELL_FROM_ANGLES, CELL_OCTAHEDRON, CELL_DODECAHEDRON = 0, 1, 2
PRED_NONE, PRED_GEAR, PRED_ASPC = 0, 1, 2
DO_ENERGY, DO_ANALYSIS, DO_GRADIENT, DO_VIRIAL, DO_DIPOLES = 1, 2, 4, 8, 16
PEN_NONE, PEN_GORDON1, PEN_GORDON2 = 0, 1, 2

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)


class amg_list(C.Structure):
    _fields_ = [("offsets", _ip), ("indices", _ip)]


class amg_params(C.Structure):
    _fields_ = [
        ("n", C.c_int32),
        ("pole", _dp),
        ("zaxis", _ip), ("xaxis", _ip), ("yaxis", _ip), ("polaxe", _ip),
        ("molcule", _ip),
        ("polarity", _dp), ("thole", _dp), ("pdamp", _dp),
        ("i12", amg_list), ("i13", amg_list), ("i14", amg_list), ("i15", amg_list),
        ("ip11", amg_list), ("ip12", amg_list), ("ip13", amg_list), ("ip14", amg_list),
        ("m_scale", C.c_double * 4), ("p_scale", C.c_double * 4), ("p_iscale", C.c_double * 4),
        ("d_scale", C.c_double * 4), ("u_scale", C.c_double * 4),
        ("use_ewald", C.c_int32), ("use_bounds", C.c_int32),
        ("aewald", C.c_double), ("nfft", C.c_int32 * 3), ("bsorder", C.c_int32),
        ("cutoff", C.c_double),
        ("poltyp", C.c_int32), ("poleps", C.c_double), ("politer", C.c_int32),
        ("electric", C.c_double), ("dielec", C.c_double), ("debye", C.c_double),
        ("precision", C.c_int32), ("pcg_guess", C.c_int32), ("device", C.c_int32),
        ("pcg_prec", C.c_int32), ("usolvcut", C.c_double),
        ("cell_shape", C.c_int32),
        ("opt_coef", C.c_double * 7),
        ("pentype", C.c_int32), ("pcore", _dp), ("palpha", _dp),
        ("cflux", C.c_int32),
        ("nbond", C.c_int32), ("bond_atoms", _ip), ("bond_flux", _dp),
        ("nangle", C.c_int32), ("angle_atoms", _ip), ("angle_flux", _dp),
    ]


class amg_results(C.Structure):
    _fields_ = [
        ("em", C.c_double), ("ep", C.c_double), ("einter", C.c_double),
        ("nem", C.c_int64), ("nep", C.c_int64),
        ("vir", C.c_double * 9),
        ("dem", _dp), ("dep", _dp), ("aem", _dp), ("aep", _dp),
        ("uind", _dp), ("uinp", _dp), ("rpole", _dp),
        ("pcg_iters", C.c_int32), ("pcg_eps", C.c_double),
    ]


class amg_cotangents(C.Structure):
    _fields_ = [("d_energy", C.c_double), ("d_uind", _dp), ("d_uinp", _dp)]


class amg_param_grads(C.Structure):
    _fields_ = [("d_pole", _dp), ("d_polarity", _dp), ("d_thole", _dp), ("d_xyz", _dp)]


def dptr(a):
    """double* of a C-contiguous float64 numpy array (or NULL for None)."""
    if a is None:
        return C.cast(None, _dp)
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"], "need contiguous float64"
    return a.ctypes.data_as(_dp)


def iptr(a):
    if a is None:
        return C.cast(None, _ip)
    assert a.dtype == np.int32 and a.flags["C_CONTIGUOUS"], "need contiguous int32"
    return a.ctypes.data_as(_ip)


def header_functions(path: str = HEADER) -> list[str]:
    """Names of the functions the public header declares."""
    text = open(path).read()
    return sorted(set(re.findall(r"^\s*(?:int|void|const char\*)\s+\**(amg_\w+)\s*\(", text, re.M)))


_lib = None


def load_library(path: str = LIB_PATH) -> C.CDLL:
    """Loads libamoeba_gpu.so and declares argument types.  Raises if absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(f"libamoeba_gpu.so not built at {path}; run polmdqc_b200.build.build()")
    lib = C.CDLL(path)
    P = C.POINTER
    lib.amg_create.argtypes = [P(amg_params), P(C.c_void_p)]
    lib.amg_set_coords.argtypes = [C.c_void_p, _dp, _dp]
    lib.amg_forward.argtypes = [C.c_void_p, C.c_int32, P(amg_results)]
    lib.amg_backward.argtypes = [C.c_void_p, P(amg_cotangents), P(amg_param_grads)]
    lib.amg_last_timing.argtypes = [C.c_void_p, _dp]
    lib.amg_bench.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.c_int64, _dp, C.POINTER(C.c_int64)]
    lib.amg_time_tu_kernel.argtypes = [C.c_void_p, C.c_int32, C.c_int64, _dp, _dp, C.POINTER(C.c_int64)]
    lib.amg_last_stats.argtypes = [C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.c_int32), C.POINTER(C.c_int32)]
    lib.amg_last_virial.argtypes = [C.c_void_p, _dp, _dp]
    lib.amg_fma_peak.argtypes = [C.c_int32, C.c_int32, _dp]
    lib.amg_set_predictor.argtypes = [C.c_void_p, C.c_int32]
    lib.amg_last_error.argtypes = [C.c_void_p]
    lib.amg_last_error.restype = C.c_char_p
    lib.amg_abi_version.argtypes = []
    lib.amg_destroy.argtypes = [C.c_void_p]
    lib.amg_destroy.restype = None
    for name in ("amg_create", "amg_set_coords", "amg_forward", "amg_backward", "amg_last_timing",
                 "amg_abi_version", "amg_bench", "amg_last_stats", "amg_time_tu_kernel", "amg_last_virial",
                 "amg_fma_peak", "amg_set_predictor"):
        getattr(lib, name).restype = C.c_int
    _lib = lib
    return lib
