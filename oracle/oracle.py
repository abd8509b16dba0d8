"""ctypes front end of the FP64 CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, never by the product package.  Builds the
shared library from oracle/amoeba_oracle.cpp on first use if it is missing.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from polmdqc_b200 import abi
from polmdqc_b200.engine import Params, Settings, collect, new_results

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "amoeba_oracle.cpp")
LIB = os.path.join(HERE, "liboracle.so")
REF = os.path.join(HERE, "_ref")


class orc_options(C.Structure):
    _fields_ = [("kmax", C.c_double), ("tol", C.c_double), ("maxit", C.c_int32), ("alpha", C.c_double),
                ("raw_virial", C.c_int32)]


def build(force=False):
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(SRC):
        subprocess.check_call(["g++", "-std=c++17", "-O3", "-fopenmp", "-fPIC", "-shared", SRC, "-o", LIB])
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(LIB)
        L.orc_forward.argtypes = [C.POINTER(abi.amg_params), C.POINTER(C.c_double), C.POINTER(C.c_double),
                                  C.c_int32, C.POINTER(orc_options), C.POINTER(abi.amg_results)]
        L.orc_forward.restype = C.c_int
        L.orc_pair_count.argtypes = [C.POINTER(C.c_double), C.c_int32, C.POINTER(C.c_double), C.c_int32, C.c_double]
        L.orc_dipole_field.argtypes = [C.POINTER(abi.amg_params), C.POINTER(C.c_double), C.POINTER(C.c_double),
                                       C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.orc_dipole_field.restype = C.c_int
        L.orc_pair_count.restype = C.c_int64
        _lib = L
    return _lib


def forward(system, settings: Settings, xyz=None, flags=abi.DO_ENERGY | abi.DO_GRADIENT | abi.DO_DIPOLES,
            kmax=0.0, tol=0.0, maxit=0, alpha=0.0, params=None, check=True, raw_virial=False):
    """FP64 evaluation of em/ep (+gradients, dipoles) for `system`."""
    P = params or Params(system, settings)
    x = np.ascontiguousarray(system.xyz if xyz is None else xyz, np.float64).reshape(-1)
    box = np.ascontiguousarray(system.box, np.float64)
    r, bufs = new_results(system.n)
    opt = orc_options(kmax, tol, maxit, alpha, int(raw_virial))
    rc = lib().orc_forward(C.byref(P.struct), abi.dptr(x), abi.dptr(box), flags, C.byref(opt), C.byref(r))
    if check and rc not in (abi.AMG_OK,):
        raise RuntimeError(f"oracle failed: {abi.STATUS.get(rc, rc)}")
    res = collect(r, bufs, system.n)
    res.status = rc
    return res


def pair_count(system, cutoff):
    x = np.ascontiguousarray(system.xyz, np.float64).reshape(-1)
    box = np.ascontiguousarray(system.box, np.float64)
    return int(lib().orc_pair_count(abi.dptr(x), system.n, abi.dptr(box), int(system.use_bounds), cutoff))


def dipole_field(system, settings: Settings, u, params=None):
    """Field [n,3] of the dipoles u [n,3] (the T of (1/alpha - T) u = E)."""
    P = params or Params(system, settings)
    x = np.ascontiguousarray(system.xyz, np.float64).reshape(-1)
    box = np.ascontiguousarray(system.box, np.float64)
    uu = np.ascontiguousarray(u, np.float64).reshape(-1)
    out = np.zeros(3 * system.n)
    rc = lib().orc_dipole_field(C.byref(P.struct), abi.dptr(x), abi.dptr(box), abi.dptr(uu), abi.dptr(out))
    if rc != abi.AMG_OK:
        raise RuntimeError(f"oracle failed: {abi.STATUS.get(rc, rc)}")
    return out.reshape(system.n, 3)
