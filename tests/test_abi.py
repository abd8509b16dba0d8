"""The C ABI surface: the library builds for sm_100a, loads without a GPU,
exports every function include/amoeba_gpu.h declares, and the ctypes
structures have the C layout (checked against a C++ compile of the header)."""
import ctypes
import os
import subprocess
import tempfile

import pytest

from polmdqc_b200 import abi, build


def test_library_exports_header_symbols():
    build.build()
    lib = ctypes.CDLL(abi.LIB_PATH)
    declared = abi.header_functions()
    assert {"amg_create", "amg_set_coords", "amg_forward", "amg_backward", "amg_destroy"} <= set(declared)
    for name in declared:
        assert hasattr(lib, name), name
    assert lib.amg_abi_version() == 4


def test_struct_layout_matches_header():
    src = r"""
    #include <cstdio>
    #include <cstddef>
    #include "amoeba_gpu.h"
    int main() {
      printf("%zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu\n", sizeof(amg_params), sizeof(amg_results), sizeof(amg_cotangents),
             sizeof(amg_param_grads), offsetof(amg_params, precision), offsetof(amg_results, pcg_eps),
             offsetof(amg_params, u_scale), offsetof(amg_results, rpole), offsetof(amg_params, cell_shape),
             offsetof(amg_params, pentype), offsetof(amg_params, angle_flux));
    }"""
    with tempfile.TemporaryDirectory() as t:
        c = os.path.join(t, "s.cpp")
        open(c, "w").write(src)
        exe = os.path.join(t, "s")
        subprocess.check_call(["g++", "-I", os.path.dirname(abi.HEADER), c, "-o", exe])
        vals = [int(v) for v in subprocess.check_output([exe]).split()]
    P, R = abi.amg_params, abi.amg_results
    assert vals == [ctypes.sizeof(P), ctypes.sizeof(R), ctypes.sizeof(abi.amg_cotangents),
                    ctypes.sizeof(abi.amg_param_grads), P.precision.offset, R.pcg_eps.offset,
                    P.u_scale.offset, R.rpole.offset, P.cell_shape.offset, P.pentype.offset, P.angle_flux.offset]


def test_create_without_gpu_fails_cleanly():
    """No device (this check runs where there is none): amg_create returns a
    status instead of aborting, and bad arguments are rejected first."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    lib = abi.load_library()
    ctx = ctypes.c_void_p()
    assert lib.amg_create(None, ctypes.byref(ctx)) == 1          # BAD_ARG
    from polmdqc_b200 import systems
    from polmdqc_b200.engine import Params, Settings
    s = systems.water_box(8, 12.0, seed=0)
    p = Params(s, Settings(nfft=(12, 12, 12), cutoff=5.0))
    assert lib.amg_create(ctypes.byref(p.struct), ctypes.byref(ctx)) == 6   # NO_DEVICE


def test_parameter_validation_before_any_device_call():
    """amg_create checks its parameters before it touches a device, so the
    statuses of bad inputs hold on any host: unknown polarization model
    (UNSUPPORTED), OPT without coefficients, unknown cell shape, the sparse
    preconditioner without usolvcut (BAD_ARG); valid OPT and cell-shape
    parameters get as far as the device (NO_DEVICE here)."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from polmdqc_b200 import systems
    from polmdqc_b200.engine import Params, Settings
    BAD_ARG, UNSUPPORTED, NO_DEVICE = 1, 2, 6
    lib = abi.load_library()
    ctx = ctypes.c_void_p()
    s = systems.water_box(8, 12.0, seed=0)

    def status(**changes):
        p = Params(s, Settings(nfft=(12, 12, 12), cutoff=5.0))
        for k, v in changes.items():
            setattr(p.struct, k, v)
        return lib.amg_create(ctypes.byref(p.struct), ctypes.byref(ctx))

    assert status(poltyp=7) == UNSUPPORTED
    assert status(poltyp=abi.POL_OPT) == BAD_ARG          # all opt_coef zero
    assert status(cell_shape=5) == BAD_ARG
    assert status(pcg_prec=1, usolvcut=0.0) == BAD_ARG
    p = Params(s, Settings(nfft=(12, 12, 12), cutoff=5.0, poltyp=abi.POL_OPT, opt_order=4))
    assert lib.amg_create(ctypes.byref(p.struct), ctypes.byref(ctx)) == NO_DEVICE
    assert status(cell_shape=abi.CELL_OCTAHEDRON) == NO_DEVICE
