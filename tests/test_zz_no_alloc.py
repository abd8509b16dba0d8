"""The allocation-free entry point, amg_empole_direct_noalloc.

It serves callers that cannot let a library allocate device memory (all
device memory taken from one arena at start-up, or no cudaMalloc/cudaFree
between steps because they synchronize the device): every buffer is the
caller's, and the kernels' scratch lives in one fixed device array inside the
library.  Checked here through the C ABI against the regular entry point
(amg_create/amg_forward, FP64, the same non-Ewald multipole mode) on two calls
in a row, the second reusing the scratch the first left behind.  Collected
last on purpose, so that a failure here comes after every other test.
"""
import ctypes as C

import numpy as np
import pytest

from polmdqc_b200 import abi, systems
from polmdqc_b200.engine import Engine, Settings

pytestmark = pytest.mark.gpu


def _declare(lib):
    f = lib.amg_empole_direct_noalloc
    f.argtypes = [C.c_int32] + [C.c_void_p] * 6 + [C.POINTER(abi.amg_list), C.POINTER(C.c_double),
                                                    C.POINTER(C.c_double), C.c_double, C.c_double, C.c_void_p,
                                                    C.c_void_p, C.c_void_p]
    f.restype = C.c_int
    return f


def test_noalloc_matches_regular_entry_point_twice():
    import torch
    lib = abi.load_library()
    fn = _declare(lib)
    s = systems.water_box(216, 18.643, seed=0)
    st = Settings(use_ewald=False, cutoff=7.0, poltyp=abi.POL_NONE, precision=abi.PREC_FP64)
    eng = Engine(s, st)
    try:
        ref = eng.forward(abi.DO_ENERGY | abi.DO_GRADIENT)
    finally:
        eng.close()

    dev = torch.device("cuda", 0)
    keep = []

    def d(a, dtype):
        t = torch.as_tensor(np.ascontiguousarray(a), dtype=dtype, device=dev).contiguous()
        keep.append(t)
        return C.c_void_p(t.data_ptr())

    n = s.n
    xyz = d(s.xyz.reshape(-1), torch.float64)
    pole = d(s.pole.reshape(-1), torch.float64)
    frames = [d(getattr(s, k), torch.int32) for k in ("zaxis", "xaxis", "yaxis", "polaxe")]
    lists = (abi.amg_list * 4)()
    for b, name in enumerate(("i12", "i13", "i14", "i15")):
        off, idx = s.csr(name)
        if idx.size == 0:
            idx = np.zeros(1, np.int32)
        lists[b] = abi.amg_list(C.cast(d(off, torch.int32), abi._ip), C.cast(d(idx, torch.int32), abi._ip))
    ms = (C.c_double * 4)(*s.m_scale)
    box = (C.c_double * 3)(*s.box[:3])
    em = torch.zeros(1, dtype=torch.float64, device=dev)
    dem = torch.zeros(3 * n, dtype=torch.float64, device=dev)
    f = st.electric / st.dielec
    torch.cuda.synchronize()
    for call in range(2):
        em.zero_()
        dem.zero_()
        torch.cuda.synchronize()
        rc = fn(n, xyz, pole, *frames, lists, ms, box, 7.0, f, C.c_void_p(em.data_ptr()),
                C.c_void_p(dem.data_ptr()), None)
        assert rc == abi.AMG_OK, (call, abi.STATUS.get(rc, rc))
        e = float(em.item())
        g = dem.cpu().numpy().reshape(n, 3)
        assert abs(e - ref.em) < 1e-10 * abs(ref.em), (call, e, ref.em)
        np.testing.assert_allclose(g, ref.dem, atol=1e-8, rtol=0)


def test_noalloc_rejects_oversized_systems():
    lib = abi.load_library()
    fn = _declare(lib)
    lists = (abi.amg_list * 4)()
    ms = (C.c_double * 4)(0, 0, 0.4, 0.8)
    p = C.c_void_p(1)
    rc = fn(16385, p, p, p, p, p, p, lists, ms, None, 7.0, 332.0, p, p, None)
    assert rc == 7   # AMG_ERR_OUT_OF_RANGE
