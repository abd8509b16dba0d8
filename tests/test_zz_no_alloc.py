"""The allocation-free entry point, amg_empole_direct_noalloc.

It serves callers that cannot let a library allocate device memory: codes
that take all device memory from one arena at start-up and forbid later
allocation, and codes that must not call cudaMalloc/cudaFree between steps
because those calls synchronize the whole device.  Every buffer is the
caller's, and the kernels' scratch lives in one fixed device array inside the
library.  Checked here through the C ABI against the regular entry point
(amg_create/amg_forward, FP64, the same non-Ewald multipole mode) on two calls
in a row, the second reusing the scratch the first left behind, and on a
smaller open cluster right after a larger periodic call.  Collected last on
purpose, so that a failure here comes after every other test.
"""
import ctypes as C
import dataclasses

import numpy as np
import pytest

from polmdqc_b200 import abi, systems
from polmdqc_b200.engine import Engine, Settings

pytestmark = pytest.mark.gpu

CUT = 7.0


def _declare(lib):
    f = lib.amg_empole_direct_noalloc
    f.argtypes = [C.c_int32] + [C.c_void_p] * 6 + [C.POINTER(abi.amg_list), C.POINTER(C.c_double),
                                                    C.POINTER(C.c_double), C.c_double, C.c_double, C.c_void_p,
                                                    C.c_void_p, C.c_void_p]
    f.restype = C.c_int
    return f


def _regular(s):
    """em and dem of the regular entry point (FP64, non-Ewald, no polarization)."""
    st = Settings(use_ewald=False, cutoff=CUT, poltyp=abi.POL_NONE, precision=abi.PREC_FP64)
    eng = Engine(s, st)
    try:
        return eng.forward(abi.DO_ENERGY | abi.DO_GRADIENT), st.electric / st.dielec
    finally:
        eng.close()


class _Call:
    """Device copies of one system's inputs and one call of the entry point."""

    def __init__(self, s, periodic):
        import torch
        self.torch = torch
        self.dev = torch.device("cuda", 0)
        self.keep = []
        self.n = s.n
        self.xyz = self._d(s.xyz.reshape(-1), torch.float64)
        self.pole = self._d(s.pole.reshape(-1), torch.float64)
        self.frames = [self._d(getattr(s, k), torch.int32) for k in ("zaxis", "xaxis", "yaxis", "polaxe")]
        self.lists = (abi.amg_list * 4)()
        for b, name in enumerate(("i12", "i13", "i14", "i15")):
            off, idx = s.csr(name)
            if idx.size == 0:
                idx = np.zeros(1, np.int32)
            self.lists[b] = abi.amg_list(C.cast(self._d(off, torch.int32), abi._ip),
                                         C.cast(self._d(idx, torch.int32), abi._ip))
        self.ms = (C.c_double * 4)(*s.m_scale)
        self.box = (C.c_double * 3)(*s.box[:3]) if periodic else None
        self.em = torch.zeros(1, dtype=torch.float64, device=self.dev)
        self.dem = torch.zeros(3 * self.n, dtype=torch.float64, device=self.dev)

    def _d(self, a, dtype):
        t = self.torch.as_tensor(np.ascontiguousarray(a), dtype=dtype, device=self.dev).contiguous()
        self.keep.append(t)
        return C.c_void_p(t.data_ptr())

    def run(self, fn, f):
        self.em.fill_(12345.0)   # overwritten by the call
        self.dem.zero_()         # added to by the call
        self.torch.cuda.synchronize()
        rc = fn(self.n, self.xyz, self.pole, *self.frames, self.lists, self.ms, self.box, CUT, f,
                C.c_void_p(self.em.data_ptr()), C.c_void_p(self.dem.data_ptr()), None)
        assert rc == abi.AMG_OK, abi.STATUS.get(rc, rc)
        return float(self.em.item()), self.dem.cpu().numpy().reshape(self.n, 3)


def _check(e, g, ref):
    assert abs(e - ref.em) < 1e-10 * abs(ref.em), (e, ref.em)
    np.testing.assert_allclose(g, ref.dem, atol=1e-8, rtol=0)


def test_noalloc_matches_regular_entry_point_twice():
    fn = _declare(abi.load_library())
    s = systems.water_box(216, 18.643, seed=0)
    ref, f = _regular(s)
    call = _Call(s, periodic=True)
    for _ in range(2):
        e, g = call.run(fn, f)
        _check(e, g, ref)


def test_noalloc_open_cluster_after_a_larger_call():
    """No box (no wrapping), 105 atoms (a partial last block of sites), run
    right after a 648-atom periodic call that left its scratch behind."""
    fn = _declare(abi.load_library())
    big = systems.water_box(216, 18.643, seed=3)
    ref_big, f = _regular(big)
    e, g = _Call(big, periodic=True).run(fn, f)
    _check(e, g, ref_big)
    small = dataclasses.replace(systems.water_box(35, 10.5, seed=4), use_bounds=False)
    assert small.n % 4 != 0
    ref_small, f = _regular(small)
    e, g = _Call(small, periodic=False).run(fn, f)
    _check(e, g, ref_small)


def test_noalloc_rejects_oversized_systems():
    lib = abi.load_library()
    fn = _declare(lib)
    lists = (abi.amg_list * 4)()
    ms = (C.c_double * 4)(0, 0, 0.4, 0.8)
    p = C.c_void_p(1)
    rc = fn(16385, p, p, p, p, p, p, lists, ms, None, 7.0, 332.0, p, p, None)
    assert rc == 7   # AMG_ERR_OUT_OF_RANGE
