"""Host-side API over libamoeba_gpu.so (the C ABI of include/amoeba_gpu.h).

`Settings` carries the keyfile-level options the reference reads in
cutoffs/kewald/kpolar (cutoff, Ewald alpha, PME grid and order, polarization
model, convergence); `make_params` marshals a `System` plus `Settings` into
the C struct; `Engine` owns one device context and exposes forward/backward
in the reference's result layout (em, ep, dem, dep, uind, uinp).
"""
from __future__ import annotations

import ctypes as C
import dataclasses

import numpy as np

from . import abi
from .prm import COULOMB, DEBYE
from .systems import System


# OPT extrapolation coefficients copt_0..copt_k per order, the reference's
# table (src/md/kpolar.cpp:115-153)
OPT_COEF = {
    1: (0.530, 0.604),
    2: (0.042, 0.635, 0.414),
    3: (-0.132, 0.218, 0.637, 0.293),
    4: (-0.071, -0.096, 0.358, 0.587, 0.216),
    5: (-0.005, -0.129, -0.026, 0.465, 0.528, 0.161),
    6: (0.014, -0.041, -0.172, 0.073, 0.535, 0.467, 0.122),
}


@dataclasses.dataclass
class Settings:
    use_ewald: bool = True
    aewald: float = 0.5446            # 1/Angstrom
    nfft: tuple = (24, 24, 24)
    bsorder: int = 5
    cutoff: float = 7.0               # ewald-cutoff (mpole-cutoff without Ewald)
    poltyp: int = abi.POL_MUTUAL
    poleps: float = 1e-6              # Debye RMS
    politer: int = 100
    precision: int = abi.PREC_MIXED
    pcg_guess: bool = True
    pcg_prec: bool = True             # sparse preconditioner within usolvcut (reference default)
    usolvcut: float = 4.5             # Angstrom
    opt_order: int = 4                # poltyp POL_OPT: OPT1..OPT6 (the reference's "OPT" is OPT4)
    electric: float = COULOMB
    dielec: float = 1.0
    device: int = 0


class Params:
    """amg_params plus the numpy arrays it points into (kept alive)."""

    def __init__(self, s: System, st: Settings):
        self.keep = []
        p = abi.amg_params()
        p.n = s.n
        pole = np.ascontiguousarray(s.pole.reshape(-1), np.float64)
        ints = {k: np.ascontiguousarray(getattr(s, k), np.int32) for k in ("zaxis", "xaxis", "yaxis", "polaxe", "molcule")}
        self.keep += [pole] + list(ints.values())
        p.pole = abi.dptr(pole)
        for k, v in ints.items():
            setattr(p, k, abi.iptr(v))
        if st.poltyp != abi.POL_NONE:
            pol = np.ascontiguousarray(s.polarity, np.float64)
            thl = np.ascontiguousarray(s.thole, np.float64)
            pdp = np.ascontiguousarray(s.pdamp, np.float64)
            self.keep += [pol, thl, pdp]
            p.polarity, p.thole, p.pdamp = abi.dptr(pol), abi.dptr(thl), abi.dptr(pdp)
        for name in ("i12", "i13", "i14", "i15", "ip11", "ip12", "ip13", "ip14"):
            off, idx = s.csr(name)
            if idx.size == 0:
                idx = np.zeros(1, np.int32)
            self.keep += [off, idx]
            setattr(p, name, abi.amg_list(abi.iptr(off), abi.iptr(idx)))
        for name in ("m_scale", "p_scale", "p_iscale", "d_scale", "u_scale"):
            arr = getattr(p, name)
            for j, v in enumerate(getattr(s, name)):
                arr[j] = v
        p.use_ewald = int(st.use_ewald)
        p.use_bounds = int(s.use_bounds)
        p.cell_shape = int(getattr(s, "cell_shape", 0))
        p.aewald = st.aewald
        for j in range(3):
            p.nfft[j] = st.nfft[j]
        p.bsorder = st.bsorder
        p.cutoff = st.cutoff
        p.poltyp = st.poltyp
        p.poleps = st.poleps
        p.politer = st.politer
        p.electric = st.electric
        p.dielec = st.dielec
        p.debye = DEBYE
        p.precision = st.precision
        p.pcg_guess = int(st.pcg_guess)
        p.device = st.device
        p.pcg_prec = int(st.pcg_prec)
        p.usolvcut = st.usolvcut
        if st.poltyp == abi.POL_OPT:
            for k, c in enumerate(OPT_COEF[st.opt_order]):
                p.opt_coef[k] = c
        if getattr(s, "pentype", 0):
            pc = np.ascontiguousarray(s.pcore, np.float64)
            pa = np.ascontiguousarray(s.palpha, np.float64)
            self.keep += [pc, pa]
            p.pentype, p.pcore, p.palpha = int(s.pentype), abi.dptr(pc), abi.dptr(pa)
        if getattr(s, "cflux", False):
            ba = np.ascontiguousarray(s.bond_atoms, np.int32).reshape(-1)
            bf = np.ascontiguousarray(s.bond_flux, np.float64).reshape(-1)
            aa = np.ascontiguousarray(s.angle_atoms, np.int32).reshape(-1)
            af = np.ascontiguousarray(s.angle_flux, np.float64).reshape(-1)
            self.keep += [ba, bf, aa, af]
            p.cflux = 1
            p.nbond, p.bond_atoms, p.bond_flux = len(s.bond_atoms), abi.iptr(ba), abi.dptr(bf)
            p.nangle, p.angle_atoms, p.angle_flux = len(s.angle_atoms), abi.iptr(aa), abi.dptr(af)
        self.struct = p
        self.n = s.n


@dataclasses.dataclass
class Result:
    em: float
    ep: float
    einter: float
    nem: int
    nep: int
    dem: np.ndarray
    dep: np.ndarray
    aem: np.ndarray
    aep: np.ndarray
    uind: np.ndarray
    uinp: np.ndarray
    rpole: np.ndarray
    pcg_iters: int
    pcg_eps: float
    vir: np.ndarray


def new_results(n):
    bufs = {k: np.zeros(3 * n) for k in ("dem", "dep", "uind", "uinp")}
    bufs.update(aem=np.zeros(n), aep=np.zeros(n), rpole=np.zeros(13 * n))
    r = abi.amg_results()
    for k, v in bufs.items():
        setattr(r, k, abi.dptr(v))
    return r, bufs


def collect(r, bufs, n) -> Result:
    return Result(em=r.em, ep=r.ep, einter=r.einter, nem=r.nem, nep=r.nep,
                  dem=bufs["dem"].reshape(n, 3), dep=bufs["dep"].reshape(n, 3),
                  aem=bufs["aem"], aep=bufs["aep"], uind=bufs["uind"].reshape(n, 3),
                  uinp=bufs["uinp"].reshape(n, 3), rpole=bufs["rpole"].reshape(n, 13),
                  pcg_iters=r.pcg_iters, pcg_eps=r.pcg_eps, vir=np.array(r.vir[:]).reshape(3, 3))


class AmgError(RuntimeError):
    pass


def fma_peak(device=0, fp64=False):
    """Measured FMA throughput of the device in GFLOP/s (amg_fma_peak)."""
    lib = abi.load_library()
    out = C.c_double(0)
    rc = lib.amg_fma_peak(device, int(fp64), C.byref(out))
    if rc != abi.AMG_OK:
        raise AmgError(f"amg_fma_peak: {abi.STATUS.get(rc, rc)}")
    return out.value


class Engine:
    """One device context (amg_create .. amg_destroy)."""

    def __init__(self, s: System, st: Settings):
        self.lib = abi.load_library()
        self.params = Params(s, st)
        self.n = s.n
        self.ctx = C.c_void_p()
        rc = self.lib.amg_create(C.byref(self.params.struct), C.byref(self.ctx))
        if rc != abi.AMG_OK:
            raise AmgError(f"amg_create failed: {abi.STATUS.get(rc, rc)}")
        self.box = np.ascontiguousarray(s.box, np.float64)
        self.set_coords(s.xyz)

    def _check(self, rc, what):
        if rc != abi.AMG_OK:
            msg = self.lib.amg_last_error(self.ctx)
            raise AmgError(f"{what}: {abi.STATUS.get(rc, rc)}: {msg.decode() if msg else ''}")

    def set_coords(self, xyz, box=None):
        xyz = np.ascontiguousarray(xyz, np.float64).reshape(-1)
        if box is not None:
            self.box = np.ascontiguousarray(box, np.float64)
        self._check(self.lib.amg_set_coords(self.ctx, abi.dptr(xyz), abi.dptr(self.box)), "amg_set_coords")

    def forward(self, flags=abi.DO_ENERGY | abi.DO_GRADIENT | abi.DO_DIPOLES) -> Result:
        r, bufs = new_results(self.n)
        self._check(self.lib.amg_forward(self.ctx, flags, C.byref(r)), "amg_forward")
        return collect(r, bufs, self.n)

    def forward_into(self, flags, dem=None, dep=None):
        """amg_forward writing only the given gradient buffers (added to);
        returns (em, ep, pcg_iters, pcg_eps)."""
        r = abi.amg_results()
        r.dem, r.dep = abi.dptr(dem), abi.dptr(dep)
        self._check(self.lib.amg_forward(self.ctx, flags, C.byref(r)), "amg_forward")
        return r.em, r.ep, r.pcg_iters, r.pcg_eps

    def backward(self, d_energy=1.0, d_uind=None, d_uinp=None):
        cot = abi.amg_cotangents(d_energy, abi.dptr(d_uind), abi.dptr(d_uinp))
        out = {"d_pole": np.zeros(13 * self.n), "d_polarity": np.zeros(self.n),
               "d_thole": np.zeros(self.n), "d_xyz": np.zeros(3 * self.n)}
        g = abi.amg_param_grads(*(abi.dptr(out[k]) for k in ("d_pole", "d_polarity", "d_thole", "d_xyz")))
        self._check(self.lib.amg_backward(self.ctx, C.byref(cot), C.byref(g)), "amg_backward")
        out["d_pole"] = out["d_pole"].reshape(self.n, 13)
        out["d_xyz"] = out["d_xyz"].reshape(self.n, 3)
        return out

    def set_predictor(self, kind):
        """Induced-dipole predictor (abi.PRED_*); clears the dipole history."""
        self._check(self.lib.amg_set_predictor(self.ctx, kind), "amg_set_predictor")

    def bench(self, steps, flags=abi.DO_ENERGY | abi.DO_GRADIENT, flush_bytes=0):
        """Device-resident evaluations: per-step ms (CUDA events) and the
        number of this library's kernel launches."""
        ms = np.zeros(steps)
        launches = C.c_int64(0)
        self._check(self.lib.amg_bench(self.ctx, flags, steps, flush_bytes, abi.dptr(ms), C.byref(launches)),
                    "amg_bench")
        return ms, int(launches.value)

    def time_tu_kernel(self, reps=20, flush_bytes=256 << 20):
        """(avg ms, algorithmic bytes per launch, directed pairs) of the PCG's
        stored-coefficient T.u kernel, each launch after an L2 flush."""
        ms, by, pairs = C.c_double(0), C.c_double(0), C.c_int64(0)
        self._check(self.lib.amg_time_tu_kernel(self.ctx, reps, flush_bytes, C.byref(ms), C.byref(by), C.byref(pairs)),
                    "amg_time_tu_kernel")
        return ms.value, by.value, int(pairs.value)

    def stats(self):
        launches, graphed, lpa = C.c_int64(0), C.c_int32(0), C.c_int32(0)
        self._check(self.lib.amg_last_stats(self.ctx, C.byref(launches), C.byref(graphed), C.byref(lpa)),
                    "amg_last_stats")
        return {"launches": int(launches.value), "graphed": bool(graphed.value), "lanes_per_site": int(lpa.value)}

    def virial_parts(self):
        """The em and ep parts (3x3 each) of the last forward's virial."""
        vm, vp = np.zeros(9), np.zeros(9)
        self._check(self.lib.amg_last_virial(self.ctx, abi.dptr(vm), abi.dptr(vp)), "amg_last_virial")
        return vm.reshape(3, 3), vp.reshape(3, 3)

    def timing(self):
        ms = np.zeros(5)
        self._check(self.lib.amg_last_timing(self.ctx, abi.dptr(ms)), "amg_last_timing")
        return ms

    def close(self):
        if self.ctx:
            self.lib.amg_destroy(self.ctx)
            self.ctx = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
