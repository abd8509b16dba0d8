"""The headline configurations at full size against the FP64 oracle.

  * 32,768 rigid waters (98,304 atoms, water03) in a 99.3 A box, PME 108^3
    order 5, alpha 0.5446, cutoff 7 A, mutual polarization;
  * the ion solution: 8,000 waters + 22 Na+ + 22 Cl- (amoebabio18, 24,044
    atoms) in a 62.1 A box, PME 72^3.

The oracle runs once per configuration (module fixtures, OpenMP on every
host core) with the PCG converged to 1e-10 D.  Bounds:
  FP64 GPU path (poleps 1e-8 D): em 1e-10 and ep 1e-8 relative, induced
    dipoles 1e-7 D RMS, gradients 1e-5 kcal/mol/A;
  mixed path (poleps 1e-6 D, the production setting): em and ep 1e-6
    relative, force RMS 1e-4 kcal/mol/A, induced dipoles 1e-5 D RMS.
"""
import numpy as np
import pytest

from oracle import oracle
from polmdqc_b200 import abi, systems
from polmdqc_b200.engine import Engine, Settings
from polmdqc_b200.prm import DEBYE

pytestmark = pytest.mark.gpu

FP64, MIXED = abi.PREC_FP64, abi.PREC_MIXED
ALL = abi.DO_ENERGY | abi.DO_GRADIENT | abi.DO_DIPOLES


def rel(a, b):
    return abs(a - b) / abs(b)


def run(s, st):
    e = Engine(s, st)
    try:
        return e.forward(ALL)
    finally:
        e.close()


def dipole_rms_debye(g, o):
    d = np.concatenate([g.uind - o.uind, g.uinp - o.uinp])
    return DEBYE * float(np.sqrt(np.mean(np.sum(d * d, axis=1))))


def force_rms(g, o):
    return float(np.sqrt(np.mean((g.dem + g.dep - o.dem - o.dep) ** 2)))


CONFIGS = {
    "32768_waters": (lambda: systems.water_box(32768, 99.3, seed=0), (108, 108, 108)),
    "ion_solution": (lambda: systems.ion_solution(seed=0), (72, 72, 72)),
}


@pytest.fixture(scope="module", params=list(CONFIGS))
def case(request):
    make, grid = CONFIGS[request.param]
    s = make()
    o = oracle.forward(s, Settings(nfft=grid, precision=FP64), tol=1e-10)
    return request.param, s, grid, o


def test_fp64_path_matches_oracle(case):
    name, s, grid, o = case
    g = run(s, Settings(nfft=grid, precision=FP64, poleps=1e-8))
    assert rel(g.em, o.em) < 1e-10, (name, g.em, o.em)
    assert rel(g.ep, o.ep) < 1e-8, (name, g.ep, o.ep)
    assert dipole_rms_debye(g, o) < 1e-7, name
    assert np.abs(g.dem + g.dep - o.dem - o.dep).max() < 1e-5, name


def test_mixed_path_meets_the_target_against_oracle(case):
    name, s, grid, o = case
    g = run(s, Settings(nfft=grid, precision=MIXED))
    assert g.pcg_eps <= 1e-6
    assert rel(g.em, o.em) < 1e-6, (name, rel(g.em, o.em))
    assert rel(g.ep, o.ep) < 1e-6, (name, rel(g.ep, o.ep))
    assert force_rms(g, o) < 1e-4, (name, force_rms(g, o))
    assert dipole_rms_debye(g, o) < 1e-5, (name, dipole_rms_debye(g, o))


def test_32768_waters_grid_shift_invariance():
    """A shift by whole PME grid spacings changes no B-spline weight and no
    pair distance: the FP64 energies are unchanged to round-off (an arbitrary
    shift changes the PME interpolation error, ~1e-5 relative at this grid)."""
    s = systems.water_box(32768, 99.3, seed=0)
    st = Settings(nfft=(108, 108, 108), precision=FP64)
    g = run(s, st)
    s.xyz = s.xyz + np.array([3.0, -2.0, 5.0]) * (99.3 / 108)
    gs = run(s, st)
    assert rel(gs.em, g.em) < 1e-10 and rel(gs.ep, g.ep) < 1e-8
