"""The induced-dipole predictor (amg_set_predictor; the reference's uprior
module, include/md/uprior.h, which it declares and leaves off).

A short smooth trajectory of the 216-water box (every atom moves along its
own seeded quadratic path, 0.004 A per step), evaluated step by step by one
context with the predictor and one without.  Once the predictor's history is
full (after AMG_PRED_STEPS evaluations) the PCG starts from the extrapolated
dipoles: the results agree with the unpredicted ones within the convergence
(FP64, poleps 1e-9 D: em 1e-12 and ep 1e-9 relative, dipoles 1e-8 D RMS)
while the PCG takes fewer iterations.  The mixed path (graph replays) keeps
its targets against the unpredicted FP64 results.
"""
import numpy as np
import pytest

from polmdqc_b200 import abi, systems
from polmdqc_b200.engine import Engine, Settings
from polmdqc_b200.prm import DEBYE

pytestmark = pytest.mark.gpu

ALL = abi.DO_ENERGY | abi.DO_GRADIENT | abi.DO_DIPOLES
STEPS = 12


def trajectory():
    s = systems.water_box(216, 18.643, seed=0)
    rng = np.random.default_rng(9)
    v = rng.standard_normal(s.xyz.shape) * 0.004
    a = rng.standard_normal(s.xyz.shape) * 0.0004
    return s, [s.xyz + v * t + 0.5 * a * t * t for t in range(STEPS)]


def run(s, frames, st, kind):
    e = Engine(s, st)
    out = []
    try:
        if kind is not None:
            e.set_predictor(kind)
        for x in frames:
            e.set_coords(x)
            out.append(e.forward(ALL))
    finally:
        e.close()
    return out


def dipole_rms(g, o):
    d = np.concatenate([g.uind - o.uind, g.uinp - o.uinp])
    return DEBYE * float(np.sqrt(np.mean(np.sum(d * d, axis=1))))


@pytest.fixture(scope="module")
def plain():
    s, frames = trajectory()
    st = Settings(nfft=(24, 24, 24), precision=abi.PREC_FP64, poleps=1e-9)
    return s, frames, run(s, frames, st, None)


@pytest.mark.parametrize("kind", [abi.PRED_GEAR, abi.PRED_ASPC])
def test_predictor_keeps_results_and_saves_iterations(plain, kind):
    s, frames, ref = plain
    st = Settings(nfft=(24, 24, 24), precision=abi.PREC_FP64, poleps=1e-9)
    got = run(s, frames, st, kind)
    for g, o in zip(got, ref):
        assert abs(g.em - o.em) < 1e-12 * abs(o.em)
        assert abs(g.ep - o.ep) < 1e-9 * abs(o.ep)
        assert dipole_rms(g, o) < 1e-8
    # the first AMG_PRED_STEPS evaluations start from the direct dipoles
    assert [g.pcg_iters for g in got[:6]] == [o.pcg_iters for o in ref[:6]]
    it_pred = sum(g.pcg_iters for g in got[6:])
    it_plain = sum(o.pcg_iters for o in ref[6:])
    assert it_pred < 0.75 * it_plain, (it_pred, it_plain)


def test_mixed_path_with_predictor(plain):
    s, frames, ref = plain
    got = run(s, frames, Settings(nfft=(24, 24, 24), precision=abi.PREC_MIXED), abi.PRED_ASPC)
    for g, o in zip(got, ref):
        assert g.pcg_eps <= 1e-6
        assert abs(g.em - o.em) < 1e-6 * abs(o.em) and abs(g.ep - o.ep) < 1e-6 * abs(o.ep)
        assert float(np.sqrt(np.mean((g.dem + g.dep - o.dem - o.dep) ** 2))) < 1e-4
    assert sum(g.pcg_iters for g in got[6:]) < sum(g.pcg_iters for g in got[:6])


def test_unknown_predictor_is_refused():
    s = systems.water_box(8, 12.0, seed=0)
    e = Engine(s, Settings(nfft=(16, 16, 16), cutoff=5.0))
    try:
        with pytest.raises(Exception, match="BAD_ARG"):
            e.set_predictor(7)
    finally:
        e.close()
