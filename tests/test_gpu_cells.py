"""Ewald and PME in the truncated octahedron and the rhombic dodecahedron,
the two non-prism cells of the reference's image() (src/md/image.cpp:92-121).

A truncated octahedron of box length L is the cell of the cube's lattice
plus its body centre, a rhombic dodecahedron the cell of the L x L x sqrt(2) L
prism's lattice plus its centre.  So the same periodic system written as the
orthogonal prism with two copies of the cell (`systems.doubled_prism`) has
exactly twice the cell's energies, and on each copy the cell's forces,
dipoles and, halved, its virial.  The FP64 oracle runs that prism (its
orthogonal Ewald and PME, converged to 1e-10 D); the GPU runs the cell
itself (minimum image of the cell in real space, the prism's PME grid with
the odd reciprocal vectors removed).  Both shapes, FP64 and mixed, mutual
polarization with the sparse preconditioner, cutoff 7 A.

Bounds: FP64 em 1e-10 and ep 1e-8 relative, induced dipoles 1e-7 D RMS,
gradients 1e-6 kcal/mol/A, virial 1e-7 of its largest entry; mixed em and
ep 1e-6 relative, force RMS 1e-4 kcal/mol/A, dipoles 1e-5 D RMS.
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
SHAPES = {"octahedron": (abi.CELL_OCTAHEDRON, (24, 24, 24)),
          "dodecahedron": (abi.CELL_DODECAHEDRON, (24, 24, 36))}


@pytest.fixture(scope="module", params=list(SHAPES))
def case(request):
    shape, grid = SHAPES[request.param]
    s = systems.water_cell(shape, seed=2)
    o = oracle.forward(systems.doubled_prism(s), Settings(nfft=grid, precision=FP64), tol=1e-10,
                       flags=ALL | abi.DO_VIRIAL)
    return request.param, s, grid, o


def run(s, st, flags=ALL):
    e = Engine(s, st)
    try:
        return e.forward(flags)
    finally:
        e.close()


def first(a, n):
    return np.asarray(a).reshape(-1, 3)[:n]


def dipole_rms(g, o, n):
    d = np.concatenate([g.uind - first(o.uind, n), g.uinp - first(o.uinp, n)])
    return DEBYE * float(np.sqrt(np.mean(np.sum(d * d, axis=1))))


def test_fp64_cell_is_half_the_doubled_prism(case):
    name, s, grid, o = case
    n = s.n
    g = run(s, Settings(nfft=grid, precision=FP64, poleps=1e-8), ALL | abi.DO_VIRIAL)
    assert abs(g.em - o.em / 2) < 1e-10 * abs(o.em / 2), (name, g.em, o.em / 2)
    assert abs(g.ep - o.ep / 2) < 1e-8 * abs(o.ep / 2), (name, g.ep, o.ep / 2)
    assert dipole_rms(g, o, n) < 1e-7, name
    np.testing.assert_allclose(g.dem, first(o.dem, n), atol=1e-6, rtol=0)
    np.testing.assert_allclose(g.dep, first(o.dep, n), atol=1e-6, rtol=0)
    v = np.asarray(o.vir).reshape(3, 3) / 2
    np.testing.assert_allclose(g.vir, v, atol=1e-7 * np.abs(v).max(), rtol=0)


def test_mixed_cell_meets_the_target(case):
    name, s, grid, o = case
    n = s.n
    g = run(s, Settings(nfft=grid, precision=MIXED))
    assert g.pcg_eps <= 1e-6
    assert abs(g.em - o.em / 2) < 1e-6 * abs(o.em / 2), name
    assert abs(g.ep - o.ep / 2) < 1e-6 * abs(o.ep / 2), name
    frms = float(np.sqrt(np.mean((g.dem + g.dep - first(o.dem, n) - first(o.dep, n)) ** 2)))
    assert frms < 1e-4, (name, frms)
    assert dipole_rms(g, o, n) < 1e-5, name
