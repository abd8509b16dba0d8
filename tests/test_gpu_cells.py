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


LARGE = {"octahedron": (abi.CELL_OCTAHEDRON, (48, 48, 48)),
         "dodecahedron": (abi.CELL_DODECAHEDRON, (48, 48, 64))}


@pytest.mark.parametrize("name", list(LARGE))
def test_centred_cell_lists_at_size(name):
    """A 43 A box of liquid density (1,372 and 2,058 waters): the neighbour
    lists come from the cell grid of the enclosing prism (6 cells per axis, 8
    along the dodecahedron's sqrt(2) L), searching
    the 27 cells around each cell and the 27 around the cell half a prism away
    (the centring translation), instead of the all-pairs search.  Without
    Ewald the oracle runs the cell itself (the reference's image(), every
    pair): the pair count is exact, FP64 energies and gradients agree.  With
    Ewald the oracle runs the doubled prism, as above."""
    shape, grid = LARGE[name]
    s = systems.water_cell(shape, L=43.0, seed=4, per_edge=14)
    flags = ALL | abi.DO_ANALYSIS
    st = Settings(use_ewald=False, precision=FP64, poleps=1e-8)
    o = oracle.forward(s, st, tol=1e-11, flags=flags)
    g = run(s, st, flags)
    assert g.nem == o.nem and o.nem > 0, (name, g.nem, o.nem)
    assert abs(g.em - o.em) < 1e-10 * abs(o.em) and abs(g.ep - o.ep) < 1e-8 * abs(o.ep), name
    np.testing.assert_allclose(g.dem, o.dem, atol=1e-8, rtol=0)
    np.testing.assert_allclose(g.dep, o.dep, atol=1e-5, rtol=0)  # dipoles converged to 1e-8 D

    n = s.n
    o2 = oracle.forward(systems.doubled_prism(s), Settings(nfft=grid, precision=FP64), tol=1e-10, flags=ALL)
    g64 = run(s, Settings(nfft=grid, precision=FP64, poleps=1e-8))
    assert abs(g64.em - o2.em / 2) < 1e-10 * abs(o2.em / 2), (name, g64.em, o2.em / 2)
    assert abs(g64.ep - o2.ep / 2) < 1e-8 * abs(o2.ep / 2), (name, g64.ep, o2.ep / 2)
    assert dipole_rms(g64, o2, n) < 1e-7, name
    np.testing.assert_allclose(g64.dem, first(o2.dem, n), atol=1e-6, rtol=0)
    gm = run(s, Settings(nfft=grid, precision=MIXED))
    assert abs(gm.em - o2.em / 2) < 1e-6 * abs(o2.em / 2) and abs(gm.ep - o2.ep / 2) < 1e-6 * abs(o2.ep / 2), name
    frms = float(np.sqrt(np.mean((gm.dem + gm.dep - first(o2.dem, n) - first(o2.dep, n)) ** 2)))
    assert frms < 1e-4, (name, frms)
