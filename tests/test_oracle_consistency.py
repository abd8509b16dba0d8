"""Internal consistency of the oracle's restatement of the parts the reference
does not implement (Ewald real space, PME, self terms, induced dipoles,
polarization forces): the checks that pin it in place of golden vectors."""
import copy
import dataclasses

import numpy as np
import pytest

from oracle import oracle
from polmdqc_b200 import abi, systems
from polmdqc_b200.engine import Settings


@pytest.fixture(scope="module")
def box27():
    return systems.water_box(27, 9.32, seed=3)


def test_pme_converges_to_explicit_ewald_sum(box27):
    """PME (B-splines, order 5) -> explicit k-space sum as the grid is refined,
    for charges, dipoles and quadrupoles separately."""
    for mask in ([0], [1, 2, 3], list(range(4, 13))):
        s = copy.deepcopy(box27)
        keep = np.zeros(13, bool)
        keep[mask] = True
        s.pole = s.pole * keep
        st = Settings(aewald=0.7, nfft=(64, 64, 64), cutoff=4.6, poltyp=abi.POL_NONE)
        ek = oracle.forward(s, st, flags=abi.DO_ENERGY, kmax=9.0).em
        ep = oracle.forward(s, st, flags=abi.DO_ENERGY).em
        assert abs(ep - ek) < 2e-5 * abs(ek) + 2e-5


def test_ewald_total_independent_of_alpha():
    """With converged real-space cutoff and reciprocal sum, em does not depend on alpha."""
    s = systems.water_box(216, 18.643, seed=0)
    vals = []
    for a in (0.55, 0.6, 0.65):
        st = Settings(aewald=a, nfft=(24, 24, 24), cutoff=9.0, poltyp=abi.POL_NONE)
        vals.append(oracle.forward(s, st, flags=abi.DO_ENERGY, kmax=7.0).em)
    assert max(vals) - min(vals) < 2e-6 * abs(vals[0])


@pytest.mark.parametrize("ewald", [True, False])
def test_forces_match_finite_differences(box27, ewald):
    """Analytic em/ep gradients (real, reciprocal, self, torques, mutual dipoles)
    against central differences of the energies (the reference's testgrad
    pattern, src/md/testgrad.cpp:273-333)."""
    s = copy.deepcopy(box27)
    if not ewald:
        s.use_bounds = False
    st = (Settings(aewald=0.7, nfft=(24, 24, 24), cutoff=4.6, poleps=1e-11) if ewald
          else Settings(use_ewald=False, cutoff=100.0, poleps=1e-11))
    r = oracle.forward(s, st)
    h = 1e-5
    for (i, a) in ((0, 0), (1, 2), (40, 1), (77, 2)):
        x = s.xyz.copy()
        x[i, a] += h
        p = oracle.forward(s, st, xyz=x, flags=abi.DO_ENERGY)
        x[i, a] -= 2 * h
        m = oracle.forward(s, st, xyz=x, flags=abi.DO_ENERGY)
        assert abs((p.em - m.em) / (2 * h) - r.dem[i, a]) < 1e-6
        assert abs((p.ep - m.ep) / (2 * h) - r.dep[i, a]) < 1e-6


def test_dipoles_solve_the_linear_system(box27):
    """Converged PCG dipoles satisfy (1/alpha) u - T u = E: the direct
    polarization model gives u = alpha E exactly, and the mutual solution's
    energy is stationary (a perturbed solve changes ep at second order)."""
    st = Settings(aewald=0.7, nfft=(24, 24, 24), cutoff=4.6, poleps=1e-12)
    r = oracle.forward(box27, st)
    assert r.pcg_eps < 1e-12
    loose = oracle.forward(box27, Settings(aewald=0.7, nfft=(24, 24, 24), cutoff=4.6, poleps=1e-5), check=False)
    assert abs(loose.ep - r.ep) < 1e-3 * abs(r.ep)
    d = oracle.forward(box27, Settings(aewald=0.7, nfft=(24, 24, 24), cutoff=4.6, poltyp=abi.POL_DIRECT))
    assert d.pcg_iters == 0 and d.ep != 0


def test_sparse_preconditioner_same_solution_fewer_iterations():
    """pcgprec (the reference's default, src/md/kpolar.cpp:84): the sparse
    preconditioner over pairs within usolvcut (4.5 A, src/md/cutoffs.cpp:61)
    converges to the same dipoles as the diagonal one in fewer iterations."""
    s = systems.water_box(216, 18.643, seed=0)
    base = Settings(nfft=(24, 24, 24), precision=abi.PREC_FP64, poleps=1e-9)
    jac = oracle.forward(s, dataclasses.replace(base, pcg_prec=False))
    spr = oracle.forward(s, dataclasses.replace(base, pcg_prec=True))
    assert spr.pcg_iters < jac.pcg_iters
    assert np.abs(spr.uind - jac.uind).max() < 1e-8
    assert np.abs(spr.uinp - jac.uinp).max() < 1e-8
    assert abs(spr.ep - jac.ep) < 1e-9 * abs(jac.ep)
    # at the production tolerance (1e-6 D) too
    j6 = oracle.forward(s, dataclasses.replace(base, poleps=1e-6, pcg_prec=False))
    s6 = oracle.forward(s, dataclasses.replace(base, poleps=1e-6, pcg_prec=True))
    assert s6.pcg_iters < j6.pcg_iters


def _strained(s, a, b, h):
    """Copy of s with coordinates (and, for a diagonal strain of a periodic
    box, the box edge) deformed by 1 + h e_a e_b^T."""
    t = copy.deepcopy(s)
    E = np.eye(3)
    E[a, b] += h
    t.xyz = s.xyz @ E.T
    if s.use_bounds:
        t.box = s.box.copy()
        t.box[a] *= 1 + h
    return t


@pytest.mark.parametrize("case", ["ewald_mutual", "ewald_direct", "ewald_opt", "periodic_bare"])
def test_virial_is_the_strain_derivative(box27, case):
    """CalcMode::Virial: W = dE/d(strain) of em + ep, with the box deformed
    with the coordinates (PME grid and alpha fixed).  An orthogonal box admits
    diagonal strains only, so the off-diagonal part is pinned by the rotation
    invariance of the energy: the unsymmetrised W has no antisymmetric part."""
    s = copy.deepcopy(box27)
    s.box = np.array([9.32, 9.9, 10.4, 90.0, 90.0, 90.0])
    st = {"ewald_mutual": Settings(aewald=0.7, nfft=(24, 25, 27), cutoff=4.6, poleps=1e-11),
          "ewald_direct": Settings(aewald=0.7, nfft=(24, 25, 27), cutoff=4.6, poltyp=abi.POL_DIRECT),
          "ewald_opt": Settings(aewald=0.7, nfft=(24, 25, 27), cutoff=4.6, poltyp=abi.POL_OPT, opt_order=3),
          "periodic_bare": Settings(use_ewald=False, cutoff=4.6, poleps=1e-11)}[case]
    W = oracle.forward(s, st, flags=abi.DO_ENERGY | abi.DO_VIRIAL, raw_virial=True).vir
    h = 1e-5
    for a in range(3):
        p = oracle.forward(_strained(s, a, a, h), st, flags=abi.DO_ENERGY)
        m = oracle.forward(_strained(s, a, a, -h), st, flags=abi.DO_ENERGY)
        fd = (p.em + p.ep - m.em - m.ep) / (2 * h)
        assert abs(W[a, a] - fd) < 1e-8 * np.abs(W).max()
    assert np.abs(W - W.T).max() < 1e-9 * np.abs(W).max()
    sym = oracle.forward(s, st, flags=abi.DO_ENERGY | abi.DO_VIRIAL).vir
    np.testing.assert_allclose(sym, 0.5 * (W + W.T), rtol=0, atol=1e-12 * np.abs(W).max())


def test_virial_shear_components_without_a_box(box27):
    """Off-diagonal strains of an open (non-periodic) cluster, all terms."""
    s = copy.deepcopy(box27)
    s.use_bounds = False
    st = Settings(use_ewald=False, cutoff=100.0, poleps=1e-11)
    W = oracle.forward(s, st, flags=abi.DO_ENERGY | abi.DO_VIRIAL, raw_virial=True).vir
    h = 1e-5
    for (a, b) in ((0, 1), (0, 2), (1, 2), (2, 0)):
        p = oracle.forward(_strained(s, a, b, h), st, flags=abi.DO_ENERGY)
        m = oracle.forward(_strained(s, a, b, -h), st, flags=abi.DO_ENERGY)
        assert abs(W[a, b] - (p.em + p.ep - m.em - m.ep) / (2 * h)) < 1e-8 * np.abs(W).max()


@pytest.mark.parametrize("order", [1, 4, 6])
def test_opt_forces_match_finite_differences(box27, order):
    """OPT (extrapolated perturbation theory, coefficients of the reference's
    kpolar): u = sum_k copm_k u^(k) is not a stationary point, so its forces
    carry the dipole-dipole terms of every pair of perturbation orders; they
    must equal central differences of ep."""
    st = Settings(aewald=0.7, nfft=(24, 24, 24), cutoff=4.6, poltyp=abi.POL_OPT, opt_order=order)
    r = oracle.forward(box27, st)
    assert r.pcg_iters == order
    h = 1e-5
    for (i, a) in ((0, 0), (1, 2), (40, 1)):
        x = box27.xyz.copy()
        x[i, a] += h
        p = oracle.forward(box27, st, xyz=x, flags=abi.DO_ENERGY)
        x[i, a] -= 2 * h
        m = oracle.forward(box27, st, xyz=x, flags=abi.DO_ENERGY)
        assert abs((p.ep - m.ep) / (2 * h) - r.dep[i, a]) < 1e-6


def test_opt_approaches_the_mutual_solution(box27):
    """Higher OPT orders land nearer the converged mutual solution: OPT1 is
    8% off in ep here, OPT4 (the reference's default OPT) 5e-5, as the
    extrapolation is designed to do."""
    mu = oracle.forward(box27, Settings(aewald=0.7, nfft=(24, 24, 24), cutoff=4.6, poleps=1e-10))
    errs = []
    for order in (1, 2, 4, 6):
        o = oracle.forward(box27, Settings(aewald=0.7, nfft=(24, 24, 24), cutoff=4.6, poltyp=abi.POL_OPT,
                                           opt_order=order))
        errs.append(abs(o.ep - mu.ep) / abs(mu.ep))
    assert errs[2] < 1e-3 and errs[3] < 1e-2
    assert max(errs[1:]) < errs[0]


TRICLINIC = np.array([9.9, 10.1, 10.4, 86.0, 95.0, 92.0])


def _rows(box):
    """Lattice rows of a (a, b, c, alpha, beta, gamma) cell, a along x and b
    in the xy plane (the reference's lattice, src/md/lattice.cpp:122-140)."""
    a, b, c = box[:3]
    al, be, ga = np.radians(box[3:])
    bterm = (np.cos(al) - np.cos(be) * np.cos(ga)) / np.sin(ga)
    return np.array([[a, 0, 0], [b * np.cos(ga), b * np.sin(ga), 0],
                     [c * np.cos(be), c * bterm, c * np.sqrt(np.sin(be) ** 2 - bterm ** 2)]])


def _box_of(rows):
    L = np.linalg.norm(rows, axis=1)
    ang = lambda u, v: np.degrees(np.arccos(np.dot(u, v) / (np.linalg.norm(u) * np.linalg.norm(v))))
    return np.array([L[0], L[1], L[2], ang(rows[1], rows[2]), ang(rows[0], rows[2]), ang(rows[0], rows[1])])


@pytest.fixture(scope="module")
def tric27(box27):
    s = copy.deepcopy(box27)
    s.box = TRICLINIC.copy()
    return s


def test_triclinic_pme_converges_to_explicit_ewald_sum(tric27):
    """PME in a triclinic cell (fractional multipoles through the inverse
    lattice, derivatives back through it) against the explicit k-space sum."""
    for mask in ([0], [1, 2, 3], list(range(4, 13))):
        s = copy.deepcopy(tric27)
        keep = np.zeros(13, bool)
        keep[mask] = True
        s.pole = s.pole * keep
        st = Settings(aewald=0.7, nfft=(64, 64, 64), cutoff=4.6, poltyp=abi.POL_NONE)
        ek = oracle.forward(s, st, flags=abi.DO_ENERGY, kmax=9.0).em
        ep = oracle.forward(s, st, flags=abi.DO_ENERGY).em
        assert abs(ep - ek) < 2e-5 * abs(ek) + 2e-5


def test_triclinic_ewald_forces_and_virial(tric27):
    """Triclinic Ewald with mutual polarization: gradients against central
    differences, and the virial's diagonal against strains of the cell (the
    strained rows keep a along x and b in the xy plane)."""
    s = tric27
    st = Settings(aewald=0.7, nfft=(24, 25, 27), cutoff=4.6, poleps=1e-11)
    r = oracle.forward(s, st, flags=abi.DO_ENERGY | abi.DO_GRADIENT | abi.DO_VIRIAL, raw_virial=True)
    h = 1e-5
    for (i, a) in ((0, 0), (40, 1), (77, 2)):
        x = s.xyz.copy()
        x[i, a] += h
        p = oracle.forward(s, st, xyz=x, flags=abi.DO_ENERGY)
        x[i, a] -= 2 * h
        m = oracle.forward(s, st, xyz=x, flags=abi.DO_ENERGY)
        assert abs((p.em - m.em) / (2 * h) - r.dem[i, a]) < 1e-6
        assert abs((p.ep - m.ep) / (2 * h) - r.dep[i, a]) < 1e-6
    W = r.vir
    rows = _rows(s.box)
    for a in range(3):
        e = []
        for sgn in (1, -1):
            E = np.eye(3)
            E[a, a] += sgn * h
            t = copy.deepcopy(s)
            t.xyz = s.xyz @ E.T
            t.box = _box_of(rows @ E.T)
            q = oracle.forward(t, st, flags=abi.DO_ENERGY)
            e.append(q.em + q.ep)
        assert abs(W[a, a] - (e[0] - e[1]) / (2 * h)) < 1e-8 * np.abs(W).max()
    assert np.abs(W - W.T).max() < 1e-9 * np.abs(W).max()


def test_triclinic_ewald_total_independent_of_alpha(tric27):
    """Real space (the reference's fractional-coordinate image), reciprocal
    space and self terms together: em does not depend on alpha."""
    vals = []
    for a in (0.8, 0.9, 1.0):
        st = Settings(aewald=a, nfft=(24, 24, 24), cutoff=4.9, poltyp=abi.POL_NONE)
        vals.append(oracle.forward(tric27, st, flags=abi.DO_ENERGY, kmax=11.0).em)
    assert max(vals) - min(vals) < 1e-6 * abs(vals[0])


@pytest.mark.parametrize("poltyp", [abi.POL_NONE, abi.POL_MUTUAL])
def test_periodic_ewald_virial_shear_components(box27, poltyp):
    """Off-diagonal virial of a periodic Ewald system: shearing the cubic cell
    (x += h y, x += h z, y += h z keep a along x and b in the xy plane) makes
    it triclinic, which the PME handles, so the shear derivative of em + ep
    pins W_xy, W_xz and W_yz directly."""
    st = Settings(aewald=0.7, nfft=(24, 24, 24), cutoff=4.6, poltyp=poltyp, poleps=1e-11)
    W = oracle.forward(box27, st, flags=abi.DO_ENERGY | abi.DO_VIRIAL).vir
    rows, h = _rows(box27.box), 1e-5
    for (a, b) in ((0, 1), (0, 2), (1, 2)):
        e = []
        for sgn in (1, -1):
            E = np.eye(3)
            E[a, b] += sgn * h
            t = copy.deepcopy(box27)
            t.xyz = box27.xyz @ E.T
            t.box = _box_of(rows @ E.T)
            q = oracle.forward(t, st, flags=abi.DO_ENERGY)
            e.append(q.em + q.ep)
        assert abs(W[a, b] - (e[0] - e[1]) / (2 * h)) < 1e-8 * np.abs(W).max()


def test_pcg_dipoles_equal_a_dense_solve(box27):
    """The PCG solution of (1/alpha - T) u = E against Gaussian elimination on
    the explicit 3N x 3N operator (columns from the field of unit dipoles),
    for both right-hand sides, with Ewald."""
    from polmdqc_b200.engine import Params
    st = Settings(aewald=0.7, nfft=(24, 24, 24), cutoff=4.6)
    P = Params(box27, st)
    n3 = 3 * box27.n
    T = np.zeros((n3, n3))
    for j in range(n3):
        e = np.zeros(n3)
        e[j] = 1.0
        T[:, j] = oracle.dipole_field(box27, st, e.reshape(-1, 3), params=P).reshape(-1)
    assert np.abs(T - T.T).max() < 1e-10 * np.abs(T).max()       # symmetric operator
    alpha = np.repeat(box27.polarity, 3)
    direct = oracle.forward(box27, dataclasses.replace(st, poltyp=abi.POL_DIRECT))
    mutual = oracle.forward(box27, dataclasses.replace(st, poleps=1e-12))
    A = np.diag(1.0 / alpha) - T
    for u_direct, u_pcg in ((direct.uind, mutual.uind), (direct.uinp, mutual.uinp)):
        E = u_direct.reshape(-1) / alpha                             # direct dipoles are alpha E
        u = np.linalg.solve(A, E)
        assert np.abs(u - u_pcg.reshape(-1)).max() < 1e-10


def test_ewald_dimer_approaches_the_isolated_reference():
    """The reference's water dimer (test/amoeba.h, isolated, its em golden)
    in growing periodic cubes with Ewald: the difference is the periodic
    images' dipolar energy, shrinking as 1/V (tinfoil boundary)."""
    from conftest import golden, ref_dump, ref_fixture
    d = ref_dump(ref_fixture("amoeba", "water09.xyz"))
    s = systems.from_dump(d)
    em_isolated = golden("ref_tests.json")["amoeba1"]["em"]
    diffs = []
    for L, K in ((40.0, 48), (60.0, 64), (90.0, 96)):
        t = copy.deepcopy(s)
        t.use_bounds = True
        t.box = np.array([L, L, L, 90.0, 90.0, 90.0])
        t.xyz = t.xyz - t.xyz.mean(0) + L / 2
        st = Settings(aewald=0.25, nfft=(K,) * 3, cutoff=min(25.0, L / 2 - 1), poltyp=abi.POL_NONE)
        diffs.append((L, oracle.forward(t, st, flags=abi.DO_ENERGY).em - em_isolated))
    vol_scaled = [dv * L ** 3 for L, dv in diffs]
    assert abs(diffs[-1][1]) < 3e-4
    assert max(vol_scaled) - min(vol_scaled) < 0.1 * abs(vol_scaled[0])
