"""Parity of the CUDA path (called through the C ABI) with the reference's
golden vectors and with the FP64 oracle.

Tolerances:
  FP64 path vs oracle/reference: energies 1e-10 relative (reference goldens
    at their own eps, 1e-10 / 1e-8), gradients 1e-8 absolute without
    polarization; with polarization the PCG tolerance sets the floor
    (dipoles converged to 1e-8 D: gradients 1e-5, ep 1e-8 relative).
  mixed path (FP32 pairs/grids): |em - em_ref| / |em_ref| < 1e-6,
    |ep - ep_ref| / |ep_ref| < 1e-6, force RMS < 1e-4 kcal/mol/A, as the
    accuracy target of the mixed-precision design states.
"""
import numpy as np
import pytest

from conftest import golden, ref_dump, ref_fixture
from oracle import oracle
from polmdqc_b200 import abi, systems
from polmdqc_b200.engine import AmgError, Engine, Settings

pytestmark = pytest.mark.gpu

FP64, MIXED = abi.PREC_FP64, abi.PREC_MIXED
ALL = abi.DO_ENERGY | abi.DO_GRADIENT | abi.DO_DIPOLES


def rel(a, b):
    return abs(a - b) / max(abs(b), 1e-300)


def frms(g, o):
    return float(np.sqrt(np.mean((g.dem + g.dep - o.dem - o.dep) ** 2)))


def run(s, st, flags=ALL):
    e = Engine(s, st)
    try:
        return e.forward(flags)
    finally:
        e.close()


# ---------------------------------------------------------------- reference goldens
@pytest.mark.parametrize("prec", [FP64, MIXED])
def test_water_dimer_golden(prec):
    """test/amoeba.cpp amoeba-1/-2 through the C ABI (non-Ewald multipoles)."""
    g = golden("ref_tests.json")
    d = ref_dump(ref_fixture("amoeba", "water09.xyz"))
    s = systems.from_dump(d)
    st = Settings(use_ewald=False, cutoff=d["mpolecut"], poltyp=abi.POL_NONE, precision=prec)
    r = run(s, st, abi.DO_ENERGY | abi.DO_GRADIENT | abi.DO_ANALYSIS)
    a1, a2 = g["amoeba1"], g["amoeba2"]
    tol_e = a1["eps"] if prec == FP64 else 2e-6 * abs(a1["em"])
    tol_g = a2["eps1"] if prec == FP64 else 1e-4
    assert r.nem == a1["nem"]
    assert abs(r.em - a1["em"]) < tol_e
    assert abs(r.einter - a1["einter"]) < tol_e
    np.testing.assert_allclose(r.aem, a1["aem"], atol=tol_e, rtol=0)
    np.testing.assert_allclose(r.dem.reshape(-1), a2["dem"], atol=tol_g, rtol=0)


def test_waterbox30_orthogonal_golden():
    """test/bounds.cpp bounds-1: periodic 2,700 atoms, cutoff 9, em/nem/einter."""
    g = golden("ref_tests.json")["bounds1"]
    d = ref_dump(ref_fixture("bounds", "waterbox30.xyz"), ref_fixture("bounds", "orthogonal.key"))
    s = systems.from_dump(d)
    st = Settings(use_ewald=False, cutoff=d["mpolecut"], poltyp=abi.POL_NONE, precision=FP64)
    r = run(s, st, abi.DO_ENERGY | abi.DO_GRADIENT | abi.DO_ANALYSIS)
    assert r.nem == g["nem"]
    assert abs(r.em - g["em"]) < g["eps"]
    assert abs(r.einter - g["einter"]) < g["eps"]
    np.testing.assert_allclose(r.dem.reshape(-1), d["dem"], atol=1e-8, rtol=0)


@pytest.mark.parametrize("prec", [FP64, MIXED])
@pytest.mark.parametrize("case,shape", [("bounds2", "monoclinic"), ("bounds3", "triclinic"),
                                        ("bounds4", "octahedron"), ("bounds5", "dodecahedron")])
def test_waterbox30_cell_shapes_golden(case, shape, prec):
    """test/bounds.cpp bounds-2..5: monoclinic, triclinic, truncated
    octahedron and rhombic dodecahedron cells through the C ABI (the
    reference's image(), one candidate cell and an FP64 list decision)."""
    g = golden("ref_tests.json")[case]
    d = ref_dump(ref_fixture("bounds", "waterbox30.xyz"), ref_fixture("bounds", shape + ".key"))
    s = systems.from_dump(d)
    st = Settings(use_ewald=False, cutoff=d["mpolecut"], poltyp=abi.POL_NONE, precision=prec)
    r = run(s, st, abi.DO_ENERGY | abi.DO_GRADIENT | abi.DO_ANALYSIS)
    assert r.nem == g["nem"]
    if prec == FP64:
        assert abs(r.em - g["em"]) < g["eps"]
        assert abs(r.einter - g["einter"]) < g["eps"]
        np.testing.assert_allclose(r.dem.reshape(-1), d["dem"], atol=1e-8, rtol=0)
    else:
        # the 30 A water box put into these cells brings image atoms nearly on
        # top of each other (per-atom energies up to 3e4 kcal/mol): FP32
        # coordinate differences carry the error, bounded against the sum of
        # the per-atom energy magnitudes
        scale = np.abs(r.aem).sum()
        assert abs(r.em - g["em"]) < 1e-4 * scale
        assert abs(r.einter - g["einter"]) < 1e-4 * scale


def test_ewald_in_the_reference_octahedron():
    """The reference's bounds-4 input (its waterbox30 coordinates read as a
    truncated octahedron of box length 30) with Ewald, cutoff 9: em and its
    gradient are half those of the same system written as the enclosing cube
    with two copies of the cell, which the oracle evaluates with its
    orthogonal Ewald and PME on the same 32^3 grid."""
    d = ref_dump(ref_fixture("bounds", "waterbox30.xyz"), ref_fixture("bounds", "octahedron.key"))
    s = systems.from_dump(d)
    st = Settings(nfft=(32, 32, 32), cutoff=9.0, poltyp=abi.POL_NONE, precision=FP64)
    g = run(s, st, abi.DO_ENERGY | abi.DO_GRADIENT)
    o = oracle.forward(systems.doubled_prism(s), st, flags=abi.DO_ENERGY | abi.DO_GRADIENT)
    assert abs(g.em - o.em / 2) < 1e-10 * abs(o.em / 2), (g.em, o.em / 2)
    # the cube's coordinates read as an octahedron bring image atoms nearly on
    # top of each other (gradients up to 2e6 kcal/mol/A): relative bound
    od = o.dem.reshape(-1, 3)[:s.n]
    np.testing.assert_allclose(g.dem, od, atol=1e-10 * np.abs(od).max(), rtol=0)


def test_ewald_in_the_reference_dodecahedron_is_refused():
    """The reference's bounds-5 dodecahedron has c = sqrt(2) a (its unitcell()),
    for which its minimum image is no lattice: Ewald returns UNSUPPORTED
    (the non-Ewald bounds-5 golden above uses the image as it stands)."""
    d = ref_dump(ref_fixture("bounds", "waterbox30.xyz"), ref_fixture("bounds", "dodecahedron.key"))
    s = systems.from_dump(d)
    with pytest.raises(AmgError, match="UNSUPPORTED"):
        run(s, Settings(nfft=(32, 32, 48), cutoff=9.0, poltyp=abi.POL_NONE))


@pytest.mark.parametrize("prec", [FP64, MIXED])
@pytest.mark.parametrize("box", [(18.9, 19.3, 19.6, 90.0, 97.0, 90.0), (18.9, 19.3, 19.6, 84.0, 97.0, 93.0)])
def test_ewald_in_prism_cells_matches_oracle(w216, box, prec):
    """Monoclinic and triclinic cells with Ewald and mutual polarization: the
    pair kernels' cell-image instances, the PME through the inverse lattice
    (fractional multipoles, stencils, derivative transform, influence
    function on the general reciprocal vectors) and the virial."""
    import copy
    s = copy.deepcopy(w216)
    s.box = np.array(box)
    flags = ALL | abi.DO_VIRIAL
    o = oracle.forward(s, Settings(nfft=(24, 24, 24), precision=FP64), tol=1e-11, flags=flags)
    g = run(s, Settings(nfft=(24, 24, 24), precision=prec, poleps=1e-8 if prec == FP64 else 1e-6), flags)
    if prec == FP64:
        assert rel(g.em, o.em) < 1e-10 and rel(g.ep, o.ep) < 1e-8
        assert np.abs(g.dem - o.dem).max() < 1e-8 and np.abs(g.dep - o.dep).max() < 1e-5
        assert np.abs(g.vir - o.vir).max() < 1e-7 * np.abs(o.vir).max()
    else:
        assert rel(g.em, o.em) < 1e-6 and rel(g.ep, o.ep) < 1e-6
        assert frms(g, o) < 1e-4
        assert np.abs(g.vir - o.vir).max() < 1e-5 * np.abs(o.vir).max()


@pytest.mark.parametrize("prec", [FP64, MIXED])
@pytest.mark.parametrize("box", [(28.3, 28.7, 29.0, 90.0, 97.0, 90.0), (28.3, 28.7, 29.0, 84.0, 97.0, 93.0)])
def test_prism_cell_lists_at_size(box, prec):
    """729 waters in a monoclinic and a triclinic cell wide enough for 3
    lattice cells per axis at a 7 A cutoff: the neighbour lists come from the
    cell grid of the lattice's parallelepipeds (every pair decided by the
    cell's FP64 image) instead of the all-pairs search; energies, gradients
    and virial against the oracle, with Ewald and mutual polarization."""
    s = systems.water_box(729, 28.3, seed=4)
    s.box = np.array(box)
    flags = ALL | abi.DO_VIRIAL | abi.DO_ANALYSIS
    st = Settings(nfft=(30, 30, 30), precision=FP64)
    o = oracle.forward(s, st, tol=1e-11, flags=flags)
    g = run(s, Settings(nfft=(30, 30, 30), precision=prec, poleps=1e-8 if prec == FP64 else 1e-6), flags)
    assert g.nem == o.nem
    if prec == FP64:
        assert rel(g.em, o.em) < 1e-10 and rel(g.ep, o.ep) < 1e-8
        assert np.abs(g.dem - o.dem).max() < 1e-8 and np.abs(g.dep - o.dep).max() < 1e-5
        assert np.abs(g.vir - o.vir).max() < 1e-7 * np.abs(o.vir).max()
    else:
        assert rel(g.em, o.em) < 1e-6 and rel(g.ep, o.ep) < 1e-6
        assert frms(g, o) < 1e-4


def test_synthetic_box_matches_reference_run():
    """Seeded 216-water box: the compiled reference's em/nem/dem (non-Ewald, 7 A)."""
    d = golden("ref_water216.json")
    s = systems.water_box(216, 18.643, seed=0)
    s.xyz = np.stack([d["x"], d["y"], d["z"]], 1)
    st = Settings(use_ewald=False, cutoff=d["mpolecut"], poltyp=abi.POL_NONE, precision=FP64)
    r = run(s, st, abi.DO_ENERGY | abi.DO_GRADIENT | abi.DO_ANALYSIS | abi.DO_VIRIAL)
    assert r.nem == d["nem"]
    assert rel(r.em, d["em"]) < 1e-10
    np.testing.assert_allclose(r.dem.reshape(-1), d["dem"], atol=1e-8, rtol=0)
    # the reference's CalcMode::Virial: pair terms plus the torque share
    np.testing.assert_allclose(r.vir.reshape(-1), d["vir"], atol=1e-8 * np.abs(d["vir"]).max(), rtol=0)


# ---------------------------------------------------------------- oracle (Ewald + polarization)
@pytest.fixture(scope="module")
def w216():
    return systems.water_box(216, 18.643, seed=0)


@pytest.fixture(scope="module")
def w216_oracle(w216):
    st = Settings(nfft=(24, 24, 24), precision=FP64)
    return oracle.forward(w216, st, tol=1e-11)


def test_fp64_matches_oracle(w216, w216_oracle):
    o = w216_oracle
    g = run(w216, Settings(nfft=(24, 24, 24), precision=FP64, poleps=1e-8))
    assert rel(g.em, o.em) < 1e-10
    assert rel(g.ep, o.ep) < 1e-8
    assert np.abs(g.dem - o.dem).max() < 1e-8
    assert np.abs(g.dep - o.dep).max() < 1e-5
    assert np.abs(g.uind - o.uind).max() < 1e-7
    assert np.abs(g.uinp - o.uinp).max() < 1e-7
    assert g.pcg_eps <= 1e-8


@pytest.mark.parametrize("sparse", [False, True])
def test_preconditioners_follow_the_oracle(w216, sparse):
    """Diagonal and sparse (pcgprec, usolvcut 4.5 A) preconditioners: the
    FP64 path takes the oracle's iteration count and lands on its dipoles."""
    # converged to 1e-8 D: the GPU's final FP64 correction step (which the
    # oracle does not take) then moves ep by less than 1e-8 relative
    st = Settings(nfft=(24, 24, 24), precision=FP64, pcg_prec=sparse, poleps=1e-8)
    o = oracle.forward(w216, st)
    g = run(w216, st)
    assert g.pcg_iters == o.pcg_iters
    assert rel(g.ep, o.ep) < 1e-8
    assert np.abs(g.uind - o.uind).max() < 1e-7
    m = run(w216, Settings(nfft=(24, 24, 24), precision=MIXED, pcg_prec=sparse))
    o6 = oracle.forward(w216, Settings(nfft=(24, 24, 24), precision=FP64, pcg_prec=sparse))
    assert abs(m.pcg_iters - o6.pcg_iters) <= 1
    assert rel(m.ep, o6.ep) < 1e-6


@pytest.mark.parametrize("nfft", [(30, 25, 32), (28, 28, 28)])
def test_pme_grid_sizes_match_oracle(w216, nfft):
    """The packed complex dipole grid (d + i p) and its influence function
    on non-cubic grids and odd lengths, FP64 against the oracle."""
    st = Settings(nfft=nfft, precision=FP64, poleps=1e-8)
    o = oracle.forward(w216, st, tol=1e-11)
    g = run(w216, st)
    assert rel(g.em, o.em) < 1e-10
    assert rel(g.ep, o.ep) < 1e-8
    assert np.abs(g.dep - o.dep).max() < 1e-5
    assert np.abs(g.uind - o.uind).max() < 1e-7


@pytest.mark.parametrize("prec", [FP64, MIXED])
def test_virial_matches_oracle(w216, prec):
    """CalcMode::Virial with Ewald and mutual polarization: real-space pairs,
    torque share, the reciprocal k-space and multipole terms and the net
    charge term, summed (symmetric 3x3) and split into the em and ep parts.
    The oracle's virial is pinned to the reference (non-Ewald) and to strain
    derivatives of the energy.  Tolerances relative to max |W|: 1e-8 (FP64;
    dipoles converged to 1e-8 D), 1e-5 (mixed)."""
    st = Settings(nfft=(24, 24, 24), precision=prec, poleps=1e-8 if prec == FP64 else 1e-6)
    flags = ALL | abi.DO_VIRIAL
    o = oracle.forward(w216, Settings(nfft=(24, 24, 24), precision=FP64), tol=1e-11, flags=flags)
    om = oracle.forward(w216, Settings(nfft=(24, 24, 24), precision=FP64, poltyp=abi.POL_NONE),
                        flags=abi.DO_ENERGY | abi.DO_VIRIAL)
    e = Engine(w216, st)
    try:
        g = e.forward(flags)
        vm, vp = e.virial_parts()
    finally:
        e.close()
    scale = np.abs(o.vir).max()
    tol = 1e-8 if prec == FP64 else 1e-5
    err, err_m = np.abs(g.vir - o.vir).max() / scale, np.abs(vm - om.vir).max() / scale
    print(f"virial prec={prec} max|W|={scale:.4g} err={err:.3g} em-part err={err_m:.3g}")
    assert np.allclose(g.vir, g.vir.T, rtol=0, atol=1e-12 * scale)
    assert err < tol and err_m < tol
    np.testing.assert_allclose(vm + vp, g.vir, rtol=0, atol=1e-12 * scale)
    # Virial mode implies the gradient
    assert np.abs(g.dem - o.dem).max() < (1e-8 if prec == FP64 else 1e-3)


@pytest.mark.parametrize("prec,order", [(FP64, 4), (FP64, 1), (MIXED, 4)])
def test_opt_polarization_matches_oracle(w216, prec, order):
    """OPT (extrapolated perturbation theory, the reference's kpolar
    coefficients): orders u^(k) by repeated dipole-field applications, their
    mix, and the forces with the dipole-dipole terms between every pair of
    orders (real, scaled and reciprocal), plus the virial."""
    st = Settings(nfft=(24, 24, 24), precision=prec, poltyp=abi.POL_OPT, opt_order=order)
    flags = ALL | abi.DO_VIRIAL
    o = oracle.forward(w216, Settings(nfft=(24, 24, 24), precision=FP64, poltyp=abi.POL_OPT, opt_order=order),
                       flags=flags)
    g = run(w216, st, flags)
    tol = 1e-10 if prec == FP64 else 1e-6
    assert g.pcg_iters == order
    assert rel(g.em, o.em) < tol and rel(g.ep, o.ep) < tol
    assert np.abs(g.uind - o.uind).max() < (1e-10 if prec == FP64 else 1e-5)
    if prec == FP64:
        assert np.abs(g.dep - o.dep).max() < 1e-8
    else:
        assert frms(g, o) < 1e-4
    assert np.abs(g.vir - o.vir).max() < (1e-8 if prec == FP64 else 1e-5) * np.abs(o.vir).max()


def test_virial_non_ewald_polarization_matches_oracle():
    s = systems.water_box(64, 12.4, seed=5)
    st = Settings(use_ewald=False, cutoff=6.0, precision=FP64, poleps=1e-9)
    o = oracle.forward(s, st, tol=1e-11, flags=ALL | abi.DO_VIRIAL)
    g = run(s, st, ALL | abi.DO_VIRIAL)
    assert np.abs(g.vir - o.vir).max() < 1e-7 * np.abs(o.vir).max()


def test_mixed_meets_accuracy_target(w216, w216_oracle):
    o = w216_oracle
    g = run(w216, Settings(nfft=(24, 24, 24), precision=MIXED))
    assert rel(g.em, o.em) < 1e-6
    assert rel(g.ep, o.ep) < 1e-6
    assert frms(g, o) < 1e-4
    assert g.pcg_eps <= 1e-6


def test_multipoles_only_and_direct_polarization(w216):
    for pol in (abi.POL_NONE, abi.POL_DIRECT):
        st = Settings(nfft=(24, 24, 24), precision=FP64, poltyp=pol)
        o = oracle.forward(w216, st)
        g = run(w216, st)
        assert rel(g.em, o.em) < 1e-10
        if pol == abi.POL_DIRECT:
            assert rel(g.ep, o.ep) < 1e-10
            assert np.abs(g.dep - o.dep).max() < 1e-8
        assert np.abs(g.dem - o.dem).max() < 1e-8


def test_non_ewald_polarization_matches_oracle():
    """Reference mode (no Ewald, finite cutoff) with mutual polarization."""
    s = systems.water_box(64, 12.4, seed=5)
    st = Settings(use_ewald=False, cutoff=6.0, precision=FP64, poleps=1e-9)
    o = oracle.forward(s, st, tol=1e-11)
    g = run(s, st)
    assert rel(g.em, o.em) < 1e-10
    assert rel(g.ep, o.ep) < 1e-8
    assert np.abs(g.dep - o.dep).max() < 1e-5


@pytest.mark.parametrize("prec", [FP64, MIXED])
def test_ion_solution_matches_oracle(prec):
    """amoebabio18 waters + Na+/Cl- (frame-less sites, large polarizability)."""
    s = systems.ion_solution(n_waters=250, n_pairs=3, box_len=20.0, seed=4)
    st = Settings(nfft=(25, 25, 25), precision=FP64)
    o = oracle.forward(s, st, tol=1e-11)
    g = run(s, Settings(nfft=(25, 25, 25), precision=prec, poleps=1e-8 if prec == FP64 else 1e-6))
    if prec == FP64:
        assert rel(g.em, o.em) < 1e-10 and rel(g.ep, o.ep) < 1e-8
        assert np.abs(g.dem + g.dep - o.dem - o.dep).max() < 1e-5
    else:
        assert rel(g.em, o.em) < 1e-6 and rel(g.ep, o.ep) < 1e-6
        assert frms(g, o) < 1e-4


def test_gradients_match_finite_differences():
    """GPU FP64 gradients vs central differences of GPU energies."""
    s = systems.water_box(27, 9.32, seed=3)
    st = Settings(aewald=0.7, nfft=(24, 24, 24), cutoff=4.6, precision=FP64, poleps=1e-10)
    e = Engine(s, st)
    try:
        r = e.forward()
        h = 1e-5
        for (i, a) in ((0, 0), (2, 1), (40, 2)):
            x = s.xyz.copy()
            x[i, a] += h
            e.set_coords(x)
            p = e.forward(abi.DO_ENERGY)
            x[i, a] -= 2 * h
            e.set_coords(x)
            m = e.forward(abi.DO_ENERGY)
            assert abs((p.em - m.em) / (2 * h) - r.dem[i, a]) < 1e-6
            assert abs((p.ep - m.ep) / (2 * h) - r.dep[i, a]) < 1e-5
    finally:
        e.close()


# ---------------------------------------------------------------- benchmark sizes
@pytest.fixture(scope="module")
def w4096():
    return systems.water_box(4096, 49.7, seed=0)


def test_config_4096_waters_vs_oracle(w4096):
    """The benchmark workload (4,096 waters, 54^3 grid): FP64 GPU vs oracle,
    mixed GPU vs FP64 GPU at the accuracy target."""
    st = Settings(nfft=(54, 54, 54), precision=FP64, poleps=1e-8)
    o = oracle.forward(w4096, st, tol=1e-10)
    g64 = run(w4096, st)
    assert rel(g64.em, o.em) < 1e-10 and rel(g64.ep, o.ep) < 1e-8
    assert np.abs(g64.dem + g64.dep - o.dem - o.dep).max() < 1e-5
    gm = run(w4096, Settings(nfft=(54, 54, 54), precision=MIXED))
    assert rel(gm.em, o.em) < 1e-6 and rel(gm.ep, o.ep) < 1e-6
    assert frms(gm, o) < 1e-4


# ---------------------------------------------------------------- status codes
def test_status_codes():
    s = systems.water_box(64, 12.4, seed=5)
    with pytest.raises(AmgError, match="NO_CONVERGE"):
        run(s, Settings(nfft=(16, 16, 16), cutoff=6.0, politer=1, poleps=1e-9))
    bad = systems.water_box(8, 10.0, seed=0)
    with pytest.raises(AmgError, match="BAD_ARG"):
        run(bad, Settings(nfft=(16, 16, 16), cutoff=7.0))   # cutoff > box/2
    e = Engine(s, Settings(nfft=(16, 16, 16), cutoff=6.0))
    try:
        x = s.xyz.copy()
        x[3, 1] = np.nan
        with pytest.raises(AmgError, match="NAN"):
            e.set_coords(x)
    finally:
        e.close()


@pytest.mark.parametrize("prec,tol", [(FP64, 1e-12), (MIXED, 1e-6)])
def test_repeated_calls_reuse_the_captured_graph(w216, prec, tol):
    """Replaying the captured evaluation, and again after new coordinates.
    PME spreading adds with atomics, so results agree to round-off only
    (FP32 grids in the mixed path)."""
    e = Engine(w216, Settings(nfft=(24, 24, 24), precision=prec))
    try:
        a = e.forward()
        b = e.forward()
        x = w216.xyz + 0.01
        e.set_coords(x)
        c = e.forward()
        e.set_coords(w216.xyz)
        d = e.forward()
    finally:
        e.close()
    assert rel(a.em, b.em) < tol and rel(a.ep, b.ep) < tol
    assert rel(a.em + a.ep, c.em + c.ep) > 1e-5
    assert rel(a.em, d.em) < tol and np.abs(a.dep - d.dep).max() < 1e3 * tol
