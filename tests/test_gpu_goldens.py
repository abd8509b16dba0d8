"""The reference's remaining AMOEBA goldens through the CUDA path (C ABI),
FP64 and mixed: chiral Z-then-X sites (chkpole-1/-2), the reader cases
(amoebaMisc-1/-2/-3/-5), the water dimer's analytic gradient of the testgrad
run (amoeba-3), and the Z-Only, Z-Bisect and 3-Fold frames (rotpole-2/-3:
rotated multipoles; the torques of those frames against central differences
of the GPU's own energies and against the oracle).

Tolerances: FP64 at the reference's own eps (1e-10); mixed 2e-6 of |em| for
energies and 1e-4 kcal/mol/A for gradients.
"""
import os

import numpy as np
import pytest

from conftest import golden, last_structure, ref_dump, ref_fixture
from oracle import oracle
from polmdqc_b200 import abi, systems
from polmdqc_b200.engine import Engine, Settings
from test_oracle_reference import flip_chiral_sites

pytestmark = pytest.mark.gpu

FP64, MIXED = abi.PREC_FP64, abi.PREC_MIXED
FLAGS = abi.DO_ENERGY | abi.DO_GRADIENT | abi.DO_ANALYSIS


def run(s, cut, prec, flags=FLAGS):
    e = Engine(s, Settings(use_ewald=False, cutoff=cut, poltyp=abi.POL_NONE, precision=prec))
    try:
        return e.forward(flags)
    finally:
        e.close()


def check_analysis(r, g, prec, eps_key="eps"):
    tol = g[eps_key] if prec == FP64 else 2e-6 * abs(g["em"])
    assert r.nem == g["nem"]
    assert abs(r.em - g["em"]) < tol, (r.em, g["em"])
    assert abs(r.einter - g["einter"]) < tol
    np.testing.assert_allclose(r.aem, g["aem"], atol=tol, rtol=0)


@pytest.mark.parametrize("prec", [FP64, MIXED])
def test_chiral_sites_golden(prec):
    """chkpole-1/-2 (alanine tetrapeptide, amoebabio09): em, nem, einter, aem
    and dem; then every chiral site given the opposite chirality, which the
    GPU's sign test must undo (src/md/chkpole.cpp:44-89)."""
    g = golden("ref_tests.json")
    d = ref_dump(ref_fixture("chkpole", "alatet.xyz"))
    s = systems.from_dump(d)
    r = run(s, d["mpolecut"], prec)
    check_analysis(r, g["chkpole1"], prec)
    tol_g = g["chkpole2"]["eps1"] if prec == FP64 else 1e-4
    np.testing.assert_allclose(r.dem.reshape(-1), g["chkpole2"]["dem"], atol=tol_g, rtol=0)
    assert flip_chiral_sites(s) == 3
    f = run(s, d["mpolecut"], prec)
    check_analysis(f, g["chkpole1"], prec)
    np.testing.assert_allclose(f.dem.reshape(-1), g["chkpole2"]["dem"], atol=tol_g, rtol=0)


@pytest.mark.parametrize("prec", [FP64, MIXED])
@pytest.mark.parametrize("case", ["amoebaMisc1", "amoebaMisc2", "amoebaMisc5"])
def test_reader_cases_golden(tmp_path, case, prec):
    """amoebaMisc-1/-2/-3/-5: the inputs as the reference's reader produces
    them (a versioned file name, the last structure of a concatenated file,
    non-sequential atom numbers)."""
    g = golden("ref_tests.json")
    base = os.path.dirname(ref_fixture("amoebaMisc", "water09.xyz"))
    if case == "amoebaMisc1":
        d = ref_dump(os.path.join(base, "water09"))
    elif case == "amoebaMisc2":
        xyz, key = last_structure(os.path.join(base, "alatet_water09.xyz"),
                                  os.path.join(base, "alatet_water09.key"), str(tmp_path))
        d = ref_dump(xyz, key)
    else:
        d = ref_dump(os.path.join(base, "water09NSeq.xyz"))
    r = run(systems.from_dump(d), d["mpolecut"], prec)
    check_analysis(r, g[case], prec)
    if case == "amoebaMisc2":
        tol_g = g["amoebaMisc3"]["eps1"] if prec == FP64 else 1e-4
        np.testing.assert_allclose(r.dem.reshape(-1), g["amoebaMisc3"]["dem"], atol=tol_g, rtol=0)


def test_water_dimer_testgrad_golden():
    """amoeba-3 (testgrad, analytic only): em at amoeba-1's eps and dem at
    amoeba-2's eps1, from a gradient evaluation without Analysis outputs."""
    g = golden("ref_tests.json")
    d = ref_dump(ref_fixture("amoeba", "water09.xyz"))
    r = run(systems.from_dump(d), d["mpolecut"], FP64, abi.DO_ENERGY | abi.DO_GRADIENT)
    assert abs(r.em - g["amoeba1"]["em"]) < g["amoeba1"]["eps"]
    np.testing.assert_allclose(r.dem.reshape(-1), g["amoeba2"]["dem"], atol=g["amoeba2"]["eps1"], rtol=0)


@pytest.mark.parametrize("case,name,fd_tol", [("rotpole2", "benzene_ethyne_water.xyz", 1e-6),
                                              ("rotpole3", "ammonia.xyz", 1e-4)])
def test_frames_rotated_multipoles_and_torques(case, name, fd_tol):
    """rotpole-2 (Z-Only) and rotpole-3 (Z-Bisect, 3-Fold): the GPU's rotated
    multipoles against the reference's golden at 1e-14; then, with the charge
    penetration of these HIPPO inputs switched off so that only the frames and
    torques are under test, dem against the oracle at 1e-9 and against central
    differences (step 1e-5 A) of the GPU's own FP64 energies for every atom.
    The reference's torque for Z-Bisect and 3-Fold sites is not the exact
    derivative of its energy (the oracle, which restates it, differs from its
    own finite differences by 4e-5 on ammonia, and the reference's testgrad
    run of ammonia, rotpole-6, allows 1e-4); those frames are held to that
    tolerance, Z-Only to 1e-6."""
    import dataclasses
    g = golden("ref_tests.json")[case]
    d = ref_dump(ref_fixture("rotpole", name))
    s = dataclasses.replace(systems.from_dump(d), pentype=0)
    cut = d["mpolecut"]
    st = Settings(use_ewald=False, cutoff=cut, poltyp=abi.POL_NONE, precision=FP64)
    e = Engine(s, st)
    try:
        r = e.forward(abi.DO_ENERGY | abi.DO_GRADIENT)
        np.testing.assert_allclose(r.rpole, np.array(g["rpole"]), atol=1e-14, rtol=0)
        o = oracle.forward(s, st, flags=abi.DO_ENERGY | abi.DO_GRADIENT)
        assert abs(r.em - o.em) < 1e-10 * abs(o.em)
        np.testing.assert_allclose(r.dem, o.dem, atol=1e-9, rtol=0)
        h = 1e-5
        for i in range(s.n):
            for a in range(3):
                x = s.xyz.copy()
                x[i, a] += h
                e.set_coords(x)
                p = e.forward(abi.DO_ENERGY).em
                x[i, a] -= 2 * h
                e.set_coords(x)
                m = e.forward(abi.DO_ENERGY).em
                assert abs((p - m) / (2 * h) - r.dem[i, a]) < fd_tol, (i, a)
    finally:
        e.close()


CP_CASES = [("amoebap1", "amoebap2", ("amoebap", "waterap.xyz")),      # Gordon f2 + charge flux (AMOEBA+)
            ("hippo1", "hippo2", ("hippo", "water21.xyz")),            # Gordon f1 + charge flux (HIPPO)
            ("rotpole3", "rotpole6", ("rotpole", "ammonia.xyz")),      # Gordon f1, Z-Bisect and 3-Fold frames
            ("rotpole2", "rotpole5", ("rotpole", "benzene_ethyne_water.xyz"))]  # Gordon f1, Z-Only frames


@pytest.mark.parametrize("prec", [FP64, MIXED])
@pytest.mark.parametrize("analysis,gradient,parts", CP_CASES)
def test_charge_penetration_goldens(analysis, gradient, parts, prec):
    """amoebap-1/-2, hippo-1/-2 and rotpole-2/-3/-5/-6 through the C ABI:
    charge penetration of the multipoles (the FP64 core/valence pair kernels
    in both precisions) and, for the two water dimers, charge flux: em, nem,
    einter, aem at the reference's eps and dem at eps1 (1e-10)."""
    g = golden("ref_tests.json")
    ga, gg = g[analysis], g[gradient]
    d = ref_dump(ref_fixture(*parts))
    r = run(systems.from_dump(d), d["mpolecut"], prec)
    check_analysis(r, ga, FP64)
    np.testing.assert_allclose(r.dem.reshape(-1), gg["dem"], atol=gg["eps1"], rtol=0)
