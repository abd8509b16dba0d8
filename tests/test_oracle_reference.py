"""The FP64 oracle against the reference's own golden vectors and against the
compiled reference run on the seeded synthetic box (non-Ewald multipoles,
the only electrostatics mode the reference implements)."""
import numpy as np
import pytest

from conftest import golden, ref_dump, ref_fixture
from oracle import oracle
from polmdqc_b200 import abi, systems
from polmdqc_b200.engine import Settings


def nonewald(cut):
    return Settings(use_ewald=False, cutoff=cut, poltyp=abi.POL_NONE)


def test_water_dimer_golden():
    """test/amoeba.cpp amoeba-1/-2: em, aem, nem, einter at 1e-10; analytic dem at 1e-10."""
    g = golden("ref_tests.json")
    d = ref_dump(ref_fixture("amoeba", "water09.xyz"))
    s = systems.from_dump(d)
    r = oracle.forward(s, nonewald(d["mpolecut"]), flags=abi.DO_ENERGY | abi.DO_GRADIENT | abi.DO_ANALYSIS)
    a1, a2 = g["amoeba1"], g["amoeba2"]
    assert abs(r.em - a1["em"]) < a1["eps"]
    assert abs(r.einter - a1["einter"]) < a1["eps"]
    assert r.nem == a1["nem"]
    np.testing.assert_allclose(r.aem, a1["aem"], atol=a1["eps"], rtol=0)
    np.testing.assert_allclose(r.dem.reshape(-1), a2["dem"], atol=a2["eps1"], rtol=0)


@pytest.mark.parametrize("case,shape", [("bounds2", "monoclinic"), ("bounds3", "triclinic"),
                                        ("bounds4", "octahedron"), ("bounds5", "dodecahedron")])
def test_waterbox30_cell_shapes_golden(case, shape):
    """test/bounds.cpp bounds-2..5: the same box as a monoclinic, triclinic,
    truncated-octahedron and rhombic-dodecahedron cell (the reference's
    image(), src/md/image.cpp:37-124): em, nem, einter at 1e-8."""
    g = golden("ref_tests.json")[case]
    d = ref_dump(ref_fixture("bounds", "waterbox30.xyz"), ref_fixture("bounds", shape + ".key"))
    s = systems.from_dump(d)
    r = oracle.forward(s, nonewald(d["mpolecut"]), flags=abi.DO_ENERGY | abi.DO_GRADIENT | abi.DO_ANALYSIS)
    assert r.nem == g["nem"]
    assert abs(r.em - g["em"]) < g["eps"]
    assert abs(r.einter - g["einter"]) < g["eps"]
    np.testing.assert_allclose(r.dem.reshape(-1), d["dem"], atol=1e-8, rtol=0)


def test_waterbox30_orthogonal_golden():
    """test/bounds.cpp bounds-1: 2,700-atom periodic box, cutoff 9, em and nem at 1e-8."""
    g = golden("ref_tests.json")["bounds1"]
    d = ref_dump(ref_fixture("bounds", "waterbox30.xyz"), ref_fixture("bounds", "orthogonal.key"))
    s = systems.from_dump(d)
    r = oracle.forward(s, nonewald(d["mpolecut"]), flags=abi.DO_ENERGY | abi.DO_GRADIENT | abi.DO_ANALYSIS)
    assert r.nem == g["nem"]
    assert abs(r.em - g["em"]) < g["eps"]
    assert abs(r.einter - g["einter"]) < g["eps"]
    np.testing.assert_allclose(r.dem.reshape(-1), d["dem"], atol=1e-9, rtol=0)


def test_synthetic_box_matches_reference_run():
    """216-water seeded box: oracle = compiled reference (em, nem, dem, virial,
    rpole).  The virial is the reference's CalcMode::Virial result: pair terms
    (include/md/pairMpole.h:166-173) plus the frame atoms' torque share
    (src/md/torque.cpp:360-395)."""
    d = golden("ref_water216.json")
    s = systems.water_box(216, 18.643, seed=0)
    s.xyz = np.stack([d["x"], d["y"], d["z"]], 1)   # the coordinates the reference read
    r = oracle.forward(s, nonewald(d["mpolecut"]),
                       flags=abi.DO_ENERGY | abi.DO_GRADIENT | abi.DO_ANALYSIS | abi.DO_VIRIAL)
    assert r.nem == d["nem"]
    assert abs(r.em - d["em"]) < 1e-9 * abs(d["em"])
    np.testing.assert_allclose(r.dem.reshape(-1), d["dem"], atol=1e-9, rtol=0)
    np.testing.assert_allclose(r.vir.reshape(-1), d["vir"], atol=1e-8, rtol=0)
    np.testing.assert_allclose(r.rpole.reshape(-1)[: len(d["rpole"])], d["rpole"], atol=1e-13, rtol=0)


@pytest.mark.parametrize("name", ["water03", "amoebabio18"])
def test_parameter_assignment_matches_reference(name):
    """systems.* assigns the same pole/frames/polarizabilities/groups as the
    reference's mechanic() (kmpole, kpolar, polargrp) for the synthetic inputs."""
    p = golden("ref_params.json")[name]
    s = (systems.water_box(27, 9.32, seed=1) if name == "water03"
         else systems.ion_solution(n_waters=60, n_pairs=2, box_len=14.0, seed=2))
    idx = p["atoms"]
    assert s.n == p["n"]
    np.testing.assert_allclose(s.pole[idx], p["pole"], atol=1e-15)
    for k in ("zaxis", "xaxis", "yaxis", "polaxe", "molcule"):
        np.testing.assert_array_equal(getattr(s, k)[idx], p[k], err_msg=k)
    for k in ("polarity", "thole", "pdamp"):
        np.testing.assert_allclose(getattr(s, k)[idx], p[k], rtol=1e-14, err_msg=k)
    for k in ("i12", "i13", "ip11", "ip12"):
        assert [sorted(s.lists[k][i]) for i in idx] == [sorted(v) for v in p[k]], k
    for k, ref in (("m_scale", "mscale"), ("p_scale", "pscale"), ("p_iscale", "piscale"), ("d_scale", "dscale"),
                   ("u_scale", "uscale")):
        assert getattr(s, k) == p[ref], k
    assert p["aeewald"] == 0.5446 and p["nefft"] == [24, 24, 24] and p["bseorder"] == 5


@pytest.mark.parametrize("model,order", [("OPT1", 1), ("OPT2", 2), ("OPT3", 3), ("OPT", 4), ("OPT4", 4),
                                         ("OPT5", 5), ("OPT6", 6)])
def test_opt_coefficients_match_the_reference(tmp_path, model, order):
    """The OPT coefficients of polmdqc_b200.engine.OPT_COEF are the reference's
    own (kpolar, src/md/kpolar.cpp:108-153; plain "OPT" is OPT4), read from
    its copt after mechanic() with the keyword 'polarization <model>'."""
    import os
    from conftest import REF_BUILD
    from polmdqc_b200.engine import OPT_COEF
    s = systems.water_box(27, 9.32, seed=1)
    xyz, key = str(tmp_path / "w.xyz"), str(tmp_path / "w.key")
    prm = os.path.join(REF_BUILD, "params", "water03.prm")
    if not os.path.exists(prm):
        pytest.skip("reference build (oracle/_ref) not present")
    systems.write_tinker(s, xyz, key, prm, [f"polarization {model}"])
    d = ref_dump(xyz, key)
    assert d["poltyp"] == "OPT"
    want = list(OPT_COEF[order]) + [0.0] * (7 - len(OPT_COEF[order]))
    # the reference zeroes copt below index maxopt only (kpolar.cpp:110-113),
    # so its last entry can hold a leftover denormal for orders below 6
    np.testing.assert_allclose(d["copt"], want, rtol=0, atol=1e-300)


def _analysis(d):
    s = systems.from_dump(d)
    return s, oracle.forward(s, nonewald(d["mpolecut"]), flags=abi.DO_ENERGY | abi.DO_GRADIENT | abi.DO_ANALYSIS)


def flip_chiral_sites(s):
    """The other chirality at every chiral Z-then-X site: yaxis and the
    y-components of the local multipoles (dipole y, quadrupole xy/yx/yz/zy)
    change sign, which is what the reference's chkpole undoes when the
    site's chirality disagrees with the sign of yaxis
    (src/md/chkpole.cpp:44-89).  Returns the number of sites flipped."""
    sites = [i for i in range(s.n) if s.polaxe[i] == abi.FRAME_ZTHENX and s.yaxis[i] != 0]
    for i in sites:
        s.yaxis[i] = -s.yaxis[i]
        for c in (2, 5, 7, 9, 11):
            s.pole[i, c] = -s.pole[i, c]
    return len(sites)


def test_chiral_sites_golden():
    """test/chkpole.cpp chkpole-1/-2: alanine tetrapeptide (amoebabio09),
    chiral Z-then-X sites: em, nem, einter, aem and dem at 1e-10; the same
    values when every chiral site is given the opposite chirality first."""
    g = golden("ref_tests.json")
    d = ref_dump(ref_fixture("chkpole", "alatet.xyz"))
    s, r = _analysis(d)
    c1, c2 = g["chkpole1"], g["chkpole2"]
    assert r.nem == c1["nem"]
    assert abs(r.em - c1["em"]) < c1["eps"] and abs(r.einter - c1["einter"]) < c1["eps"]
    np.testing.assert_allclose(r.aem, c1["aem"], atol=c1["eps"], rtol=0)
    np.testing.assert_allclose(r.dem.reshape(-1), c2["dem"], atol=c2["eps1"], rtol=0)
    assert flip_chiral_sites(s) == 3
    f = oracle.forward(s, nonewald(d["mpolecut"]), flags=abi.DO_ENERGY | abi.DO_GRADIENT)
    assert abs(f.em - c1["em"]) < c1["eps"]
    np.testing.assert_allclose(f.dem.reshape(-1), c2["dem"], atol=c2["eps1"], rtol=0)


@pytest.mark.parametrize("case,parts", [("amoebaMisc1", ("amoebaMisc", "water09")),
                                        ("amoebaMisc2", ("amoebaMisc", "alatet_water09.xyz")),
                                        ("amoebaMisc5", ("amoebaMisc", "water09NSeq.xyz"))])
def test_reader_cases_golden(tmp_path, case, parts):
    """test/amoebaMisc.cpp amoebaMisc-1/-2/-3/-5: a versioned file name, the
    last structure of a concatenated file, non-sequential atom numbers."""
    import os
    g = golden("ref_tests.json")[case]
    xyz = ref_fixture(*parts) if parts[1] != "water09" else os.path.join(
        os.path.dirname(ref_fixture("amoebaMisc", "water09.xyz")), "water09")
    if case == "amoebaMisc2":
        from conftest import last_structure
        xyz, key = last_structure(xyz, ref_fixture("amoebaMisc", "alatet_water09.key"), str(tmp_path))
        d = ref_dump(xyz, key)
    else:
        d = ref_dump(xyz)
    _, r = _analysis(d)
    assert r.nem == g["nem"]
    assert abs(r.em - g["em"]) < g["eps"] and abs(r.einter - g["einter"]) < g["eps"]
    np.testing.assert_allclose(r.aem, g["aem"], atol=g["eps"], rtol=0)
    if case == "amoebaMisc2":
        g3 = golden("ref_tests.json")["amoebaMisc3"]
        np.testing.assert_allclose(r.dem.reshape(-1), g3["dem"], atol=g3["eps1"], rtol=0)


@pytest.mark.parametrize("case,name", [("rotpole2", "benzene_ethyne_water.xyz"), ("rotpole3", "ammonia.xyz")])
def test_frames_golden_rotated_multipoles(case, name):
    """test/rotpole.cpp rotpole-2 (Z-Only) and rotpole-3 (Z-Bisect, 3-Fold):
    the rotated multipoles at 1e-14 (the reference holds them at 1e-16 against
    its own Eigen rotation; the restatement here rounds differently)."""
    g = golden("ref_tests.json")[case]
    d = ref_dump(ref_fixture("rotpole", name))
    s = systems.from_dump(d)
    r = oracle.forward(s, nonewald(d["mpolecut"]), flags=abi.DO_ENERGY)
    np.testing.assert_allclose(r.rpole, np.array(g["rpole"]), atol=1e-14, rtol=0)


CP_CASES = [("amoebap1", "amoebap2", ("amoebap", "waterap.xyz")),      # Gordon f2 + charge flux (AMOEBA+)
            ("hippo1", "hippo2", ("hippo", "water21.xyz")),            # Gordon f1 + charge flux (HIPPO)
            ("rotpole3", "rotpole6", ("rotpole", "ammonia.xyz")),      # Gordon f1, Z-Bisect and 3-Fold frames
            ("rotpole2", "rotpole5", ("rotpole", "benzene_ethyne_water.xyz"))]  # Gordon f1, Z-Only frames


@pytest.mark.parametrize("analysis,gradient,parts", CP_CASES)
def test_charge_penetration_goldens(analysis, gradient, parts):
    """test/amoebap.cpp, test/hippo.cpp and test/rotpole.cpp: charge
    penetration of the multipoles (include/md/pairMpole.h:186-389), with charge
    flux for the AMOEBA+ and HIPPO water dimers (src/md/alterchg.cpp,
    src/md/dcflux.cpp): em, nem, einter, aem at eps and the analytic dem at
    eps1 (1e-10)."""
    g = golden("ref_tests.json")
    ga, gg = g[analysis], g[gradient]
    d = ref_dump(ref_fixture(*parts))
    assert d["pentype"] in (1, 2)
    _, r = _analysis(d)
    assert r.nem == ga["nem"]
    assert abs(r.em - ga["em"]) < ga["eps"] and abs(r.einter - ga["einter"]) < ga["eps"]
    np.testing.assert_allclose(r.aem, ga["aem"], atol=ga["eps"], rtol=0)
    np.testing.assert_allclose(r.dem.reshape(-1), gg["dem"], atol=gg["eps1"], rtol=0)


def test_charge_flux_gradient_matches_finite_differences():
    """The charge-flux chain rule of the oracle (dE/dq times dq/dx for bonds
    and angles) against central differences of its energies, on the HIPPO
    water dimer with its bonds and angles bent away from their ideal values."""
    d = ref_dump(ref_fixture("hippo", "water21.xyz"))
    s = systems.from_dump(d)
    rng = np.random.default_rng(2)
    s.xyz = s.xyz + 0.05 * rng.standard_normal(s.xyz.shape)
    st = nonewald(d["mpolecut"])
    r = oracle.forward(s, st, flags=abi.DO_ENERGY | abi.DO_GRADIENT)
    h = 1e-5
    for i in range(s.n):
        for a in range(3):
            x = s.xyz.copy()
            x[i, a] += h
            p = oracle.forward(s, st, xyz=x, flags=abi.DO_ENERGY).em
            x[i, a] -= 2 * h
            m = oracle.forward(s, st, xyz=x, flags=abi.DO_ENERGY).em
            assert abs((p - m) / (2 * h) - r.dem[i, a]) < 1e-7, (i, a)
