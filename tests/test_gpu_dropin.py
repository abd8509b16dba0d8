"""The drop-in shim (polmdqc_b200/host/polmdqc_shim.cpp) inside the
reference's own program: the reference's set-up (parameter loading,
mechanic) and energy() with empole/epolar running on the GPU through the C
ABI.  Uses oracle/_ref/ref_dump_gpu, the reference dump driver linked with the
shim in place of empole.o."""
import json
import os
import subprocess
import tempfile

import numpy as np
import pytest

from conftest import REF_BUILD, golden, ref_fixture
from oracle import oracle
from polmdqc_b200 import abi, systems
from polmdqc_b200.engine import Settings

pytestmark = pytest.mark.gpu


def dump_gpu(xyz, key=None, precision="fp64"):
    exe = os.path.join(REF_BUILD, "ref_dump_gpu")
    if not os.path.exists(exe):
        pytest.skip("shim-linked reference build not present")
    env = dict(os.environ, AMG_PRECISION=precision)
    with tempfile.TemporaryDirectory() as tmp:
        out = os.path.join(tmp, "d.json")
        args = [exe, "--out", out] + (["-k", key] if key else []) + [xyz]
        subprocess.check_call(args, cwd=os.path.dirname(xyz), env=env, stdout=subprocess.DEVNULL)
        return json.load(open(out))


def test_dropin_water_dimer_golden():
    """amoeba-1/-2 through the reference's analyze path with the shim."""
    g = golden("ref_tests.json")
    d = dump_gpu(ref_fixture("amoeba", "water09.xyz"))
    a1, a2 = g["amoeba1"], g["amoeba2"]
    assert d["nem"] == a1["nem"]
    assert abs(d["em"] - a1["em"]) < a1["eps"]
    assert abs(d["einter"] - a1["einter"]) < a1["eps"]
    np.testing.assert_allclose(d["aem"], a1["aem"], atol=a1["eps"], rtol=0)
    np.testing.assert_allclose(d["dem"], a2["dem"], atol=a2["eps1"], rtol=0)


@pytest.mark.parametrize("case,shape", [("bounds1", "orthogonal"), ("bounds2", "monoclinic"),
                                        ("bounds3", "triclinic"), ("bounds4", "octahedron"),
                                        ("bounds5", "dodecahedron")])
def test_dropin_waterbox30_golden(case, shape):
    """test/bounds.cpp bounds-1..5 through the reference's program with the
    shim: the keyfile's cell shape reaches the library."""
    g = golden("ref_tests.json")[case]
    d = dump_gpu(ref_fixture("bounds", "waterbox30.xyz"), ref_fixture("bounds", shape + ".key"))
    assert d["nem"] == g["nem"]
    assert abs(d["em"] - g["em"]) < g["eps"]
    assert abs(d["einter"] - g["einter"]) < g["eps"]


def test_dropin_virial_matches_reference():
    """energy<CalcMode::Virial> with the shim: the seeded 216-water box in the
    reference's non-Ewald mode gives the reference's own vir."""
    g = golden("ref_water216.json")
    s = systems.water_box(216, 18.643, seed=0)
    with tempfile.TemporaryDirectory() as tmp:
        xyz, key = os.path.join(tmp, "w.xyz"), os.path.join(tmp, "w.key")
        prm = os.path.join(REF_BUILD, "params", "water03.prm")
        systems.write_tinker(s, xyz, key, prm, ["multipoleterm only", "mpole-cutoff 7.0", "digits 10"])
        d = dump_gpu(xyz, key)
    np.testing.assert_allclose(d["vir"], g["vir"], atol=1e-8 * np.abs(g["vir"]).max(), rtol=0)


def test_dropin_ewald_polarization_matches_oracle():
    """Keyfile with ewald + mutual polarization: the reference's parameter
    loading feeds the GPU path through the shim; em, ep and both gradients
    match the oracle run on the parameters the reference assigned."""
    s = systems.water_box(216, 18.643, seed=0)
    with tempfile.TemporaryDirectory() as tmp:
        xyz, key = os.path.join(tmp, "w.xyz"), os.path.join(tmp, "w.key")
        prm = os.path.join(REF_BUILD, "params", "water03.prm")
        systems.write_tinker(s, xyz, key, prm, ["ewald", "ewald-alpha 0.5446", "ewald-cutoff 7.0",
                                                "pme-grid 24 24 24", "pme-order 5", "polarization mutual",
                                                "polar-eps 0.00000001"])
        d = dump_gpu(xyz, key)
    sd = systems.from_dump(d)
    st = Settings(aewald=d["aeewald"], nfft=tuple(d["nefft"]), cutoff=d["ewaldcut"], precision=abi.PREC_FP64)
    o = oracle.forward(sd, st, tol=1e-11, flags=abi.DO_ENERGY | abi.DO_GRADIENT | abi.DO_DIPOLES | abi.DO_VIRIAL)
    assert abs(d["em"] - o.em) < 1e-9 * abs(o.em)
    np.testing.assert_allclose(d["vir"], o.vir.reshape(-1), atol=1e-7 * np.abs(o.vir).max(), rtol=0)
    assert abs(d["ep"] - o.ep) < 1e-7 * abs(o.ep)
    np.testing.assert_allclose(d["dem"], o.dem.reshape(-1), atol=1e-7)
    np.testing.assert_allclose(d["dep"], o.dep.reshape(-1), atol=1e-5)
    np.testing.assert_allclose(d["uind"], o.uind.reshape(-1), atol=1e-7)


def test_dropin_chiral_sites_golden():
    """chkpole-1/-2 (alanine tetrapeptide, chiral Z-then-X sites) through the
    reference's own set-up and energy() with the shim."""
    g = golden("ref_tests.json")
    d = dump_gpu(ref_fixture("chkpole", "alatet.xyz"))
    c1, c2 = g["chkpole1"], g["chkpole2"]
    assert d["nem"] == c1["nem"]
    assert abs(d["em"] - c1["em"]) < c1["eps"]
    np.testing.assert_allclose(d["aem"], c1["aem"], atol=c1["eps"], rtol=0)
    np.testing.assert_allclose(d["dem"], c2["dem"], atol=c2["eps1"], rtol=0)


def test_dropin_analyze_program_reads_every_structure():
    """amoebaMisc-2: the reference's own analyze program, linked with the
    shim, on a concatenated file (alanine tetrapeptide, then the water
    dimer).  The shim rebuilds its device context when the system changes;
    the last structure's line ' Atomic Multipoles  <em> <nem>' (8 decimals,
    the keyfile's 'digits 8') matches the golden."""
    exe = os.path.join(REF_BUILD, "analyze_gpu")
    if not os.path.exists(exe):
        pytest.skip("shim-linked reference build not present")
    g = golden("ref_tests.json")["amoebaMisc2"]
    xyz = ref_fixture("amoebaMisc", "alatet_water09.xyz")
    env = dict(os.environ, AMG_PRECISION="fp64")
    out = subprocess.run([exe, xyz, "e"], cwd=os.path.dirname(xyz), env=env, capture_output=True, text=True,
                         check=True).stdout
    rows = [line.split() for line in out.splitlines() if line.startswith(" Atomic Multipoles")]
    assert len(rows) == 2, out[-2000:]
    em, nem = float(rows[-1][2]), int(rows[-1][3])
    assert nem == g["nem"]
    assert abs(em - g["em"]) < 1e-8
    assert abs(float(rows[0][2]) - g["em"]) > 1.0     # the first structure is the peptide


@pytest.mark.parametrize("analysis,gradient,name", [("amoebap1", "amoebap2", ("amoebap", "waterap.xyz")),
                                                    ("hippo1", "hippo2", ("hippo", "water21.xyz"))])
def test_dropin_charge_penetration_and_flux_golden(analysis, gradient, name):
    """amoebap-1/-2 and hippo-1/-2 through the reference's own set-up and
    energy() with the shim: its alterchg rewrites the monopoles each call, the
    shim hands the library the unaltered ones and the bond / angle flux terms,
    and the library's charge penetration and charge flux reproduce the
    goldens."""
    g = golden("ref_tests.json")
    d = dump_gpu(ref_fixture(*name))
    ga, gg = g[analysis], g[gradient]
    assert d["nem"] == ga["nem"]
    assert abs(d["em"] - ga["em"]) < ga["eps"]
    np.testing.assert_allclose(d["aem"], ga["aem"], atol=ga["eps"], rtol=0)
    np.testing.assert_allclose(d["dem"], gg["dem"], atol=gg["eps1"], rtol=0)
