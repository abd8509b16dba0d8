"""Host-side behaviour of the drop-in shim (polmdqc_b200/host/polmdqc_shim.cpp)
that needs no GPU: inputs the library does not cover stop the reference's
program the way its own fatal() does, before any device call."""
import os
import subprocess

import pytest

from conftest import REF_BUILD, ref_fixture


def test_charge_penetration_with_ewald_stops_the_program(tmp_path):
    """AMOEBA+ water (test/testFiles/amoebap: charge penetration and charge
    flux) with Ewald summation: the library covers charge penetration only in
    the reference's non-Ewald multipole mode, so amg_create returns
    AMG_ERR_UNSUPPORTED (status 2) from its argument check and the shim stops
    the program instead of returning other energies."""
    exe = os.path.join(REF_BUILD, "ref_dump_gpu")
    if not os.path.exists(exe):
        pytest.skip("shim-linked reference build not present")
    xyz = ref_fixture("amoebap", "waterap.xyz")
    prm = os.path.join(REF_BUILD, "params", "amoebaplus.prm")
    key = tmp_path / "ewald.key"
    key.write_text(f"parameters {prm}\nmultipoleterm only\newald\na-axis 20.0\newald-cutoff 7.0\n")
    p = subprocess.run([exe, "--out", os.devnull, xyz, "-k", str(key)], cwd=os.path.dirname(xyz),
                       capture_output=True, text=True, timeout=120)
    assert p.returncode != 0
    assert "amg_create failed (status 2)" in p.stdout
