"""Host-side behaviour of the drop-in shim (polmdqc_b200/host/polmdqc_shim.cpp)
that needs no GPU: inputs the library does not cover stop the reference's
program the way its own fatal() does, before any device call."""
import os
import subprocess

import pytest

from conftest import REF_BUILD, ref_fixture


def test_charge_penetration_stops_the_program():
    """AMOEBA+ water (test/testFiles/amoebap, charge penetration and charge
    flux): the shim refuses instead of returning plain multipole energies."""
    exe = os.path.join(REF_BUILD, "ref_dump_gpu")
    if not os.path.exists(exe):
        pytest.skip("shim-linked reference build not present")
    xyz = ref_fixture("amoebap", "waterap.xyz")
    p = subprocess.run([exe, "--out", os.devnull, xyz, "-k", "waterap.key"], cwd=os.path.dirname(xyz),
                       capture_output=True, text=True, timeout=120)
    assert p.returncode != 0
    assert "charge penetration / charge flux are not supported" in p.stdout
