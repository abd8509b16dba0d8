"""Generates the committed golden fixtures of tests/golden/ from the reference.

    python tests/golden/make_golden.py <reference-root>

Needs the compiled reference (oracle/_ref, built by `make -f oracle/ref.mk`)
and the reference source tree.  Writes:

  ref_tests.json        the expected values the reference's own Catch2 tests
                        hold (test/amoeba.h, bounds.h, chkpole.h,
                        amoebaMisc.h, rotpole.h), parsed from the headers,
                        with the input files they apply to;
  ref_water216.json     the reference run (oracle/_ref/ref_dump) on the
                        seeded 216-water box in its only electrostatics mode
                        (non-Ewald multipoles, 7 A cutoff): em, nem, dem, vir,
                        einter, rotated multipoles, and the coordinates it read;
  ref_params.json       the reference's parameter assignment (mechanic() with
                        Ewald + mutual polarization keys) for the first
                        molecules of the water03 box and of the amoebabio18
                        ion solution: pole, frames, polarity, thole, pdamp,
                        groups, scale factors, Ewald/PME settings.
"""
from __future__ import annotations

import json
import os
import re
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from polmdqc_b200 import systems  # noqa: E402

REF_BUILD = os.path.join(ROOT, "oracle", "_ref")
DUMP = os.path.join(REF_BUILD, "ref_dump")


def parse_header(path):
    """namespace name { real x = v; std::vector<real> y = {..}; } -> dict"""
    text = open(path).read().replace("namespace polmdqc", "", 1)
    text = text[text.index("{") + 1:]
    out = {}
    for m in re.finditer(r"namespace\s+(\w+)\s*\{(.*?)\n\}", text, re.S):
        name, body = m.group(1), m.group(2)
        d = {}
        for mm in re.finditer(r"(?:real|int)\s+(\w+)\s*=\s*([-+0-9.eE]+)\s*;", body):
            d[mm.group(1)] = float(mm.group(2))
        for mm in re.finditer(r"std::vector<real>\s+(\w+)\s*=\s*\{(.*?)\};", body, re.S):
            d[mm.group(1)] = [float(v) for v in mm.group(2).replace("\n", " ").split(",") if v.strip()]
        for mm in re.finditer(r"std::vector<std::vector<real>>\s+(\w+)\s*=\s*\{(.*?)\};", body, re.S):
            rows = re.findall(r"\{([^{}]*)\}", mm.group(2))
            d[mm.group(1)] = [[float(v) for v in r.replace("\n", " ").split(",") if v.strip()] for r in rows]
        out[name] = d
    return out


def run_dump(xyz, key, cwd):
    out = os.path.join(cwd, "dump.json")
    subprocess.check_call([DUMP, "--out", out, "-k", key, xyz], cwd=cwd, stdout=subprocess.DEVNULL,
                          stderr=subprocess.DEVNULL)
    return json.load(open(out))


def main(ref_root):
    # ---- golden values of the reference's own tests
    hdr = {h: parse_header(os.path.join(ref_root, "test", h + ".h"))
           for h in ("amoeba", "bounds", "chkpole", "amoebaMisc", "rotpole", "amoebap", "hippo")}
    amoeba, bounds = hdr["amoeba"], hdr["bounds"]
    tests = {
        "source": "test/amoeba.h, bounds.h, chkpole.h, amoebaMisc.h, rotpole.h, amoebap.h, hippo.h of momokchung/polmdqc",
        "amoeba1": {"inputs": "test/testFiles/amoeba/water09.xyz (+ water09.key)", **amoeba["amoeba1"]},
        "amoeba2": {"inputs": "test/testFiles/amoeba/water09.xyz (+ water09.key)", **amoeba["amoeba2"]},
    }
    # chiral Z-then-X sites (alanine tetrapeptide, amoebabio09, multipoles only)
    for k in ("chkpole1", "chkpole2"):
        tests[k] = {"inputs": "test/testFiles/chkpole/alatet.xyz (+ alatet.key)", **hdr["chkpole"][k]}
    # reader cases: a versioned file name (water09 -> water09.xyz_2), a
    # concatenated file (the goldens hold its last structure, the water
    # dimer) and non-sequential atom numbers
    misc_inputs = {"amoebaMisc1": "test/testFiles/amoebaMisc/water09 (the reader opens water09.xyz_2)",
                   "amoebaMisc2": "test/testFiles/amoebaMisc/alatet_water09.xyz (last structure)",
                   "amoebaMisc3": "test/testFiles/amoebaMisc/alatet_water09.xyz (last structure)",
                   "amoebaMisc5": "test/testFiles/amoebaMisc/water09NSeq.xyz"}
    for k, inp in misc_inputs.items():
        tests[k] = {"inputs": inp, **hdr["amoebaMisc"][k]}
    # frames: Z-Only (rotpole2/5) and Z-Bisect + 3-Fold (rotpole3/6) in HIPPO
    # inputs (charge penetration, Gordon f1, no charge flux)
    for k, inp in (("rotpole2", "test/testFiles/rotpole/benzene_ethyne_water.xyz"),
                   ("rotpole3", "test/testFiles/rotpole/ammonia.xyz"),
                   ("rotpole5", "test/testFiles/rotpole/benzene_ethyne_water.xyz"),
                   ("rotpole6", "test/testFiles/rotpole/ammonia.xyz")):
        tests[k] = {"inputs": inp, **hdr["rotpole"][k]}
    # charge penetration with charge flux: the AMOEBA+ water dimer (Gordon
    # f2, amoebaplus.prm) and the HIPPO water dimer (Gordon f1, water21.prm)
    for name, inp in (("amoebap", "test/testFiles/amoebap/waterap.xyz"), ("hippo", "test/testFiles/hippo/water21.xyz")):
        for k in (name + "1", name + "2"):
            tests[k] = {"inputs": inp, **hdr[name][k]}
    shapes = {"bounds1": "orthogonal", "bounds2": "monoclinic", "bounds3": "triclinic", "bounds4": "octahedron",
              "bounds5": "dodecahedron"}
    for k, shape in shapes.items():
        tests[k] = {"inputs": f"test/testFiles/bounds/waterbox30.xyz -k {shape}.key", **bounds[k]}
    json.dump(tests, open(os.path.join(HERE, "ref_tests.json"), "w"), indent=1)

    with tempfile.TemporaryDirectory() as tmp:
        prm_dir = os.path.join(REF_BUILD, "params")
        # ---- 216-water box, the reference's non-Ewald multipole path
        s = systems.water_box(216, 18.643, seed=0)
        xyz, key = os.path.join(tmp, "w.xyz"), os.path.join(tmp, "w.key")
        systems.write_tinker(s, xyz, key, os.path.join(prm_dir, "water03.prm"),
                             ["multipoleterm only", "mpole-cutoff 7.0", "digits 10"])
        d = run_dump(xyz, key, tmp)
        keep = {k: d[k] for k in ("n", "x", "y", "z", "em", "nem", "einter", "dem", "vir", "mpolecut", "box")}
        keep["rpole"] = d["rpole"][: 13 * 30]
        keep["generator"] = "systems.water_box(216, 18.643, seed=0); keys: multipoleterm only, mpole-cutoff 7.0"
        json.dump(keep, open(os.path.join(HERE, "ref_water216.json"), "w"))

        # ---- parameter assignment with the Ewald + polarization keys
        params = {}
        ewald_keys = ["ewald", "ewald-alpha 0.5446", "ewald-cutoff 7.0", "pme-grid 24 24 24", "pme-order 5",
                      "polarization mutual", "polar-eps 0.000001"]
        cases = [("water03", systems.water_box(27, 9.32, seed=1), "water03.prm"),
                 ("amoebabio18", systems.ion_solution(n_waters=60, n_pairs=2, box_len=14.0, seed=2),
                  "amoebabio18.prm")]
        for name, sy, prm in cases:
            systems.write_tinker(sy, xyz, key, os.path.join(prm_dir, prm), ewald_keys)
            d = run_dump(xyz, key, tmp)
            m = 30
            # the reference stores atom types 0-based (type - 1)
            ions = [i for i in range(d["n"]) if d["type"][i] + 1 in (352, 363)]
            sel = list(range(m)) + ions
            entry = {k: d[k] for k in ("n", "mscale", "pscale", "piscale", "dscale", "uscale", "poleps", "politer",
                                      "aewald", "aeewald", "apewald", "nefft", "bseorder", "ewaldcut", "usolvcut",
                                      "electric", "dielec", "debye")}
            entry["atoms"] = sel
            for k in ("type", "zaxis", "xaxis", "yaxis", "polaxe", "polarity", "thole", "pdamp", "molcule"):
                entry[k] = [d[k][i] for i in sel]
            entry["pole"] = [d["pole"][13 * i:13 * i + 13] for i in sel]
            for k in ("i12", "i13", "ip11", "ip12"):
                entry[k] = [d[k][i] for i in sel]
            entry["generator"] = {"water03": "systems.water_box(27, 9.32, seed=1)",
                                  "amoebabio18": "systems.ion_solution(60, 2, 14.0, seed=2)"}[name]
            params[name] = entry
        json.dump(params, open(os.path.join(HERE, "ref_params.json"), "w"), indent=0)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <reference-root>")
    main(sys.argv[1])
