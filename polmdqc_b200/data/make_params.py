"""Extracts the parameter subsets the synthetic workloads use from the
reference's Tinker parameter files (params/water03.prm and
params/amoebabio18.prm of momokchung/polmdqc) into small JSON files.

    python -m polmdqc_b200.data.make_params <reference-root>

Only the records of the listed atom types are kept: multipole (converted
units), polarize, atom, and the scale-factor / polarization keywords.
"""
import json
import os
import sys

from polmdqc_b200 import prm

SETS = {"water03": [1, 2], "amoebabio18": [349, 350, 352, 363]}


def main(root):
    here = os.path.dirname(os.path.abspath(__file__))
    for name, types in SETS.items():
        text = open(os.path.join(root, "params", f"{name}.prm")).read()
        ff = prm.read_prm(text, wanted_types=set(types))
        out = {
            "source": f"params/{name}.prm",
            "atoms": {t: list(ff.atoms[t]) for t in types},
            "multipoles": {t: [{"types": list(r.types), "pole": r.pole} for r in ff.multipoles[t]] for t in types},
            "polarize": {t: list(ff.polarize[t]) for t in types},
            "m_scale": ff.m_scale, "p_scale": ff.p_scale, "p_iscale": ff.p_iscale,
            "d_scale": ff.d_scale, "u_scale": ff.u_scale,
            "dielec": ff.dielec, "polarization": ff.polarization,
        }
        with open(os.path.join(here, f"{name}.json"), "w") as f:
            json.dump(out, f, indent=1)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python -m polmdqc_b200.data.make_params <reference-root>")
    main(sys.argv[1])
