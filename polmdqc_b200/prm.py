"""Tinker parameter-file reading for the electrostatics path.

Restates the parts of the reference's parameter loading that the path needs:
  - `atom` records (type -> class, symbol), src/md/readprm.cpp
  - `multipole` records (5 lines: monopole, dipole, 3 quadrupole rows),
    src/md/readprm.cpp:1157-1235, with the unit conversion of
    src/md/kmpole.cpp:547-550 (dipoles x bohr, quadrupoles x bohr^2/3)
  - `polarize` records (polarizability, Thole, group partner types),
    src/md/readprm.cpp:1250-1314
  - the scale-factor and polarization keywords of src/md/prmkey.cpp:497-603
    with the defaults of src/md/initprm.cpp:345-395.
"""
from __future__ import annotations

import dataclasses
import re

BOHR = 0.529177210903        # units.h:75
COULOMB = 332.0637133        # units.h:79
DEBYE = 4.80321              # units.h:81


@dataclasses.dataclass
class MultipoleRecord:
    types: tuple               # (type, ztype, xtype, ytype) as written (signs kept)
    pole: list                 # 13 components, converted units


@dataclasses.dataclass
class ForceField:
    atoms: dict = dataclasses.field(default_factory=dict)        # type -> (class, symbol)
    multipoles: dict = dataclasses.field(default_factory=dict)   # type -> [MultipoleRecord]
    polarize: dict = dataclasses.field(default_factory=dict)     # type -> (alpha, thole, [group types])
    m_scale: list = dataclasses.field(default_factory=lambda: [0.0, 0.0, 1.0, 1.0])
    p_scale: list = dataclasses.field(default_factory=lambda: [0.0, 0.0, 1.0, 1.0])
    p_iscale: list = dataclasses.field(default_factory=lambda: [0.0, 0.0, 0.5, 1.0])
    d_scale: list = dataclasses.field(default_factory=lambda: [0.0, 1.0, 1.0, 1.0])
    u_scale: list = dataclasses.field(default_factory=lambda: [1.0, 1.0, 1.0, 1.0])
    dielec: float = 1.0
    polarization: str = "MUTUAL"


def _scale(v: float) -> float:
    return 1.0 / v if v > 1.0 else v


_SCALE_KEYS = {
    "MPOLE-12-SCALE": ("m_scale", 0), "MPOLE-13-SCALE": ("m_scale", 1),
    "MPOLE-14-SCALE": ("m_scale", 2), "MPOLE-15-SCALE": ("m_scale", 3),
    "POLAR-12-SCALE": ("p_scale", 0), "POLAR-13-SCALE": ("p_scale", 1),
    "POLAR-14-SCALE": ("p_scale", 2), "POLAR-15-SCALE": ("p_scale", 3),
    "POLAR-12-INTRA": ("p_iscale", 0), "POLAR-13-INTRA": ("p_iscale", 1),
    "POLAR-14-INTRA": ("p_iscale", 2), "POLAR-15-INTRA": ("p_iscale", 3),
    "DIRECT-11-SCALE": ("d_scale", 0), "DIRECT-12-SCALE": ("d_scale", 1),
    "DIRECT-13-SCALE": ("d_scale", 2), "DIRECT-14-SCALE": ("d_scale", 3),
    "MUTUAL-11-SCALE": ("u_scale", 0), "MUTUAL-12-SCALE": ("u_scale", 1),
    "MUTUAL-13-SCALE": ("u_scale", 2), "MUTUAL-14-SCALE": ("u_scale", 3),
}


def read_prm(text: str, wanted_types=None) -> ForceField:
    """Parses a Tinker .prm text.  wanted_types limits multipole/polarize
    records to those atom types (speeds up big files)."""
    ff = ForceField()
    lines = text.splitlines()
    i = 0
    while i < len(lines):
        raw = lines[i]
        line = raw.split("!!")[0].strip()
        i += 1
        if not line or line.startswith("#"):
            continue
        words = line.split()
        key = words[0].upper()
        if key in _SCALE_KEYS:
            attr, idx = _SCALE_KEYS[key]
            getattr(ff, attr)[idx] = _scale(float(words[1]))
        elif key == "DIELECTRIC":
            ff.dielec = float(words[1])
        elif key == "POLARIZATION":
            ff.polarization = words[1].upper()
        elif key == "ATOM":
            m = re.match(r'\s*atom\s+(\d+)\s+(\d+)\s+(\S+)', raw, re.I)
            if m:
                ff.atoms[int(m.group(1))] = (int(m.group(2)), m.group(3))
        elif key == "MULTIPOLE":
            nums = [int(w) for w in words[1:-1]]
            t = nums[0]
            vals = [float(words[-1])]
            for _ in range(4):
                vals += [float(v) for v in lines[i].split("!!")[0].split()]
                i += 1
            if wanted_types is not None and t not in wanted_types:
                continue
            axes = tuple(nums[1:]) + (0,) * (3 - len(nums[1:]))
            c = vals[0]
            d = [v * BOHR for v in vals[1:4]]
            q = vals[4:10]  # qxx, qxy qyy, qxz qyz qzz (lower triangle by rows)
            f = BOHR * BOHR / 3.0
            qxx, qxy, qyy, qxz, qyz, qzz = [v * f for v in q]
            pole = [c] + d + [qxx, qxy, qxz, qxy, qyy, qyz, qxz, qyz, qzz]
            ff.multipoles.setdefault(t, []).append(MultipoleRecord((t,) + axes, pole))
        elif key == "POLARIZE":
            t = int(words[1])
            if wanted_types is not None and t not in wanted_types:
                continue
            # alpha, then optional thole and tholed (reals), then group types
            alpha, rest = float(words[2]), words[3:]
            reals = []
            while rest and ("." in rest[0] or "e" in rest[0].lower()) and len(reals) < 2:
                reals.append(float(rest[0]))
                rest = rest[1:]
            thl = reals[0] if reals else 0.0
            grp = [int(w) for w in rest]
            ff.polarize[t] = (alpha, thl, grp)
    return ff
