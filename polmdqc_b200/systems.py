"""Systems for the electrostatics path: seeded synthetic boxes and the
host-side parameter assignment that feeds amg_params.

A `System` holds exactly the inputs the reference's empole/epolar read after
mechanic() (atoms.h, mpole.h, polar.h, couple.h, polgrp.h and the scale
factors), as numpy arrays in the reference's conventions.  Two sources:

  * `water_box` / `ion_solution`: seeded synthetic inputs with the shapes of
    the benchmark configurations (rigid AMOEBA water on a jittered cubic
    lattice, uniform random orientations, O-H 0.9572 A, H-O-H 104.52 deg),
    parameters assigned here for water and monatomic ions, restating
    kmpole's frame assignment (src/md/kmpole.cpp) for these two molecule
    kinds and polargrp's group building (src/md/kpolar.cpp:592-853);
  * `from_dump`: the globals printed by the reference itself (test fixtures).
"""
from __future__ import annotations

import dataclasses
import json
import math
import os

import numpy as np

from . import abi
from . import prm as prm_mod

DATA = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data")

OH = 0.9572                    # water03.prm bond length
HOH = 104.52                   # rigid water angle (degrees)


@dataclasses.dataclass
class System:
    n: int
    xyz: np.ndarray            # [n,3] float64
    types: np.ndarray          # [n] int32 force-field atom types
    names: list
    bonds: list                # per atom: list of bonded atoms (0-based)
    pole: np.ndarray           # [n,13] local frame
    zaxis: np.ndarray          # [n] 1-based
    xaxis: np.ndarray
    yaxis: np.ndarray
    polaxe: np.ndarray
    molcule: np.ndarray
    polarity: np.ndarray
    thole: np.ndarray
    pdamp: np.ndarray
    lists: dict                # 'i12'..'i15', 'ip11'..'ip14': list of lists
    m_scale: list
    p_scale: list
    p_iscale: list
    d_scale: list
    u_scale: list
    box: np.ndarray            # [6] a,b,c,alpha,beta,gamma (zeros: no box)
    use_bounds: bool
    prm_name: str = ""
    cell_shape: int = 0        # abi.CELL_*: octahedron / dodecahedron, else from the angles
    # charge penetration (chgpen.h) and charge flux (cflux.h, bndstr.h, angbnd.h)
    pentype: int = 0           # abi.PEN_*
    pcore: np.ndarray = None   # [n] core charges
    palpha: np.ndarray = None  # [n] valence damping exponents
    cflux: bool = False        # monopoles follow the geometry; pole[:, 0] is then mono0
    bond_atoms: np.ndarray = None   # [nbond, 2] 0-based
    bond_flux: np.ndarray = None    # [nbond, 2] ideal length, flux
    angle_atoms: np.ndarray = None  # [nangle, 3] 0-based a, b (vertex), c
    angle_flux: np.ndarray = None   # [nangle, 7] theta0 (deg), r0_ab, r0_cb, pa1, pa2, pb1, pb2

    def csr(self, name):
        lists = self.lists[name]
        off = np.zeros(self.n + 1, np.int32)
        off[1:] = np.cumsum([len(l) for l in lists])
        idx = np.array([k for l in lists for k in l], np.int32)
        return off, idx


# ----------------------------------------------------------------- topology
def neighbor_shells(bonds):
    """1-2 .. 1-5 lists from bonds, each shell excluding atoms already in a
    closer shell or the atom itself (src/md/attach.cpp)."""
    n = len(bonds)
    i12 = [sorted(b) for b in bonds]
    shells = [i12]
    for _ in range(3):
        prev = shells[-1]
        nxt = []
        for i in range(n):
            seen = {i}
            for s in shells:
                seen.update(s[i])
            cand = set()
            for j in prev[i]:
                for k in i12[j]:
                    if k not in seen:
                        cand.add(k)
            nxt.append(sorted(cand))
        shells.append(nxt)
    return shells


def polarization_groups(types, bonds, polarize):
    """Group lists ip11..ip14 (src/md/kpolar.cpp:592-853 restated): atoms
    bonded to i whose type is listed in i's polarize record share i's group;
    groups are closed transitively; ip1n+1 holds atoms of groups bonded to
    the groups in ip1n."""
    n = len(types)
    grp = [-1] * n
    ng = 0
    for i in range(n):
        if grp[i] >= 0:
            continue
        grp[i] = ng
        stack = [i]
        while stack:
            a = stack.pop()
            partners = polarize.get(int(types[a]), (0, 0, []))[2]
            for b in bonds[a]:
                if grp[b] < 0 and int(types[b]) in partners:
                    grp[b] = ng
                    stack.append(b)
        ng += 1
    members = [[] for _ in range(ng)]
    for i in range(n):
        members[grp[i]].append(i)
    gbond = [set() for _ in range(ng)]
    for i in range(n):
        for b in bonds[i]:
            if grp[b] != grp[i]:
                gbond[grp[i]].add(grp[b])
    ip = []
    for level in range(4):
        cur = []
        for i in range(n):
            if level == 0:
                gs = {grp[i]}
            else:
                # groups reachable in exactly `level` group bonds
                frontier, seen = {grp[i]}, {grp[i]}
                for _ in range(level):
                    nxt = set()
                    for g in frontier:
                        nxt |= gbond[g]
                    nxt -= seen
                    seen |= nxt
                    frontier = nxt
                gs = frontier
            cur.append(sorted(a for g in gs for a in members[g]))
        ip.append(cur)
    return ip


# ----------------------------------------------------------------- builders
def random_rotations(rng, m):
    """Uniform random rotation matrices (quaternion method)."""
    u1, u2, u3 = rng.random(m), rng.random(m), rng.random(m)
    q = np.stack([np.sqrt(1 - u1) * np.sin(2 * np.pi * u2), np.sqrt(1 - u1) * np.cos(2 * np.pi * u2),
                  np.sqrt(u1) * np.sin(2 * np.pi * u3), np.sqrt(u1) * np.cos(2 * np.pi * u3)], axis=1)
    x, y, z, w = q.T
    R = np.empty((m, 3, 3))
    R[:, 0, 0] = 1 - 2 * (y * y + z * z); R[:, 0, 1] = 2 * (x * y - z * w); R[:, 0, 2] = 2 * (x * z + y * w)
    R[:, 1, 0] = 2 * (x * y + z * w); R[:, 1, 1] = 1 - 2 * (x * x + z * z); R[:, 1, 2] = 2 * (y * z - x * w)
    R[:, 2, 0] = 2 * (x * z - y * w); R[:, 2, 1] = 2 * (y * z + x * w); R[:, 2, 2] = 1 - 2 * (x * x + y * y)
    return R


def water_geometry(O, R):
    h = math.radians(HOH) / 2
    loc = np.array([[OH * math.sin(h), 0, OH * math.cos(h)], [-OH * math.sin(h), 0, OH * math.cos(h)]])
    H = np.einsum("mij,kj->mki", R, loc)
    return O[:, None, :] + H


def load_forcefield(name):
    """Parameter subset shipped with the package (polmdqc_b200/data/*.json,
    generated from the reference's .prm files by data/make_params.py)."""
    with open(os.path.join(DATA, f"{name}.json")) as f:
        d = json.load(f)
    ff = prm_mod.ForceField()
    ff.atoms = {int(k): tuple(v) for k, v in d["atoms"].items()}
    ff.multipoles = {int(k): [prm_mod.MultipoleRecord(tuple(r["types"]), r["pole"]) for r in v]
                     for k, v in d["multipoles"].items()}
    ff.polarize = {int(k): (v[0], v[1], v[2]) for k, v in d["polarize"].items()}
    for key in ("m_scale", "p_scale", "p_iscale", "d_scale", "u_scale"):
        setattr(ff, key, d[key])
    ff.dielec = d["dielec"]
    ff.polarization = d["polarization"]
    return ff


WATER_TYPES = {"water03": (1, 2), "amoebabio18": (349, 350)}
ION_TYPES = {"amoebabio18": {"Na+": 352, "Cl-": 363}}


def assign(xyz, types, names, bonds, mol, ff, box, use_bounds, prm_name):
    """Frame and parameter assignment for water (O bisector of its two H;
    H z-then-x on O and the other H) and monatomic ions (no frame), restating
    the matches kmpole makes for these records (src/md/kmpole.cpp)."""
    n = len(types)
    pole = np.zeros((n, 13))
    zax = np.zeros(n, np.int32)
    xax = np.zeros(n, np.int32)
    yax = np.zeros(n, np.int32)
    axe = np.zeros(n, np.int32)
    for i in range(n):
        t = int(types[i])
        rec = ff.multipoles[t][0]
        pole[i] = rec.pole
        _, zt, xt, yt = rec.types
        if zt == 0:
            continue
        nb = bonds[i]
        if len(nb) == 2 and zt < 0 and xt < 0:            # O: bisector of the two H
            zax[i], xax[i] = nb[0] + 1, nb[1] + 1
            axe[i] = 3
        elif len(nb) == 1:                                  # H: z on O, x on the other H
            o = nb[0]
            other = [k for k in bonds[o] if k != i][0]
            zax[i], xax[i] = o + 1, other + 1
            axe[i] = 1
        else:
            raise ValueError(f"frame assignment not restated for type {t}")
    pol = np.array([ff.polarize[int(t)][0] for t in types])
    thl = np.array([ff.polarize[int(t)][1] for t in types])
    pdamp = pol ** (1.0 / 6.0)
    shells = neighbor_shells(bonds)
    ip = polarization_groups(types, bonds, ff.polarize)
    lists = {"i12": shells[0], "i13": shells[1], "i14": shells[2], "i15": shells[3],
             "ip11": ip[0], "ip12": ip[1], "ip13": ip[2], "ip14": ip[3]}
    return System(n=n, xyz=np.ascontiguousarray(xyz, np.float64), types=np.asarray(types, np.int32),
                  names=names, bonds=bonds, pole=pole, zaxis=zax, xaxis=xax, yaxis=yax, polaxe=axe,
                  molcule=np.asarray(mol, np.int32), polarity=pol, thole=thl, pdamp=pdamp, lists=lists,
                  m_scale=list(ff.m_scale), p_scale=list(ff.p_scale), p_iscale=list(ff.p_iscale),
                  d_scale=list(ff.d_scale), u_scale=list(ff.u_scale),
                  box=np.asarray(box, np.float64), use_bounds=use_bounds, prm_name=prm_name)


def water_box(n_waters: int, box_len: float, seed: int = 0, prm: str = "water03",
              jitter: float = 0.3) -> System:
    """n_waters rigid AMOEBA waters: O on a jittered cubic lattice (uniform
    +/- jitter), uniform random orientations (seed + 1)."""
    side = int(round(n_waters ** (1 / 3)))
    if side ** 3 != n_waters:
        side = int(math.ceil(n_waters ** (1 / 3)))
    rng = np.random.default_rng(seed)
    a = box_len / side
    grid = np.stack(np.meshgrid(*[np.arange(side)] * 3, indexing="ij"), -1).reshape(-1, 3)[:n_waters]
    O = (grid + 0.5) * a + rng.uniform(-jitter, jitter, (n_waters, 3))
    H = orient_waters(O, box_len, np.random.default_rng(seed + 1))
    return _assemble_waters(O, H, [], box_len, prm)


def orient_waters(O, box_len, rng, fixed=(), min_contact=1.7, tries=200):
    """Uniform random orientations, redrawn (up to `tries` times) for a water
    whose H would come closer than `min_contact` Angstrom to an atom of an
    already placed water or to a fixed site (ions): the lattice spacing is
    ~3.1 A, so unconditioned draws can put H at < 1 A from a neighbour."""
    m = len(O)
    H = np.zeros((m, 2, 3))
    fixed = np.asarray(fixed, np.float64).reshape(-1, 3)
    cell = 3.5
    nc = max(1, int(box_len // cell))
    size = box_len / nc
    # placed atoms binned on a periodic grid of cells >= 3.5 A: positions
    # [nc, nc, nc, cap, 3] and counts per cell; a candidate is tested against
    # the 27 cells around its own
    cap = 16
    pos = np.zeros((nc, nc, nc, cap, 3))
    cnt = np.zeros((nc, nc, nc), np.int64)
    offs = np.array([(dx, dy, dz) for dx in (-1, 0, 1) for dy in (-1, 0, 1) for dz in (-1, 0, 1)])
    thr = min_contact * min_contact

    def key(p):
        return (np.floor((p % box_len) / size).astype(int)) % nc

    def add(p):
        nonlocal pos, cap
        k = tuple(key(p))
        if cnt[k] == cap:
            grown = np.zeros((nc, nc, nc, 2 * cap, 3))
            grown[:, :, :, :cap] = pos
            pos, cap = grown, 2 * cap
        pos[k + (cnt[k],)] = p
        cnt[k] += 1

    def clash(atoms):
        for atom in atoms:
            nb = (key(atom) + offs) % nc
            c = cnt[nb[:, 0], nb[:, 1], nb[:, 2]]
            q = pos[nb[:, 0], nb[:, 1], nb[:, 2]][np.arange(cap)[None, :] < c[:, None]]
            d = atom - q
            d -= box_len * np.round(d / box_len)
            if np.any(d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1] + d[:, 2] * d[:, 2] < thr):
                return True
        return False

    for p in fixed:
        add(p)
    for w in range(m):
        for t in range(tries):
            R = random_rotations(rng, 1)
            h = water_geometry(O[w:w + 1], R)[0]
            ok = not clash((h[0], h[1], O[w]))
            if ok or t == tries - 1:
                break
        H[w] = h
        for atom in (O[w], h[0], h[1]):
            add(atom)
    return H


def _assemble_waters(O, H, ions, box_len, prm):
    ot, ht = WATER_TYPES[prm]
    xyz, types, names, bonds, mol = [], [], [], [], []
    for w in range(len(O)):
        b = len(xyz)
        xyz += [O[w], H[w, 0], H[w, 1]]
        types += [ot, ht, ht]
        names += ["O", "H", "H"]
        bonds += [[b + 1, b + 2], [b], [b]]
        mol += [w] * 3
    for k, (pos, t, name) in enumerate(ions):
        xyz.append(pos)
        types.append(t)
        names.append(name)
        bonds.append([])
        mol.append(len(O) + k)
    ff = load_forcefield(prm)
    box = [box_len] * 3 + [90.0] * 3
    return assign(np.array(xyz), np.array(types), names, bonds, mol, ff, box, True, prm)


def prism_edges(cell_shape: int, L: float) -> np.ndarray:
    """Edges of the orthogonal prism that encloses two cells of a truncated
    octahedron (a cube of edge L) or a rhombic dodecahedron (L x L x sqrt(2) L:
    the reference's image wraps z by sqrt(2) times the box length,
    src/md/image.cpp:109-121)."""
    return np.array([L, L, L * (math.sqrt(2.0) if cell_shape == abi.CELL_DODECAHEDRON else 1.0)])


def cell_image(d: np.ndarray, cell_shape: int, L: float) -> np.ndarray:
    """Minimum image of difference vectors d [m, 3] in a truncated octahedron
    or rhombic dodecahedron of box length L, the reference's image()
    (src/md/image.cpp:92-121) in vector form."""
    d = np.array(d, np.float64, copy=True)
    if cell_shape == abi.CELL_OCTAHEDRON:
        d -= L * np.rint(d / L)
        far = np.abs(d).sum(axis=1) > 0.75 * L
        d[far] -= np.copysign(0.5 * L, d[far])
        return d
    r2 = math.sqrt(2.0)
    d[:, :2] -= L * np.rint(d[:, :2] / L)
    d[:, 2] -= r2 * L * np.rint(d[:, 2] / (r2 * L))
    corr = 0.5 * L * np.floor(np.abs(d[:, 0] / L) + np.abs(d[:, 1] / L) + np.abs(r2 * d[:, 2] / L))
    d[:, 0] -= np.copysign(corr, d[:, 0])
    d[:, 1] -= np.copysign(corr, d[:, 1])
    d[:, 2] -= np.copysign(corr, d[:, 2]) * r2
    return d


def water_cell(cell_shape: int, L: float = 24.8, seed: int = 0, jitter: float = 0.25, prm: str = "water03",
               min_contact: float = 1.7, tries: int = 200, per_edge: int = 8) -> System:
    """Rigid AMOEBA waters filling a truncated octahedron or a rhombic
    dodecahedron of box length L.  O sit on a jittered lattice of the
    enclosing prism (`per_edge` sites per L along x and y, an even number; as
    many along z for the octahedron, 1.5 times as many along the
    dodecahedron's sqrt(2) L), one of each pair of
    sites that the cell's centring translation (half of every prism edge)
    exchanges, so the periodic images complete the lattice; orientations are
    uniform random, redrawn while an atom comes within `min_contact` of
    another molecule's atom under the cell's minimum image."""
    edges = prism_edges(cell_shape, L)
    m = per_edge
    nz = 3 * m // 2 if cell_shape == abi.CELL_DODECAHEDRON else m
    steps = edges / np.array([m, m, nz])
    grid = np.stack(np.meshgrid(np.arange(m // 2), np.arange(m), np.arange(nz), indexing="ij"), -1).reshape(-1, 3)
    rng = np.random.default_rng(seed)
    O = (grid + 0.5) * steps - 0.5 * edges + rng.uniform(-jitter, jitter, (len(grid), 3))
    orng = np.random.default_rng(seed + 1)
    placed = np.zeros((0, 3))
    H = np.zeros((len(O), 2, 3))
    for w in range(len(O)):
        for t in range(tries):
            h = water_geometry(O[w:w + 1], random_rotations(orng, 1))[0]
            atoms = np.vstack([O[w:w + 1], h])
            if len(placed) == 0 or t == tries - 1:
                break
            d = cell_image((atoms[:, None, :] - placed[None, :, :]).reshape(-1, 3), cell_shape, L)
            if np.min(np.einsum("ij,ij->i", d, d)) >= min_contact * min_contact:
                break
        H[w] = h
        placed = np.vstack([placed, atoms])
    s = _assemble_waters(O, H, [], L, prm)
    s.cell_shape = cell_shape
    return s


def doubled_prism(s: System) -> System:
    """The same periodic system written as an orthogonal prism holding two
    copies of the cell (the atoms and their images under the centring
    translation): a truncated octahedron's lattice is the cube's plus the
    body centre, a rhombic dodecahedron's the L x L x sqrt(2) L prism's plus
    its centre.  Every pair sum over the cell's lattice is half the prism's,
    so the prism gives twice the cell's energies and, on each copy, the
    cell's forces and dipoles."""
    L = float(s.box[0])
    edges = prism_edges(s.cell_shape, L)
    n = s.n
    shift = 0.5 * edges
    xyz = np.vstack([s.xyz, s.xyz + shift])

    def ax(a):
        a = np.asarray(a)
        return np.concatenate([a, np.where(a > 0, a + n, 0)]).astype(a.dtype)

    lists = {k: [list(v) for v in vals] + [[j + n for j in v] for v in vals] for k, vals in s.lists.items()}
    mol = np.concatenate([s.molcule, s.molcule + int(s.molcule.max()) + 1])
    return dataclasses.replace(
        s, n=2 * n, xyz=xyz, types=np.concatenate([s.types, s.types]), names=list(s.names) * 2,
        bonds=[list(b) for b in s.bonds] + [[j + n for j in b] for b in s.bonds], pole=np.vstack([s.pole, s.pole]),
        zaxis=ax(s.zaxis), xaxis=ax(s.xaxis), yaxis=ax(s.yaxis), polaxe=np.concatenate([s.polaxe, s.polaxe]),
        molcule=mol, polarity=np.concatenate([s.polarity, s.polarity]), thole=np.concatenate([s.thole, s.thole]),
        pdamp=np.concatenate([s.pdamp, s.pdamp]), lists=lists,
        box=np.array([*edges, 90.0, 90.0, 90.0]), cell_shape=abi.CELL_FROM_ANGLES)


def ion_solution(n_waters=8000, n_pairs=22, box_len=62.1, seed=0, jitter=0.3) -> System:
    """Waters plus Na+/Cl- pairs (amoebabio18 types 349/350/352/363) on a
    cubic lattice: ion sites are random lattice sites; their face neighbours
    stay empty, so every ion is >= 3 A from every water O."""
    side = int(math.ceil((n_waters + 7 * 2 * n_pairs) ** (1 / 3)))
    rng = np.random.default_rng(seed)
    a = box_len / side
    nsite = side ** 3
    order = rng.permutation(nsite)
    coords = np.stack(np.unravel_index(np.arange(nsite), (side,) * 3), -1)
    blocked = np.zeros(nsite, bool)
    ion_sites = []
    for s_ in order:
        if len(ion_sites) == 2 * n_pairs:
            break
        if blocked[s_]:
            continue
        ion_sites.append(s_)
        c = coords[s_]
        for d in [(0, 0, 0), (1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1)]:
            nb = (c + d) % side
            blocked[np.ravel_multi_index(nb, (side,) * 3)] = True
    free = [s_ for s_ in rng.permutation(nsite) if not blocked[s_]][:n_waters]
    if len(free) < n_waters:
        raise ValueError("box too small for the requested waters and ions")
    free = np.sort(np.array(free))
    O = (coords[free] + 0.5) * a + rng.uniform(-jitter, jitter, (n_waters, 3))
    ions = []
    for k, s_ in enumerate(ion_sites):
        t = 352 if k % 2 == 0 else 363
        ions.append(((coords[s_] + 0.5) * a, t, "Na+" if t == 352 else "Cl-"))
    H = orient_waters(O, box_len, np.random.default_rng(seed + 1), fixed=[p for p, _, _ in ions])
    return _assemble_waters(O, H, ions, box_len, "amoebabio18")


def from_dump(d: dict, prm_name: str = "") -> System:
    """System from the reference's own globals (oracle/ref_dump JSON)."""
    n = d["n"]
    xyz = np.stack([d["x"], d["y"], d["z"]], 1)
    bonds = [list(b) for b in d["i12"]]
    has_pol = "polarity" in d
    lists = {k: d[k] for k in ("i12", "i13", "i14", "i15")}
    for k in ("ip11", "ip12", "ip13", "ip14"):
        lists[k] = d.get(k, [[] for _ in range(n)])
    box = np.array(d["box"], np.float64)
    pole = np.array(d["pole"]).reshape(n, 13)
    cp = {}
    if d.get("pentype", 0):
        cp.update(pentype=int(d["pentype"]), pcore=np.array(d["pcore"]), palpha=np.array(d["palpha"]))
    if d.get("use_chgflx", 0):
        pole[:, 0] = d["mono0"]          # the dump's pole holds the monopoles altered for its geometry
        nb, na = d["nbond"], d["nangle"]
        cp.update(cflux=True, bond_atoms=np.array(d["ibnd"], np.int32).reshape(nb, 2),
                  bond_flux=np.stack([d["bl"], d["bflx"]], 1).reshape(nb, 2),
                  angle_atoms=np.array(d["iang"], np.int32).reshape(na, 3),
                  angle_flux=np.concatenate([np.array(d["anat"]).reshape(na, 1), np.array(d["rab0"]).reshape(na, 1),
                                             np.array(d["rcb0"]).reshape(na, 1), np.array(d["aflx"]).reshape(na, 2),
                                             np.array(d["abflx"]).reshape(na, 2)], 1))
    return System(n=n, xyz=xyz, types=np.array(d["type"], np.int32), names=[""] * n, bonds=bonds,
                  pole=pole, zaxis=np.array(d["zaxis"], np.int32),
                  xaxis=np.array(d["xaxis"], np.int32), yaxis=np.array(d["yaxis"], np.int32),
                  polaxe=np.array(d["polaxe"], np.int32), molcule=np.array(d["molcule"], np.int32),
                  polarity=np.array(d["polarity"]) if has_pol else np.zeros(n),
                  thole=np.array(d["thole"]) if has_pol else np.zeros(n),
                  pdamp=np.array(d["pdamp"]) if has_pol else np.zeros(n),
                  lists=lists, m_scale=d["mscale"], p_scale=d["pscale"], p_iscale=d["piscale"],
                  d_scale=d["dscale"], u_scale=d["uscale"], box=box,
                  use_bounds=bool(d["use_bounds"]), prm_name=prm_name,
                  cell_shape=(abi.CELL_OCTAHEDRON if d.get("octahedron") else
                              abi.CELL_DODECAHEDRON if d.get("dodecadron") else abi.CELL_FROM_ANGLES), **cp)


def write_tinker(sys_: System, xyz_path: str, key_path: str, prm_path: str, keys: list):
    """Tinker .xyz + .key pair for running the reference on the same system."""
    with open(xyz_path, "w") as f:
        f.write(f"{sys_.n:6d}  synthetic\n")
        for i in range(sys_.n):
            x, y, z = sys_.xyz[i]
            nb = "".join(f"{k + 1:6d}" for k in sys_.bonds[i])
            f.write(f"{i + 1:6d}  {sys_.names[i] or 'X':3s} {x:12.6f}{y:12.6f}{z:12.6f}{sys_.types[i]:6d}{nb}\n")
    with open(key_path, "w") as f:
        f.write(f"parameters {prm_path}\n")
        if sys_.use_bounds:
            f.write(f"a-axis {sys_.box[0]:.6f}\n")
        for k in keys:
            f.write(k + "\n")
