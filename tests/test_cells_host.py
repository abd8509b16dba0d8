"""Host-side checks of the octahedron and dodecahedron test inputs: the
doubled prism (`systems.doubled_prism`) sees every pair at the distance the
cell's own minimum image gives (the reference's image(),
src/md/image.cpp:92-121), and the seeded cells have no close contacts."""
import numpy as np
import pytest

from polmdqc_b200 import abi, systems


@pytest.mark.parametrize("shape", [abi.CELL_OCTAHEDRON, abi.CELL_DODECAHEDRON])
def test_doubled_prism_reproduces_the_cell_image(shape):
    s = systems.water_cell(shape, seed=2)
    d = systems.doubled_prism(s)
    assert d.n == 2 * s.n and d.cell_shape == abi.CELL_FROM_ANGLES
    rng = np.random.default_rng(0)
    i, j = rng.integers(0, s.n, 500), rng.integers(0, s.n, 500)
    rc = np.linalg.norm(systems.cell_image(s.xyz[j] - s.xyz[i], shape, s.box[0]), axis=1)
    E = d.box[:3]

    def img(v):
        return v - E * np.rint(v / E)

    a = np.linalg.norm(img(d.xyz[j] - d.xyz[i]), axis=1)
    b = np.linalg.norm(img(d.xyz[j + s.n] - d.xyz[i]), axis=1)
    np.testing.assert_allclose(np.minimum(a, b), rc, atol=1e-12, rtol=0)
    # the copy's topology follows the original's
    assert d.zaxis[s.n] == s.zaxis[0] + s.n and d.lists["i12"][s.n] == [k + s.n for k in s.lists["i12"][0]]


@pytest.mark.parametrize("shape", [abi.CELL_OCTAHEDRON, abi.CELL_DODECAHEDRON])
def test_water_cell_has_no_close_contacts(shape):
    s = systems.water_cell(shape, seed=2)
    mol = s.molcule
    dv = systems.cell_image((s.xyz[:, None, :] - s.xyz[None, :, :]).reshape(-1, 3), shape, s.box[0])
    r = np.linalg.norm(dv, axis=1).reshape(s.n, s.n)
    r[mol[:, None] == mol[None, :]] = np.inf
    assert r.min() >= 1.7 - 1e-9


def centred_stencil_candidates(x, shape, L, cut):
    """The candidate search of the list kernel's centred mode, restated: atoms
    wrapped into the enclosing prism, binned in an even count (at least 6) of
    cells per axis; for a home atom the 27 cells around its cell and the 27
    around the cell half a prism away, each candidate's position moved by the
    stencil's translation (the centring translation, half of every edge, and
    the prism's wrap).  Returns per atom {candidate: displacement}."""
    P = systems.prism_edges(shape, L)
    nc = np.floor(P / cut).astype(int) & ~1
    assert (nc >= 6).all()
    size = P / nc
    xw = x - P * np.floor(x / P)
    cell = np.minimum(nc - 1, (xw / size).astype(int))
    members = {}
    for i, c in enumerate(map(tuple, cell)):
        members.setdefault(c, []).append(i)
    out = []
    for i in range(len(x)):
        cc = cell[i]
        cands = {}
        for half in (0, 1):
            for d in np.stack(np.meshgrid(*[np.arange(-1, 2)] * 3, indexing="ij"), -1).reshape(-1, 3):
                q = cc + (nc // 2 if half else 0) + d
                sh = -0.5 * P if half else np.zeros(3)
                sh = sh - (q < 0) * P + (q >= nc) * P
                q = q % nc
                for k in members.get(tuple(q), []):
                    assert k not in cands, "a site is a candidate twice"
                    cands[k] = xw[k] + sh - xw[i]
        out.append(cands)
    return out


@pytest.mark.parametrize("shape,L,cut", [(abi.CELL_OCTAHEDRON, 43.0, 7.0), (abi.CELL_DODECAHEDRON, 42.5, 7.0),
                                         (abi.CELL_OCTAHEDRON, 60.0, 9.5)])
def test_centred_stencil_finds_every_pair_once(shape, L, cut):
    """Every pair within the cutoff under the cell's image() (any image) is a
    candidate exactly once, at the image's displacement: the premise of the
    list kernel's centred mode (truncated octahedron, rhombic dodecahedron)."""
    rng = np.random.default_rng(7)
    x = rng.uniform(0.0, 1.0, (400, 3)) * systems.prism_edges(shape, L)
    cands = centred_stencil_candidates(x, shape, L, cut)
    pairs = 0
    for i in range(len(x)):
        d = systems.cell_image(x - x[i], shape, L)
        for k in np.nonzero((np.linalg.norm(d, axis=1) <= cut) & (np.arange(len(x)) != i))[0]:
            assert k in cands[i], (i, k)
            np.testing.assert_allclose(cands[i][k], d[k], atol=1e-9)
            pairs += 1
    assert pairs > 1000
