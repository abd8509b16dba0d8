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
