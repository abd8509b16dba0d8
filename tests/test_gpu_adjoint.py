"""The hand-written adjoint (amg_backward) against finite differences and the
analytic forces.

Configuration: the 216-water box (648 atoms, PME 24^3) with seeded per-type
1% Gaussian perturbations of the multipoles and polarizabilities, FP64,
mutual polarization converged to 1e-10 D.  Central differences of the
forward energy (step h) check d/d(pole), d/d(polarity) (through pdamp =
alpha^(1/6) as well), d/d(thole) and d/dx; the dipole cotangents check the
extra adjoint PCG solve.
"""
import copy

import numpy as np
import pytest

from polmdqc_b200 import abi, systems
from polmdqc_b200.engine import Engine, Settings

pytestmark = pytest.mark.gpu

FP64 = abi.PREC_FP64
ST = Settings(nfft=(24, 24, 24), precision=FP64, poleps=1e-10, politer=200)


def perturbed_box(seed=3):
    """216 waters with 1% per-type Gaussian perturbations of pole and polarity."""
    s = systems.water_box(216, 18.643, seed=0)
    rng = np.random.default_rng(seed)
    for t in np.unique(s.types):
        m = s.types == t
        s.pole[m] = s.pole[m] * (1 + 0.01 * rng.standard_normal(13))
        s.pole[m, 5], s.pole[m, 6], s.pole[m, 9] = s.pole[m, 7], s.pole[m, 10], s.pole[m, 11]  # keep Q symmetric
        tr = (s.pole[m, 4] + s.pole[m, 8] + s.pole[m, 12]) / 3                                  # and traceless
        s.pole[m, 4] -= tr; s.pole[m, 8] -= tr; s.pole[m, 12] -= tr
        s.polarity[m] = s.polarity[m] * (1 + 0.01 * rng.standard_normal())
        s.thole[m] = s.thole[m] * (1 + 0.01 * rng.standard_normal())
    s.pdamp = s.polarity ** (1 / 6)
    return s


def energy(s, flags=abi.DO_ENERGY, dipoles=False):
    e = Engine(s, ST)
    try:
        r = e.forward(flags | (abi.DO_DIPOLES if dipoles else 0))
    finally:
        e.close()
    return r


@pytest.fixture(scope="module")
def box():
    return perturbed_box()


@pytest.fixture(scope="module")
def grads(box):
    e = Engine(box, ST)
    try:
        r = e.forward(abi.DO_ENERGY | abi.DO_GRADIENT | abi.DO_DIPOLES)
        g = e.backward(d_energy=1.0)
    finally:
        e.close()
    return r, g


def fd(box, mutate, h):
    a, b = copy.deepcopy(box), copy.deepcopy(box)
    mutate(a, +h)
    mutate(b, -h)
    ea, eb = energy(a), energy(b)
    return ((ea.em + ea.ep) - (eb.em + eb.ep)) / (2 * h)


def test_coordinate_gradient_equals_forces(grads):
    r, g = grads
    np.testing.assert_allclose(g["d_xyz"], r.dem + r.dep, atol=1e-8, rtol=0)


# (atom, {pole entry: weight}): charges, dipoles, and symmetric traceless
# quadrupole directions (the gradient is defined on traceless quadrupoles)
DIRECTIONS = [(0, {0: 1.0}), (0, {3: 1.0}), (0, {4: 1.0, 8: -1.0}), (1, {1: 1.0}), (1, {12: 1.0, 4: -1.0}),
              (1, {5: 1.0, 7: 1.0}), (4, {9: 1.0, 11: 1.0}), (5, {3: 1.0})]


@pytest.mark.parametrize("atom,direction", DIRECTIONS)
def test_pole_gradient_matches_fd(box, grads, atom, direction):
    _, g = grads
    h = 1e-5

    def mutate(s, d):
        for c, w in direction.items():
            s.pole[atom, c] += w * d

    an = sum(w * g["d_pole"][atom, c] for c, w in direction.items())
    assert abs(fd(box, mutate, h) - an) < 1e-5 * max(1.0, abs(an))


@pytest.mark.parametrize("atom", [0, 1, 7])
def test_polarizability_and_thole_gradients_match_fd(box, grads, atom):
    _, g = grads
    h = 1e-5

    def mut_pol(s, d):
        s.polarity[atom] += d
        s.pdamp = s.polarity ** (1 / 6)

    def mut_thl(s, d):
        s.thole[atom] += d

    assert abs(fd(box, mut_pol, h) - g["d_polarity"][atom]) < 1e-5 * max(1.0, abs(g["d_polarity"][atom]))
    assert abs(fd(box, mut_thl, h) - g["d_thole"][atom]) < 1e-5 * max(1.0, abs(g["d_thole"][atom]))


def test_dipole_cotangents_need_the_adjoint_solve(box):
    """L = <g_d, uind> + <g_p, uinp>: the extra PCG solve A w = g."""
    rng = np.random.default_rng(11)
    gd = rng.standard_normal(3 * box.n)
    gp = rng.standard_normal(3 * box.n)
    e = Engine(box, ST)
    try:
        e.forward(abi.DO_ENERGY | abi.DO_GRADIENT | abi.DO_DIPOLES)
        g = e.backward(d_energy=0.0, d_uind=gd, d_uinp=gp)
    finally:
        e.close()

    def L(s):
        r = energy(s, dipoles=True)
        return gd @ r.uind.reshape(-1) + gp @ r.uinp.reshape(-1)

    h = 1e-5
    for atom, comp in ((0, 0), (2, 3)):
        a, b = copy.deepcopy(box), copy.deepcopy(box)
        a.pole[atom, comp] += h
        b.pole[atom, comp] -= h
        num = (L(a) - L(b)) / (2 * h)
        assert abs(num - g["d_pole"][atom, comp]) < 1e-5 * max(1.0, abs(num))
    a, b = copy.deepcopy(box), copy.deepcopy(box)
    a.polarity[3] += h
    b.polarity[3] -= h
    a.pdamp, b.pdamp = a.polarity ** (1 / 6), b.polarity ** (1 / 6)
    num = (L(a) - L(b)) / (2 * h)
    assert abs(num - g["d_polarity"][3]) < 1e-5 * max(1.0, abs(num))
    for atom, ax in ((3, 1),):
        a, b = copy.deepcopy(box), copy.deepcopy(box)
        a.xyz[atom, ax] += h
        b.xyz[atom, ax] -= h
        num = (L(a) - L(b)) / (2 * h)
        assert abs(num - g["d_xyz"][atom, ax]) < 1e-5 * max(1.0, abs(num))


# ---------------------------------------------------------------- torch.autograd
class _Selected:
    """A few scalar parameters of the box, as one vector theta: a charge, a
    dipole component, a polarizability (pdamp follows as alpha^(1/6)), a
    Thole factor and a coordinate."""
    SLOTS = (("pole", (0, 0)), ("pole", (1, 3)), ("polarity", (0,)), ("thole", (1,)), ("xyz", (2, 1)),
             ("polarity", (4,)))

    def __init__(self, box):
        self.box = box

    def values(self):
        return np.array([getattr(self.box, name)[idx] for name, idx in self.SLOTS])

    def system(self, theta):
        s = copy.deepcopy(self.box)
        for (name, idx), v in zip(self.SLOTS, theta):
            getattr(s, name)[idx] = v
        s.pdamp = s.polarity ** (1 / 6)
        return s

    @staticmethod
    def pick(g):
        full = {"pole": g["d_pole"], "polarity": g["d_polarity"], "thole": g["d_thole"], "xyz": g["d_xyz"]}
        return np.array([full[name][idx] for name, idx in _Selected.SLOTS])


def make_amoeba_function(sel, gd, gp):
    """torch.autograd.Function over the C ABI: forward = amg_forward (FP64),
    outputs E = em + ep and L = <gd, uind> + <gp, uinp>; backward =
    amg_backward with d_energy = dE and the dipole cotangents dL gd, dL gp
    (the adjoint PCG solve).  Test harness only: the library itself has no
    torch dependency."""
    import torch

    class AmoebaEnergy(torch.autograd.Function):
        @staticmethod
        def forward(ctx, theta):
            eng = Engine(sel.system(theta.detach().cpu().numpy()), ST)
            r = eng.forward(abi.DO_ENERGY | abi.DO_GRADIENT | abi.DO_DIPOLES)
            ctx.eng = eng
            E = r.em + r.ep
            L = gd @ r.uind.reshape(-1) + gp @ r.uinp.reshape(-1)
            return theta.new_tensor(E), theta.new_tensor(L)

        @staticmethod
        def backward(ctx, dE, dL):
            # the context stays open for repeated backward calls on one
            # forward (gradcheck makes one per output); Engine closes it when
            # the autograd node is released
            cE = 0.0 if dE is None else float(dE)
            cL = 0.0 if dL is None else float(dL)
            g = ctx.eng.backward(d_energy=cE, d_uind=cL * gd, d_uinp=cL * gp)
            return torch.tensor(_Selected.pick(g), dtype=torch.float64)

    return AmoebaEnergy


def test_autograd_function_gradcheck(box):
    """torch.autograd.gradcheck of the wrapped forward/backward against
    central differences (step 1e-4) of the GPU's own FP64 forward, for both
    outputs (energy, and a dipole functional that needs the adjoint solve)."""
    import torch
    rng = np.random.default_rng(5)
    gd, gp = rng.standard_normal(3 * box.n), rng.standard_normal(3 * box.n)
    sel = _Selected(box)
    fn = make_amoeba_function(sel, gd, gp)
    theta = torch.tensor(sel.values(), dtype=torch.float64, requires_grad=True)
    assert torch.autograd.gradcheck(fn.apply, (theta,), eps=1e-4, atol=1e-4, rtol=1e-5, nondet_tol=1e-7)


def test_adjoint_matches_oracle_finite_differences(box, grads):
    """Parameter gradients of amg_backward against central differences of the
    FP64 CPU oracle's energies (not the GPU's): a charge, a dipole component,
    a polarizability, a Thole factor and a coordinate, 1e-5 relative."""
    from oracle import oracle
    _, g = grads
    sel = _Selected(box)
    theta0 = sel.values()
    an = _Selected.pick(g)
    h = 1e-5
    for k in range(len(theta0)):
        tp, tm = theta0.copy(), theta0.copy()
        tp[k] += h
        tm[k] -= h
        ep = oracle.forward(sel.system(tp), ST, tol=1e-12, flags=abi.DO_ENERGY)
        em = oracle.forward(sel.system(tm), ST, tol=1e-12, flags=abi.DO_ENERGY)
        num = ((ep.em + ep.ep) - (em.em + em.ep)) / (2 * h)
        assert abs(num - an[k]) < 1e-5 * max(1.0, abs(num)), (k, num, an[k])


# ---------------------------------------------------------------- OPT
@pytest.mark.parametrize("order", [2, 4])
def test_opt_adjoint_matches_fd(box, order):
    """The adjoint of the OPT dipoles (extrapolated perturbation theory, no
    solve: the cotangents pass through the same polynomial in alpha T),
    against central differences of the GPU's FP64 forward: coordinates equal
    the forces; a charge, a dipole component, a polarizability and a Thole
    factor; and a dipole functional L = <gd, uind> + <gp, uinp>."""
    st = Settings(nfft=(24, 24, 24), precision=FP64, poltyp=abi.POL_OPT, opt_order=order)
    rng = np.random.default_rng(7)
    gd, gp = rng.standard_normal(3 * box.n), rng.standard_normal(3 * box.n)
    e = Engine(box, st)
    try:
        r = e.forward(abi.DO_ENERGY | abi.DO_GRADIENT | abi.DO_DIPOLES)
        g = e.backward(d_energy=1.0)
        gl = e.backward(d_energy=0.0, d_uind=gd, d_uinp=gp)
    finally:
        e.close()
    np.testing.assert_allclose(g["d_xyz"], r.dem + r.dep, atol=1e-8, rtol=0)

    def eval_(s):
        eng = Engine(s, st)
        try:
            q = eng.forward(abi.DO_ENERGY | abi.DO_DIPOLES)
        finally:
            eng.close()
        return q.em + q.ep, gd @ q.uind.reshape(-1) + gp @ q.uinp.reshape(-1)

    sel = _Selected(box)
    theta0 = sel.values()
    an_e, an_l = _Selected.pick(g), _Selected.pick(gl)
    h = 1e-5
    for k in range(len(theta0)):
        tp, tm = theta0.copy(), theta0.copy()
        tp[k] += h
        tm[k] -= h
        (ep_, lp), (em_, lm) = eval_(sel.system(tp)), eval_(sel.system(tm))
        ne, nl = (ep_ - em_) / (2 * h), (lp - lm) / (2 * h)
        assert abs(ne - an_e[k]) < 1e-5 * max(1.0, abs(ne)), (k, ne, an_e[k])
        assert abs(nl - an_l[k]) < 1e-5 * max(1.0, abs(nl)), (k, nl, an_l[k])


def test_mixed_precision_adjoint_matches_fp64(box):
    """The adjoint of a mixed-precision context: the adjoint solve runs in FP32
    on the forward's stored coefficient rows (FP64 dot products and norms, one
    FP64 correction sweep, 1e-6 D as the metric's forward), every other term in
    FP64.  Against the FP64 adjoint converged to 1e-10 D: every gradient
    (multipoles, polarizabilities, Thole factors, coordinates), for the energy
    and for a dipole functional, within 1e-5 of the array's largest entry; the
    coordinate gradient within the forward's force target (1e-4 kcal/mol/A
    RMS) of the FP64 forces."""
    rng = np.random.default_rng(5)
    gd, gp = rng.standard_normal(3 * box.n), rng.standard_normal(3 * box.n)
    out = {}
    for name, st in (("fp64", ST), ("mixed", Settings(nfft=(24, 24, 24), precision=abi.PREC_MIXED))):
        e = Engine(box, st)
        try:
            r = e.forward(abi.DO_ENERGY | abi.DO_GRADIENT | abi.DO_DIPOLES)
            out[name] = (r, e.backward(d_energy=1.0), e.backward(d_energy=0.0, d_uind=gd, d_uinp=gp),
                         e.backward(d_energy=1.0))
        finally:
            e.close()
    r32, g32, l32, again = out["mixed"]
    r64, g64, l64, _ = out["fp64"]
    assert np.sqrt(np.mean((g32["d_xyz"] - (r64.dem + r64.dep)) ** 2)) < 1e-4
    for k in ("d_pole", "d_polarity", "d_thole", "d_xyz"):
        scale = np.abs(g64[k]).max()
        # a second call agrees to the rounding of the FP32 atomic PME
        # spreading (the potentials' last bits, 1e-7 of their size)
        assert np.abs(again[k] - g32[k]).max() <= 2e-6 * scale, k
        for a, b in ((g32, g64), (l32, l64)):
            scale = np.abs(b[k]).max()
            assert np.abs(a[k] - b[k]).max() <= 1e-5 * scale, (k, np.abs(a[k] - b[k]).max(), scale)
