// polmdqc_shim.cpp -- drop-in replacement of the reference's electrostatics
// entry points, running them on the B200 through libamoeba_gpu.so.
//
// Link order: this file + the reference library built without empole.o
// (src/md/empole.cpp) + libamoeba_gpu.so.  It defines
//
//   template <CalcMode M> void polmdqc::empole();   replaces src/md/empole.cpp:49-83
//   template <CalcMode M> void polmdqc::epolar();   the term whose call is commented
//                                                   out at src/md/energy.cpp:267
//
// with the reference's explicit instantiations (src/md/empole.cpp:371-374).
// empole<M>() evaluates the whole electrostatic path in one device call: em
// (and its gradient, per-atom energies, pair count, intermolecular energy) and,
// when polarization is active (use_polar), ep, dep, aep, uind and uinp -- the
// reference's energy() already sums ep/dep/aep into esum/desum/aesum
// (src/md/energy.cpp:289-330) although it never calls epolar.  epolar<M>()
// runs the same evaluation for callers that call the term on its own.
//
// Inputs come from the module globals after mechanic(); the device context
// (parameters, plans, buffers) persists across calls and is rebuilt when the
// system changes.  Failures map to the reference's fatal() (src/md/fatal.cpp),
// which is where the library's status codes meet the reference's convention.
#include "action.h"
#include "analyz.h"
#include "angbnd.h"
#include "atmlst.h"
#include "atoms.h"
#include "bound.h"
#include "bndstr.h"
#include "boxes.h"
#include "calcMode.h"
#include "cflux.h"
#include "chgpen.h"
#include "chgpot.h"
#include "couple.h"
#include "deriv.h"
#include "energi.h"
#include "ewald.h"
#include "fatal.h"
#include "inter.h"
#include "kmulti.h"
#include "mdqclimits.h"
#include "molcul.h"
#include "mplpot.h"
#include "mpole.h"
#include "pme.h"
#include "polar.h"
#include "polgrp.h"
#include "polopt.h"
#include "polpcg.h"
#include "polpot.h"
#include "potent.h"
#include "units.h"
#include "virial.h"

#include "amoeba_gpu.h"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>

namespace polmdqc
{
namespace
{
struct Csr {
    std::vector<int32_t> off, idx;
    amg_list view() const { return amg_list{off.data(), idx.data()}; }
};

template <class CountF, class ItemF>
Csr csr(int n, CountF count, ItemF item)
{
    Csr c;
    c.off.assign(n + 1, 0);
    for (int i = 0; i < n; i++) c.off[i + 1] = c.off[i] + count(i);
    c.idx.resize(c.off[n] + 1);
    for (int i = 0; i < n; i++)
        for (int j = 0; j < count(i); j++) c.idx[c.off[i] + j] = item(i, j);
    return c;
}

struct Device {
    amg_ctx* ctx = nullptr;
    int n = -1;
    const void* key_pole = nullptr;
    double key_sig = 0;
    bool polar = false;
    // host copies the context was created from
    std::vector<double> pole13, polar_, thole_, pdamp_;
    std::vector<int32_t> zax, xax, yax, axe, mol;
    Csr l12, l13, l14, l15, g11, g12, g13, g14;
    // charge penetration and charge flux (chgpen.h, cflux.h, bndstr.h, angbnd.h)
    std::vector<double> pcore_, palpha_, bflux_, aflux_;
    std::vector<int32_t> batoms_, aatoms_;
} dev;

// the monopole the context starts from: with charge flux the reference's
// energy() rewrites pole[i][0] every call (alterchg, src/md/energy.cpp:241),
// so the unaltered mono0 is the parameter
double monopole(int i) { return use_chgflx ? mono0[i] : pole[i][0]; }

// a cheap signature of the parameters that would force a new context
double signature()
{
    double s = n + 7 * aeewald + 3 * ewaldcut + 5 * mpolecut + nefft1 + 3 * nefft2 + 5 * nefft3 + (use_ewald ? 11 : 0);
    for (int i = 0; i < n; i++) s += (i % 13 + 1) * monopole(i);
    return s;
}

void fail(const char* what, int rc)
{
    printf("\n AMOEBA GPU  --  %s failed (status %d): %s\n", what, rc, amg_last_error(dev.ctx));
    fatal();
}

void ensure_context(bool want_polar)
{
    double sig = signature();
    if (dev.ctx && dev.n == n && dev.key_pole == (const void*)pole.ptr() && dev.key_sig == sig &&
        dev.polar == want_polar)
        return;
    if (dev.ctx) amg_destroy(dev.ctx);
    dev.ctx = nullptr;
    dev.n = n;
    dev.key_pole = pole.ptr();
    dev.key_sig = sig;
    dev.polar = want_polar;
    dev.pole13.resize(13 * (size_t)n);
    dev.zax.resize(n); dev.xax.resize(n); dev.yax.resize(n); dev.axe.resize(n); dev.mol.resize(n);
    for (int i = 0; i < n; i++) {
        for (int j = 0; j < 13; j++) dev.pole13[13 * i + j] = pole[i][j];
        dev.pole13[13 * i] = monopole(i);
        dev.zax[i] = zaxis[i]; dev.xax[i] = xaxis[i]; dev.yax[i] = yaxis[i];
        dev.axe[i] = (int32_t)polaxe[i];
        dev.mol[i] = molcule[i];
    }
    dev.l12 = csr(n, [](int i) { return n12[i]; }, [](int i, int j) { return i12[i][j]; });
    dev.l13 = csr(n, [](int i) { return n13[i]; }, [](int i, int j) { return i13[i][j]; });
    dev.l14 = csr(n, [](int i) { return n14[i]; }, [](int i, int j) { return i14[i][j]; });
    dev.l15 = csr(n, [](int i) { return n15[i]; }, [](int i, int j) { return i15[i][j]; });
    amg_params p{};
    p.n = n;
    p.pole = dev.pole13.data();
    p.zaxis = dev.zax.data(); p.xaxis = dev.xax.data(); p.yaxis = dev.yax.data(); p.polaxe = dev.axe.data();
    p.molcule = dev.mol.data();
    p.i12 = dev.l12.view(); p.i13 = dev.l13.view(); p.i14 = dev.l14.view(); p.i15 = dev.l15.view();
    double ms[4] = {m2scale, m3scale, m4scale, m5scale};
    double ps[4] = {p2scale, p3scale, p4scale, p5scale};
    double pis[4] = {p2iscale, p3iscale, p4iscale, p5iscale};
    double ds[4] = {d1scale, d2scale, d3scale, d4scale};
    double us[4] = {u1scale, u2scale, u3scale, u4scale};
    for (int k = 0; k < 4; k++) {
        p.m_scale[k] = ms[k]; p.p_scale[k] = ps[k]; p.p_iscale[k] = pis[k]; p.d_scale[k] = ds[k]; p.u_scale[k] = us[k];
    }
    if (want_polar) {
        dev.polar_.assign(polarity.ptr(), polarity.ptr() + n);
        dev.thole_.assign(thole.ptr(), thole.ptr() + n);
        dev.pdamp_.assign(pdamp.ptr(), pdamp.ptr() + n);
        dev.g11 = csr(n, [](int i) { return np11[i]; }, [](int i, int j) { return ip11[i][j]; });
        dev.g12 = csr(n, [](int i) { return np12[i]; }, [](int i, int j) { return ip12[i][j]; });
        dev.g13 = csr(n, [](int i) { return np13[i]; }, [](int i, int j) { return ip13[i][j]; });
        dev.g14 = csr(n, [](int i) { return np14[i]; }, [](int i, int j) { return ip14[i][j]; });
        p.polarity = dev.polar_.data(); p.thole = dev.thole_.data(); p.pdamp = dev.pdamp_.data();
        p.ip11 = dev.g11.view(); p.ip12 = dev.g12.view(); p.ip13 = dev.g13.view(); p.ip14 = dev.g14.view();
        p.poltyp = poltyp == "DIRECT" ? AMG_POL_DIRECT : poltyp == "OPT" ? AMG_POL_OPT : AMG_POL_MUTUAL;
        // kpolar zeroes copt below index maxopt only (src/md/kpolar.cpp:110-113),
        // so the last entry may hold a leftover value for orders below 6: a
        // coefficient that small is no order of the model
        if (poltyp == "OPT")
            for (int k = 0; k <= maxopt && k <= AMG_MAX_OPT; k++)
                p.opt_coef[k] = std::fabs(copt[k]) > 1e-100 ? copt[k] : 0.0;
    } else {
        p.poltyp = AMG_POL_NONE;
    }
    p.use_ewald = use_ewald;
    p.use_bounds = use_bounds;
    p.aewald = aeewald;
    p.nfft[0] = nefft1; p.nfft[1] = nefft2; p.nfft[2] = nefft3;
    p.bsorder = bseorder;
    p.cutoff = use_ewald ? ewaldcut : mpolecut;
    p.poleps = poleps;
    p.politer = politer;
    p.electric = electric;
    p.dielec = dielec;
    p.debye = debye;
    const char* prec = getenv("AMG_PRECISION");
    p.precision = (prec && prec[0] == 'f') ? AMG_PREC_FP64 : AMG_PREC_MIXED;
    p.pcg_guess = pcgguess;
    p.device = 0;
    p.pcg_prec = pcgprec;
    p.usolvcut = usolvcut;
    p.cell_shape = octahedron ? AMG_CELL_OCTAHEDRON : dodecadron ? AMG_CELL_DODECAHEDRON : AMG_CELL_FROM_ANGLES;
    // charge penetration (pairMpoleCP) and charge flux (alterchg / dcflux):
    // the library takes them in the non-Ewald multipole mode and returns
    // UNSUPPORTED otherwise, which stops the program below
    p.pentype = pentype == PenTyp::Gordon1 ? AMG_PEN_GORDON1 : pentype == PenTyp::Gordon2 ? AMG_PEN_GORDON2 : AMG_PEN_NONE;
    if (p.pentype != AMG_PEN_NONE) {
        dev.pcore_.assign(pcore.ptr(), pcore.ptr() + n);
        dev.palpha_.assign(palpha.ptr(), palpha.ptr() + n);
        p.pcore = dev.pcore_.data();
        p.palpha = dev.palpha_.data();
    }
    if (use_chgflx) {
        p.cflux = 1;
        dev.batoms_.assign(2 * (size_t)nbond + 1, 0);
        dev.bflux_.assign(2 * (size_t)nbond + 1, 0.0);
        for (int b = 0; b < nbond; b++) {
            dev.batoms_[2 * b] = ibnd[b][0];
            dev.batoms_[2 * b + 1] = ibnd[b][1];
            dev.bflux_[2 * b] = bl[b];
            dev.bflux_[2 * b + 1] = bflx[b];
        }
        dev.aatoms_.assign(3 * (size_t)nangle + 1, 0);
        dev.aflux_.assign(7 * (size_t)nangle + 1, 0.0);
        for (int a = 0; a < nangle; a++) {
            for (int j = 0; j < 3; j++) dev.aatoms_[3 * a + j] = iang[a][j];
            double* f = &dev.aflux_[7 * (size_t)a];
            f[0] = anat[a];
            f[1] = bl[balist[a][0]];
            f[2] = bl[balist[a][1]];
            f[3] = aflx[a][0]; f[4] = aflx[a][1];
            f[5] = abflx[a][0]; f[6] = abflx[a][1];
        }
        p.nbond = nbond;
        p.bond_atoms = dev.batoms_.data();
        p.bond_flux = dev.bflux_.data();
        p.nangle = nangle;
        p.angle_atoms = dev.aatoms_.data();
        p.angle_flux = dev.aflux_.data();
    }
    int rc = amg_create(&p, &dev.ctx);
    if (rc != AMG_OK) {
        printf("\n AMOEBA GPU  --  amg_create failed (status %d)\n", rc);
        fatal();
    }
}

template <CalcMode M>
void evaluate(bool fill_mpole, bool fill_polar)
{
    constexpr CalcFlag flags = getCalculationFlags<M>();
    const bool want_polar = use_polar && polarity.size() >= n;
    ensure_context(want_polar);
    std::vector<double> xyz(3 * (size_t)n);
    for (int i = 0; i < n; i++) { xyz[3 * i] = x[i]; xyz[3 * i + 1] = y[i]; xyz[3 * i + 2] = z[i]; }
    double box[6] = {xbox, ybox, zbox, alphaA, betaA, gammaA};
    int rc = amg_set_coords(dev.ctx, xyz.data(), box);
    if (rc != AMG_OK) fail("amg_set_coords", rc);
    int32_t f = AMG_DO_ENERGY | AMG_DO_DIPOLES;
    if (flags.do_analysis) f |= AMG_DO_ANALYSIS;
    if (flags.do_gradient) f |= AMG_DO_GRADIENT;
    if (flags.do_virial) f |= AMG_DO_VIRIAL;
    amg_results r{};
    std::vector<double> gm, gp, am, ap, ui, up;
    if (flags.do_gradient && fill_mpole) { gm.assign(3 * (size_t)n, 0.0); r.dem = gm.data(); }
    if (flags.do_gradient && fill_polar && want_polar) { gp.assign(3 * (size_t)n, 0.0); r.dep = gp.data(); }
    if (flags.do_analysis) { am.assign(n, 0.0); ap.assign(n, 0.0); r.aem = am.data(); r.aep = ap.data(); }
    if (want_polar && fill_polar) { ui.assign(3 * (size_t)n, 0.0); up.assign(3 * (size_t)n, 0.0); r.uind = ui.data(); r.uinp = up.data(); }
    rc = amg_forward(dev.ctx, f, &r);
    if (rc != AMG_OK) fail("amg_forward", rc);
    if (fill_mpole) {
        em = r.em;
        if (flags.do_gradient)
            for (int k = 0; k < 3 * n; k++) dem[k] += gm[k];
        if (flags.do_analysis) {
            nem = (int)r.nem;
            einter += r.einter;
            for (int i = 0; i < n; i++) aem[i] = am[i];
        }
    }
    if (fill_polar && want_polar) {
        ep = r.ep;
        if (flags.do_gradient)
            for (int k = 0; k < 3 * n; k++) dep[k] += gp[k];
        if (flags.do_analysis) {
            nep = (int)r.nep;
            for (int i = 0; i < n; i++) aep[i] = ap[i];
        }
        for (int i = 0; i < n; i++)
            for (int j = 0; j < 3; j++) { uind[i][j] = ui[3 * i + j]; uinp[i][j] = up[3 * i + j]; }
    }
    // virial (virial.h vir, added to like the reference's empole_a and torque
    // do): both parts when this call filled em and ep, else the ep part
    if (flags.do_virial) {
        double vm[9], vp[9];
        rc = amg_last_virial(dev.ctx, vm, vp);
        if (rc != AMG_OK) fail("amg_last_virial", rc);
        const bool polar = fill_polar && want_polar;
        for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++)
                vir[a][b] += (fill_mpole ? vm[3 * a + b] : 0.0) + (polar ? vp[3 * a + b] : 0.0);
    }
}
}  // namespace

template <CalcMode CalculationMode>
void empole()
{
    if (npole == 0) return;
    evaluate<CalculationMode>(true, true);
}

template <CalcMode CalculationMode>
void epolar()
{
    if (npole == 0 || !use_polar) return;
    evaluate<CalculationMode>(false, true);
}

// explicit instantiation, as src/md/empole.cpp:371-374
template void empole<CalcMode::Energy>();
template void empole<CalcMode::Analysis>();
template void empole<CalcMode::Gradient>();
template void empole<CalcMode::Virial>();
template void epolar<CalcMode::Energy>();
template void epolar<CalcMode::Analysis>();
template void epolar<CalcMode::Gradient>();
template void epolar<CalcMode::Virial>();
}
