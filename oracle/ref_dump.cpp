// ref_dump -- test-only driver around the reference library (oracle/_ref).
//
// Runs the reference's own set-up and energy path exactly as its `analyze`
// program does (src/md/analyze.cpp:60-62: initial -> getcart -> mechanic, then
// energy<CalcMode>() from src/md/energy.cpp:31) and prints the module globals
// that the electrostatics path reads and writes as one JSON object:
//   inputs : n, x/y/z, type, pole/rpole (13), z/x/yaxis (1-based), polaxe,
//            polarity, thole, pdamp, n12..n15/i12..i15, np11..np14/ip11..ip14,
//            scale factors, box, ewald/pme parameters, cutoffs, molcule
//   outputs: em, aem, nem, einter, dem, vir (Analysis + Virial calls)
// It is the checker's source of golden vectors; the product never runs it.
//
// usage: ref_dump --out file.json [reference analyze-style args: xyz -k key]

#include "action.h"
#include "analyz.h"
#include "angbnd.h"
#include "atmlst.h"
#include "bndstr.h"
#include "cflux.h"
#include "chgpen.h"
#include "atoms.h"
#include "bound.h"
#include "boxes.h"
#include "calcMode.h"
#include "chgpot.h"
#include "couple.h"
#include "deriv.h"
#include "energi.h"
#include "energy.h"
#include "ewald.h"
#include "files.h"
#include "getcart.h"
#include "inform.h"
#include "initial.h"
#include "inter.h"
#include "kmulti.h"
#include "mdqclimits.h"
#include "mechanic.h"
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
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

using namespace polmdqc;

static FILE* fo;
static bool first_field;

static void key(const char* k) {
    fprintf(fo, "%s\n\"%s\": ", first_field ? "" : ",", k);
    first_field = false;
}
static void num(const char* k, double v) { key(k); fprintf(fo, "%.17g", v); }
static void inum(const char* k, long v) { key(k); fprintf(fo, "%ld", v); }
template <class F>
static void darr(const char* k, int m, F f) {
    key(k);
    fputc('[', fo);
    for (int i = 0; i < m; i++) fprintf(fo, "%s%.17g", i ? "," : "", (double)f(i));
    fputc(']', fo);
}
template <class F>
static void iarr(const char* k, int m, F f) {
    key(k);
    fputc('[', fo);
    for (int i = 0; i < m; i++) fprintf(fo, "%s%ld", i ? "," : "", (long)f(i));
    fputc(']', fo);
}
// ragged int lists: [[...], [...], ...]
template <class C, class F>
static void ilists(const char* k, int m, C cnt, F f) {
    key(k);
    fputc('[', fo);
    for (int i = 0; i < m; i++) {
        fputs(i ? ",[" : "[", fo);
        for (int j = 0; j < cnt(i); j++) fprintf(fo, "%s%d", j ? "," : "", (int)f(i, j));
        fputc(']', fo);
    }
    fputc(']', fo);
}

int main(int argc, char** argv)
{
    std::string out;
    std::vector<char*> args;
    args.push_back((char*)"analyze");
    for (int i = 1; i < argc; i++) {
        if (!strcmp(argv[i], "--out") && i + 1 < argc) { out = argv[++i]; continue; }
        args.push_back(argv[i]);
    }
    args.push_back((char*)"e");
    args.push_back(nullptr);
    test = true;
    initial((int)args.size() - 1, args.data());
    getcart(ffile);
    mechanic();

    energy<CalcMode::Analysis>();
    double em_a = em, einter_a = einter, ep_a = ep;
    int nem_a = nem;
    std::vector<double> aem_a(n);
    for (int i = 0; i < n; i++) aem_a[i] = aem[i];

    for (int a = 0; a < 3; a++) for (int b = 0; b < 3; b++) vir[a][b] = 0.;
    energy<CalcMode::Virial>();

    fo = out.empty() ? stdout : fopen(out.c_str(), "w");
    if (!fo) return 2;
    first_field = true;
    fputc('{', fo);
    inum("n", n);
    darr("x", n, [](int i) { return x[i]; });
    darr("y", n, [](int i) { return y[i]; });
    darr("z", n, [](int i) { return z[i]; });
    iarr("type", n, [](int i) { return type[i]; });
    iarr("molcule", n, [](int i) { return molcule[i]; });
    inum("npole", npole);
    iarr("pollist", n, [](int i) { return pollist[i]; });
    iarr("zaxis", n, [](int i) { return zaxis[i]; });
    iarr("xaxis", n, [](int i) { return xaxis[i]; });
    iarr("yaxis", n, [](int i) { return yaxis[i]; });
    iarr("polaxe", n, [](int i) { return (int)polaxe[i]; });
    darr("pole", 13 * n, [](int i) { return pole[i / 13][i % 13]; });
    darr("rpole", 13 * n, [](int i) { return rpole[i / 13][i % 13]; });
    bool have_pol = use_polar && polarity.size() >= n;
    if (have_pol) {
        darr("polarity", n, [](int i) { return polarity[i]; });
        darr("thole", n, [](int i) { return thole[i]; });
        darr("pdamp", n, [](int i) { return pdamp[i]; });
        ilists("ip11", n, [](int i) { return np11[i]; }, [](int i, int j) { return ip11[i][j]; });
        ilists("ip12", n, [](int i) { return np12[i]; }, [](int i, int j) { return ip12[i][j]; });
        ilists("ip13", n, [](int i) { return np13[i]; }, [](int i, int j) { return ip13[i][j]; });
        ilists("ip14", n, [](int i) { return np14[i]; }, [](int i, int j) { return ip14[i][j]; });
        key("poltyp");
        fprintf(fo, "\"%s\"", poltyp.c_str());
        if (poltyp == "OPT") darr("copt", maxopt + 1, [](int i) { return copt[i]; });
    }
    ilists("i12", n, [](int i) { return n12[i]; }, [](int i, int j) { return i12[i][j]; });
    ilists("i13", n, [](int i) { return n13[i]; }, [](int i, int j) { return i13[i][j]; });
    ilists("i14", n, [](int i) { return n14[i]; }, [](int i, int j) { return i14[i][j]; });
    ilists("i15", n, [](int i) { return n15[i]; }, [](int i, int j) { return i15[i][j]; });
    darr("mscale", 4, [](int i) { double s[4] = {m2scale, m3scale, m4scale, m5scale}; return s[i]; });
    darr("pscale", 4, [](int i) { double s[4] = {p2scale, p3scale, p4scale, p5scale}; return s[i]; });
    darr("piscale", 4, [](int i) { double s[4] = {p2iscale, p3iscale, p4iscale, p5iscale}; return s[i]; });
    darr("dscale", 4, [](int i) { double s[4] = {d1scale, d2scale, d3scale, d4scale}; return s[i]; });
    darr("uscale", 4, [](int i) { double s[4] = {u1scale, u2scale, u3scale, u4scale}; return s[i]; });
    darr("wscale", 4, [](int i) { double s[4] = {w2scale, w3scale, w4scale, w5scale}; return s[i]; });
    num("poleps", poleps);
    inum("politer", politer);
    inum("use_polar", use_polar);
    inum("use_ewald", use_ewald);
    inum("use_bounds", use_bounds);
    num("electric", electric);
    num("dielec", dielec);
    num("debye", debye);
    num("aewald", aewald);
    num("aeewald", aeewald);
    num("apewald", apewald);
    iarr("nefft", 3, [](int i) { int v[3] = {nefft1, nefft2, nefft3}; return v[i]; });
    inum("bseorder", bseorder);
    inum("bsporder", bsporder);
    num("ewaldcut", ewaldcut);
    num("mpolecut", mpolecut);
    num("usolvcut", usolvcut);
    darr("box", 6, [](int i) { double v[6] = {xbox, ybox, zbox, alphaA, betaA, gammaA}; return v[i]; });
    inum("orthogonal", orthogonal);
    inum("monoclinic", monoclinic);
    inum("triclinic", triclinic);
    inum("octahedron", octahedron);
    inum("dodecadron", dodecadron);
    num("em", em_a);
    num("einter", einter_a);
    inum("nem", nem_a);
    darr("aem", n, [&](int i) { return aem_a[i]; });
    num("em_virial_call", em);
    darr("dem", 3 * n, [](int i) { return dem[i]; });
    num("ep", ep_a);
    if (have_pol) {
        darr("dep", 3 * n, [](int i) { return dep[i]; });
        darr("uind", 3 * n, [](int i) { return uind[i / 3][i % 3]; });
        darr("uinp", 3 * n, [](int i) { return uinp[i / 3][i % 3]; });
    }
    darr("vir", 9, [](int i) { return vir[i / 3][i % 3]; });
    // charge penetration and charge flux (AMOEBA+ / HIPPO multipoles)
    inum("pentype", pentype == PenTyp::Gordon1 ? 1 : pentype == PenTyp::Gordon2 ? 2 : 0);
    inum("use_chgflx", use_chgflx);
    if (pentype != PenTyp::None) {
        darr("pcore", n, [](int i) { return pcore[i]; });
        darr("pval0", n, [](int i) { return pval0[i]; });
        darr("palpha", n, [](int i) { return palpha[i]; });
    }
    if (use_chgflx) {
        darr("mono0", n, [](int i) { return mono0[i]; });
        inum("nbond", nbond);
        iarr("ibnd", 2 * nbond, [](int i) { return ibnd[i / 2][i % 2]; });
        darr("bl", nbond, [](int i) { return bl[i]; });
        darr("bflx", nbond, [](int i) { return bflx[i]; });
        inum("nangle", nangle);
        iarr("iang", 3 * nangle, [](int i) { return iang[i / 3][i % 3]; });
        darr("anat", nangle, [](int i) { return anat[i]; });
        darr("rab0", nangle, [](int i) { return bl[balist[i][0]]; });
        darr("rcb0", nangle, [](int i) { return bl[balist[i][1]]; });
        darr("aflx", 2 * nangle, [](int i) { return aflx[i / 2][i % 2]; });
        darr("abflx", 2 * nangle, [](int i) { return abflx[i / 2][i % 2]; });
    }
    fputs("\n}\n", fo);
    if (fo != stdout) fclose(fo);
    return 0;
}
