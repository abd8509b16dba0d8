// kernels_cp.cuh -- charge penetration and charge flux of the permanent
// multipoles (AMOEBA+ and HIPPO), in the non-Ewald multipole mode the
// reference implements (src/md/empole.cpp:64-82).  FP64 in both precisions.
//
// Charge penetration (include/md/pairMpole.h:186-389): the monopole of each
// site is a point core charge plus a valence charge; the valence multipole
// (valence charge, dipole, quadrupole) is smeared with exponent alpha.  A
// pair's energy is
//   E = core_i core_k bare + E(V_i, core_k; B^i) + E(core_i, V_k; B^k)
//       + E(V_i, V_k; B^ik),
// each term the invariant multipole energy of pair_math.cuh with its own
// radial hierarchy B_n = bare_n (1 - Q_n(x) e^{-x}), x = alpha r: B^i the
// potential of i's valence density (seen by k's core), B^ik the overlap of
// the two valence densities.  The polynomials Q_n follow from the base
// potential by B_{n+1} = -(1/r) dB_n/dr, i.e. Q_{n+1} = Q_n + x (Q_n - Q_n')/(2n+1)
// (tabulated on the host, CpTables).
//
// Charge flux (src/md/alterchg.cpp, src/md/dcflux.cpp): the monopoles move
// with bond lengths and angles, q = q0 + dq(x); the gradient gains
// sum_i pot_i d(dq_i)/dx with pot_i = dE/dq_i, the potential at the valence
// charge of i, which the pair kernels collect.
#pragma once
#include "kernels.cuh"
#include "kernels_pair.cuh"

namespace amg {

constexpr int kCpTerms = 12;  // polynomial coefficients x^0 .. x^11

// Q_n of the three density families (n = 0..5): core-valence of Gordon f1
// (base 1 + x/2) and f2 (base 1), valence-valence of two equal f1 densities
// (base 1 + 11x/16 + 3x^2/16 + x^3/48); with unequal exponents the
// valence-valence potential is a combination of the single-density families
struct CpTables {
    double f1[6][kCpTerms], f2[6][kCpTerms], e1[6][kCpTerms];
    int pentype;  // AMG_PEN_GORDON1 / AMG_PEN_GORDON2, or AMG_PEN_NONE (charge flux alone)
};

__device__ __forceinline__ double cp_poly(const double (&c)[kCpTerms], double x) {
    double v = 0;
#pragma unroll
    for (int j = kCpTerms - 1; j >= 0; j--) v = v * x + c[j];
    return v;
}

// multipliers of bare_n (n = 0..5) for the pair (i, k): fi (valence of i with
// the core of k), fk (the reverse), fik (valence with valence).  Exponents
// closer than 1e-3 take the equal-exponent form, as the reference's
// threshold (include/md/damping.h:42-43).
__device__ __forceinline__ void cp_factors(const CpTables& T, double r, double ai, double ak, double (&fi)[6],
                                           double (&fk)[6], double (&fik)[6]) {
    const double xi = ai * r, xk = ak * r, ei = exp(-xi), ek = exp(-xk);
    const bool equal = fabs(ai - ak) < 1e-3;
    const double ti = equal ? 0.0 : ak * ak / (ak * ak - ai * ai), tk = equal ? 0.0 : ai * ai / (ai * ai - ak * ak);
    const bool g1 = T.pentype == AMG_PEN_GORDON1;
#pragma unroll
    for (int n = 0; n < 6; n++) {
        const double(&core)[kCpTerms] = g1 ? T.f1[n] : T.f2[n];
        fi[n] = 1.0 - cp_poly(core, xi) * ei;
        fk[n] = 1.0 - cp_poly(core, xk) * ek;
        if (g1)
            fik[n] = equal ? 1.0 - cp_poly(T.e1[n], xi) * ei
                           : 1.0 - ti * ti * (cp_poly(T.f1[n], xi) + 2 * tk * cp_poly(T.f2[n], xi)) * ei -
                                 tk * tk * (cp_poly(T.f1[n], xk) + 2 * ti * cp_poly(T.f2[n], xk)) * ek;
        else
            fik[n] = equal ? 1.0 - cp_poly(T.f1[n], xi) * ei
                           : 1.0 - ti * cp_poly(T.f2[n], xi) * ei - tk * cp_poly(T.f2[n], xk) * ek;
    }
}

// One directed pair seen from site i (r = x_k - x_i), all channels times the
// m-scale: energy E (whole pair), gradient gi = dE/dx_i, torque on i, and
// pot_i = dE/d(valence charge of i).  With T.pentype == AMG_PEN_NONE the cores
// are zero and every channel is bare: the plain multipole pair plus pot_i.
__device__ __forceinline__ void cp_pair_i(const CpTables& T, const Mpole<double>& Mi, double core_i, double ai,
                                          const Mpole<double>& Mk, double core_k, double ak, V3<double> r, double m,
                                          double& E, V3<double>& gi, V3<double>& ti, double& pot_i) {
    const double r2 = dot(r, r), rinv = rsqrt(r2), rr = r2 * rinv;
    double bare[6];
    bare_terms<double, 6>(rinv, rinv * rinv, bare);
    double fi[6] = {1, 1, 1, 1, 1, 1}, fk[6] = {1, 1, 1, 1, 1, 1}, fik[6] = {1, 1, 1, 1, 1, 1};
    if (T.pentype != AMG_PEN_NONE) cp_factors(T, rr, ai, ak, fi, fk, fik);
    double Bb[6], Bi[6], Bk[6], Bik[6];
#pragma unroll
    for (int n = 0; n < 6; n++) {
        Bb[n] = m * bare[n];
        Bi[n] = Bb[n] * fi[n];
        Bk[n] = Bb[n] * fk[n];
        Bik[n] = Bb[n] * fik[n];
    }
    Mpole<double> Ci{}, Ck{}, Vi = Mi, Vk = Mk;
    Ci.q = core_i;
    Ck.q = core_k;
    Vi.q -= core_i;
    Vk.q -= core_k;
    double e;
    V3<double> g, t;
    mm_pair_i<double>(Ci, Ck, r, Bb, E, gi, ti);   // core-core (no torque)
    mm_pair_i<double>(Vi, Ck, r, Bi, e, g, t);     // valence of i, core of k
    E += e; gi = gi + g; ti = ti + t;
    mm_pair_i<double>(Ci, Vk, r, Bk, e, g, t);     // core of i, valence of k
    E += e; gi = gi + g; ti = ti + t;
    mm_pair_i<double>(Vi, Vk, r, Bik, e, g, t);    // valence-valence
    E += e; gi = gi + g; ti = ti + t;
    const SiteInv<double> sk = invariants(Vk, r);
    pot_i = core_k * Bi[0] + Vk.q * Bik[0] - sk.a * Bik[1] + sk.b * Bik[2];
}

// Bulk pairs (m-scale 1) of every site over its neighbour row, FP64, a lane
// group of LPA lanes per site (sites in cell order): the i side of each
// directed pair, as k_mpole_pair, plus the charge-flux potential cfpot.
// EXTRA: per-site energy, nonzero pair count, intermolecular energy and the
// pair virial, each when its pointer is set.
template <int LPA, bool EXTRA>
__global__ void __launch_bounds__(128) k_cp_pair(int n, const int* __restrict__ order, const double* __restrict__ xyz,
                                                 const double* __restrict__ rp10, const double* __restrict__ pcore,
                                                 const double* __restrict__ palpha, CpTables T, Box bx,
                                                 const int* __restrict__ nbr, int cap, const int* __restrict__ nnb,
                                                 double f, double* __restrict__ grad, double* __restrict__ trq,
                                                 double* __restrict__ cfpot, double* __restrict__ eacc,
                                                 double* __restrict__ aem, const int* __restrict__ mol,
                                                 unsigned long long* __restrict__ npair, double* __restrict__ vir) {
    const int gi_ = (blockIdx.x * blockDim.x + threadIdx.x) / LPA, lane = threadIdx.x % LPA;
    const int i = order[min(gi_, n - 1)];
    const int cnt = gi_ < n ? nnb[i] : 0;
    const Mpole<double> Mi = mpole64(rp10 + 10 * i);
    const double ci = pcore ? pcore[i] : 0.0, ai = palpha ? palpha[i] : 0.0;
    const V3<double> xi = ld3(xyz, i);
    double e_i = 0, einter = 0, pot = 0, w[6] = {0, 0, 0, 0, 0, 0};
    long long cntnz = 0;
    V3<double> g = v3<double>(0, 0, 0), t = v3<double>(0, 0, 0);
    const int mi = EXTRA && mol ? mol[i] : 0;
    const int* row = nbr + (size_t)i * cap;
    for (int s = lane; s < cnt; s += LPA) {
        const int k = row[s];
        const V3<double> r = min_image<double>(ld3(xyz, k) - xi, bx);
        double E, p;
        V3<double> gp, tp;
        cp_pair_i(T, Mi, ci, ai, mpole64(rp10 + 10 * k), pcore ? pcore[k] : 0.0, palpha ? palpha[k] : 0.0, r, 1.0,
                  E, gp, tp, p);
        e_i += 0.5 * E;
        g = g + gp;
        t = t + tp;
        pot += p;
        if (EXTRA) {
            if (E != 0.0) cntnz++;
            if (mol && mol[k] != mi) einter += 0.5 * E;
            vir_outer(w, gp.x, gp.y, gp.z, r.x, r.y, r.z, -0.5 * f);
        }
    }
    double out[8] = {g.x, g.y, g.z, t.x, t.y, t.z, pot, e_i};
#pragma unroll
    for (int q = 0; q < 8; q++) out[q] = group_sum<LPA>(out[q]);
    if (lane == 0 && gi_ < n) {
        for (int c = 0; c < 3; c++) {
            grad[3 * i + c] += f * out[c];
            trq[3 * i + c] += f * out[3 + c];
        }
        if (cfpot) cfpot[i] += f * out[6];
        if (EXTRA && aem) aem[i] += f * out[7];
    }
    block_sum_add(f * e_i, eacc);
    if (EXTRA && npair) {
        block_sum_add(f * einter, eacc + 1);
        block_sum_add_ll(cntnz, npair);
    }
    if (EXTRA && vir) block_vir_add(w, vir);
}

// scaled pairs in the core/valence form, both sites (FP64, atomics)
__global__ void k_cp_scaled(int np, const ScaledPair* __restrict__ sp, const double* __restrict__ xyz,
                            const double* __restrict__ rp10, const double* __restrict__ pcore,
                            const double* __restrict__ palpha, CpTables T, Box bx, double cut2, double f,
                            double* __restrict__ grad, double* __restrict__ trq, double* __restrict__ cfpot,
                            double* __restrict__ eacc, double* __restrict__ aem, const int* __restrict__ mol,
                            unsigned long long* __restrict__ npair, double* __restrict__ vir) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    double e = 0, einter = 0, w[6] = {0, 0, 0, 0, 0, 0};
    long long nz = 0;
    if (t < np) {
        const ScaledPair P = sp[t];
        const int i = P.i, k = P.k;
        const V3<double> r = min_image<double>(ld3(xyz, k) - ld3(xyz, i), bx);
        if (dot(r, r) <= cut2 && P.m != 0.0) {
            const Mpole<double> Mi = mpole64(rp10 + 10 * i), Mk = mpole64(rp10 + 10 * k);
            const double ci = pcore ? pcore[i] : 0.0, ck = pcore ? pcore[k] : 0.0;
            const double ai = palpha ? palpha[i] : 0.0, ak = palpha ? palpha[k] : 0.0;
            double E, E2, pi_, pk;
            V3<double> gi, ti, gk, tk;
            cp_pair_i(T, Mi, ci, ai, Mk, ck, ak, r, P.m, E, gi, ti, pi_);
            cp_pair_i(T, Mk, ck, ak, Mi, ci, ai, (-1.0) * r, P.m, E2, gk, tk, pk);
            e = f * E;
            nz = 2 * (E != 0.0);
            add3(grad, i, f * gi);
            add3(grad, k, f * gk);
            add3(trq, i, f * ti);
            add3(trq, k, f * tk);
            if (cfpot) {
                atomicAdd(cfpot + i, f * pi_);
                atomicAdd(cfpot + k, f * pk);
            }
            if (aem) {
                atomicAdd(aem + i, 0.5 * e);
                atomicAdd(aem + k, 0.5 * e);
            }
            if (mol && mol[i] != mol[k]) einter = e;
            vir_outer(w, gk.x, gk.y, gk.z, r.x, r.y, r.z, f);
        }
    }
    block_sum_add(e, eacc);
    if (mol) block_sum_add(einter, eacc + 1);
    if (npair) block_sum_add_ll(nz, npair);
    if (vir) block_vir_add(w, vir);
}

// ---------------------------------------------------------------- charge flux
// Monopole increments of the current geometry, added to dq (which starts at
// zero): a bond a-b (bond_flux = ideal length, flux k) moves k (r_ab - r0)
// from a to b; an angle a-b-c (angle_flux = theta0 in degrees, ideal a-b and
// c-b lengths, pa1, pa2, pb1, pb2) gives a the increment pb1 (r_cb - r0_cb) +
// pa1 (theta - theta0), c the increment pb2 (r_ab - r0_ab) + pa2 (theta -
// theta0), b minus both.  One thread per bond, then per angle; plain
// coordinate differences (no images), as the reference.
__global__ void k_cflux_charges(int nb, const int2* __restrict__ bonds, const double2* __restrict__ bflux, int na,
                                const int* __restrict__ angles, const double* __restrict__ aflux,
                                const double* __restrict__ xyz, double* __restrict__ dq) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < nb) {
        const int2 b = bonds[t];
        const double2 p = bflux[t];
        const double r = sqrt(dot(ld3(xyz, b.x) - ld3(xyz, b.y), ld3(xyz, b.x) - ld3(xyz, b.y)));
        const double d = p.y * (r - p.x);
        atomicAdd(dq + b.x, -d);
        atomicAdd(dq + b.y, d);
    } else if (t < nb + na) {
        const int q = t - nb;
        const int a = angles[3 * q], b = angles[3 * q + 1], c = angles[3 * q + 2];
        const double* p = aflux + 7 * q;
        const V3<double> u = ld3(xyz, a) - ld3(xyz, b), v = ld3(xyz, c) - ld3(xyz, b);
        const double ru = sqrt(dot(u, u)), rv = sqrt(dot(v, v));
        if (!(ru > 0 && rv > 0)) return;
        const double cs = fmax(-1.0, fmin(1.0, dot(u, v) / (ru * rv)));
        const double dth = acos(cs) - p[0] * (kPi / 180.0);
        const double q1 = p[5] * (rv - p[2]) + p[3] * dth;
        const double q2 = p[6] * (ru - p[1]) + p[4] * dth;
        atomicAdd(dq + a, q1);
        atomicAdd(dq + b, -(q1 + q2));
        atomicAdd(dq + c, q2);
    }
}

// gradient through the increments, sum_i pot_i d(dq_i)/dx (pot = dE/dq,
// already times electric/dielec), added to grad; the strain derivative into
// vir (six sums) when set: each term's gradients times its atoms' offsets
// from the bond's second atom / the angle's vertex
__global__ void k_cflux_grad(int nb, const int2* __restrict__ bonds, const double2* __restrict__ bflux, int na,
                             const int* __restrict__ angles, const double* __restrict__ aflux,
                             const double* __restrict__ xyz, const double* __restrict__ pot, double* __restrict__ grad,
                             double* __restrict__ vir) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    double w[6] = {0, 0, 0, 0, 0, 0};
    if (t < nb) {
        const int2 b = bonds[t];
        const V3<double> u = ld3(xyz, b.x) - ld3(xyz, b.y);
        const double r = sqrt(dot(u, u));
        const V3<double> g = ((pot[b.y] - pot[b.x]) * bflux[t].y / r) * u;
        add3(grad, b.x, g);
        add3(grad, b.y, (-1.0) * g);
        vir_outer(w, g.x, g.y, g.z, u.x, u.y, u.z, 1.0);
    } else if (t < nb + na) {
        const int q = t - nb;
        const int a = angles[3 * q], b = angles[3 * q + 1], c = angles[3 * q + 2];
        const double* p = aflux + 7 * q;
        const V3<double> u = ld3(xyz, a) - ld3(xyz, b), v = ld3(xyz, c) - ld3(xyz, b);
        const double ru = sqrt(dot(u, u)), rv = sqrt(dot(v, v));
        if (ru > 0 && rv > 0) {
            const double cs = dot(u, v) / (ru * rv);
            const double sn = sqrt(fmax(0.0, 1.0 - cs * cs));
            const double pa = pot[a] - pot[b], pc = pot[c] - pot[b];
            // d cos / dx_a and d cos / dx_c; d theta = -d cos / sin
            const V3<double> dca = (1.0 / (ru * rv)) * v - (cs / (ru * ru)) * u;
            const V3<double> dcc = (1.0 / (ru * rv)) * u - (cs / (rv * rv)) * v;
            const double wt = -(pa * p[3] + pc * p[4]) / sn;
            const V3<double> ga = (pc * p[6] / ru) * u + wt * dca;
            const V3<double> gc = (pa * p[5] / rv) * v + wt * dcc;
            add3(grad, a, ga);
            add3(grad, c, gc);
            add3(grad, b, (-1.0) * (ga + gc));
            vir_outer(w, ga.x, ga.y, ga.z, u.x, u.y, u.z, 1.0);
            vir_outer(w, gc.x, gc.y, gc.z, v.x, v.y, v.z, 1.0);
        }
    }
    if (vir) block_vir_add(w, vir);
}

}  // namespace amg
