// kernels_adjoint.cuh -- the hand-written adjoint (amg_backward), FP64.
//
// For L = c (em + ep) + <g_d, u_d> + <g_p, u_p>, with A u_d = E_d, A u_p = E_p
// (A = alpha^-1 - T symmetric) and ep = -1/2 f u_d . E_p, one adjoint solve
// A w = g (both right-hand sides, the forward's PCG) gives every parameter
// gradient as the gradient, at fixed vectors, of the bilinear function
//   G_L = c em + U_d(b_d <-> M) + U_p(b_p <-> M) + U_u(P1 <-> Q1) + U_u(P2 <-> Q2)
// with b_d = c f/2 u_p - w_d, b_p = c f/2 u_d - w_p, (P1, Q1) = (b_d, u_d),
// (P2, Q2) = (-w_p, u_p), U(a <-> b) the interaction energy of two sets, plus
// the diagonal term -(b_d.u_d - w_p.u_p)_i / alpha_i^2 for dL/dalpha_i.
// (For c = 1, g = 0 this is the forward's force function.)  Pair
// intermediates are recomputed, never stored.
#pragma once
#include "kernels.cuh"
#include "kernels_pair.cuh"
#include "kernels_misc.cuh"

namespace amg {

// d(lambda_n)/dx of the Thole factors (n = 1..4 <-> lambda_3,5,7,9)
template <class R>
__device__ __forceinline__ void thole_dlambda_dx(R x, R e, R (&d)[5]) {
    d[0] = 0;
    d[1] = e;
    d[2] = x * e;
    d[3] = (R(0.6) * x * x - R(0.2) * x) * e;
    d[4] = (R(9.0 / 35.0) * x * x * x - R(9.0 / 35.0) * x * x - R(1.0 / 35.0) * x) * e;
}

// radial derivatives of a Thole channel: dB_n/d(damp) and dB_n/d(a)
// (B_n = ... + scale lambda_n bare_n), n = 1..4; zero without damping
template <class R>
__device__ __forceinline__ void thole_radial_derivs(R r, R damp, R a, R scale, const R (&bare)[6], R (&dBd)[6],
                                                    R (&dBa)[6]) {
    for (int k = 0; k < 6; k++) dBd[k] = dBa[k] = 0;
    if (damp == R(0)) return;
    R t = r / damp;
    R x = a * t * t * t;
    R e = exp(-x);
    R dl[5];
    thole_dlambda_dx<R>(x, e, dl);
    for (int n = 1; n <= 4; n++) {
        dBd[n] = scale * bare[n] * dl[n] * (R(-3) * x / damp);
        dBa[n] = a != R(0) ? scale * bare[n] * dl[n] * (x / a) : R(0);
    }
}

// pair energies (for the parameter derivatives) -------------------------------
template <class R>
__device__ __forceinline__ R md_energy(const Mpole<R>& Mi, const SiteInv<R>& si, V3<R> v, V3<R> r, const R (&B)[6]) {
    R av = dot(v, r);
    return (-Mi.q * av + dot(Mi.d, v)) * B[1] + (-si.a * av + 2 * dot(v, si.Qr)) * B[2] - av * si.b * B[3];
}
template <class R>
__device__ __forceinline__ R dm_energy(V3<R> w, const Mpole<R>& Mk, const SiteInv<R>& sk, V3<R> r, const R (&B)[6]) {
    R aw = dot(w, r);
    return (Mk.q * aw + dot(w, Mk.d)) * B[1] + (-aw * sk.a - 2 * dot(w, sk.Qr)) * B[2] + aw * sk.b * B[3];
}
template <class R>
__device__ __forceinline__ R dd_energy(V3<R> a, V3<R> b, V3<R> r, const R (&B)[6]) {
    return dot(a, b) * B[1] - dot(a, r) * dot(b, r) * B[2];
}

// potential derivatives (phi, grad phi, grad grad phi: 10) at the target of
// a multipole at the source, r = x_target - x_source, order xx yy zz xy xz yz
template <class R>
__device__ __forceinline__ void mpole_potential10(const Mpole<R>& M, V3<R> r, const R (&B)[6], R (&p)[10]) {
    SiteInv<R> s = invariants(M, r);
    R rr[3] = {r.x, r.y, r.z}, d[3] = {M.d.x, M.d.y, M.d.z}, qr[3] = {s.Qr.x, s.Qr.y, s.Qr.z};
    R Q[3][3] = {{M.Q.xx, M.Q.xy, M.Q.xz}, {M.Q.xy, M.Q.yy, M.Q.yz}, {M.Q.xz, M.Q.yz, M.Q.zz}};
    p[0] = M.q * B[0] + s.a * B[1] + s.b * B[2];
    for (int a = 0; a < 3; a++)
        p[1 + a] = -M.q * rr[a] * B[1] + d[a] * B[1] - s.a * rr[a] * B[2] + 2 * qr[a] * B[2] - s.b * rr[a] * B[3];
    const int ia[6] = {0, 1, 2, 0, 0, 1}, ib[6] = {0, 1, 2, 1, 2, 2};
    R c2 = M.q * B[2] + s.a * B[3] + s.b * B[4], c1 = M.q * B[1] + s.a * B[2] + s.b * B[3];
    for (int k = 0; k < 6; k++) {
        int a = ia[k], b = ib[k];
        R v = rr[a] * rr[b] * c2 - (d[a] * rr[b] + d[b] * rr[a]) * B[2] + 2 * Q[a][b] * B[2] -
              2 * (qr[a] * rr[b] + qr[b] * rr[a]) * B[3];
        if (a == b) v -= c1;
        p[4 + k] = v;
    }
}

__device__ __forceinline__ V3<double> ld3v(const double* p, int i) { return v3<double>(p[3 * i], p[3 * i + 1], p[3 * i + 2]); }

// effective vectors of the adjoint (all FP64, [3n] each)
__global__ void k_adj_vectors(int n, double cf, const double* __restrict__ ud, const double* __restrict__ up,
                              const double* __restrict__ wd, const double* __restrict__ wp, double* __restrict__ bd,
                              double* __restrict__ bp, double* __restrict__ vbar, double* __restrict__ mwp,
                              const double* __restrict__ pol, double* __restrict__ dpol) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double s = 0;
    for (int c = 0; c < 3; c++) {
        int q = 3 * i + c;
        double a = 0.5 * cf * up[q] - (wd ? wd[q] : 0.0);
        double b = 0.5 * cf * ud[q] - (wp ? wp[q] : 0.0);
        bd[q] = a;
        bp[q] = b;
        vbar[q] = a + b;
        mwp[q] = wp ? -wp[q] : 0.0;
        s += a * ud[q] - (wp ? wp[q] * up[q] : 0.0);
    }
    // diagonal part of dA/dalpha_i: d(1/alpha)/dalpha = -1/alpha^2
    dpol[i] = pol[i] > 0 ? -s / (pol[i] * pol[i]) : 0.0;
}

// Bulk real-space part of the adjoint, site i over its neighbour list:
// gradient dG_L/dx_i, torque on M_i, the per-site potentials dG_L/dM_i (10),
// and dG_L/d(pdamp_i), dG_L/d(thole_i).  Sites, vectors and partner rows in
// cell order (at = cell-order copy of the sites, nbr = cell-order partner
// positions, vec = R4 [n][5] in cell order: vbar, P1, Q1, P2, Q2); the
// results go to site i = order[g] in the original order.  Pair arithmetic in
// R (FP32 for a mixed-precision context, as its forward's pair kernels),
// every sum in FP64.  The mscale channel for M-M uses the cm factor (= c f).
template <class R, bool EWALD, int LPA>
__global__ void __launch_bounds__(128) k_adjoint_pair(int n, const int* __restrict__ order, const AtomR<R>* __restrict__ at,
                                                      const R4<R>* __restrict__ vec, Box bx, R aewald,
                                                      const int* __restrict__ nbr, int cap,
                                                      const int* __restrict__ nnb, int mutual, double cm,
                                                      double* __restrict__ grad, double* __restrict__ trq,
                                                      double* __restrict__ pot, double* __restrict__ dpd,
                                                      double* __restrict__ dth) {
    const int g = (blockIdx.x * blockDim.x + threadIdx.x) / LPA, lane = threadIdx.x % LPA;
    const int gs = min(g, n - 1), i = order[gs];
    const int cnt = g < n ? nnb[i] : 0;
    const AtomR<R> Ai = at[gs];
    const Mpole<R> Mi = load_mpole(Ai);
    const V3<R> xi = v3<R>(Ai.a.x, Ai.a.y, Ai.a.z);
    auto V = [&](int j, int k) { R4<R> t = vec[5 * (size_t)j + k]; return v3<R>(t.x, t.y, t.z); };
    const V3<R> vb_i = V(gs, 0), p1_i = V(gs, 1), q1_i = V(gs, 2), p2_i = V(gs, 3), q2_i = V(gs, 4);
    const R cmr = (R)cm;
    double acc[18] = {0};  // gradient 3, torque 3, dpdamp, dthole, potentials 10
    const int* row = nbr + (size_t)i * cap;
    for (int s = lane; s < cnt; s += LPA) {
        const int j = row[s];
        const AtomR<R> Aj = ld_atom(at, j);
        const Mpole<R> Mk = load_mpole(Aj);
        const V3<R> r = min_image<R>(v3<R>(Aj.a.x, Aj.a.y, Aj.a.z) - xi, bx);  // x_k - x_i
        const R r2 = dot(r, r), rr = sqrt(r2);
        // multipole-multipole (em), no Thole, scale 1
        R Bm[6];
        bulk_radial<R, EWALD, false>(r2, aewald, R(0), R(0), Bm);
        R E;
        V3<R> gi, ti;
        mm_pair_i<R>(Mi, Mk, r, Bm, E, gi, ti);
        V3<R> gsum = cmr * gi, tsum = cmr * ti;
        R pm[10];
        mpole_potential10<R>(Mk, R(-1) * r, Bm, pm);  // potential of M_k at i
        // polarization channels (Thole, scale 1)
        const R damp = Ai.e.y * Aj.e.y, a = pair_thole<R>(Ai.e.z, Aj.e.z);
        R B[6];
        bulk_radial<R, EWALD, true>(r2, aewald, damp, a, B);
        const V3<R> vb_k = V(j, 0), p1_k = V(j, 1), q1_k = V(j, 2), p2_k = V(j, 3), q2_k = V(j, 4);
        const SiteInv<R> si = invariants(Mi, r), sk = invariants(Mk, r);
        V3<R> d1, t1;
        md_pair<R>(Mi, si, vb_k, r, B, d1, t1);
        V3<R> dEdr = d1 + dm_pair<R>(vb_i, Mk, sk, r, B);
        if (mutual)
            dEdr = dEdr + dd_pair<R>(p1_i, q1_k, r, B) + dd_pair<R>(q1_i, p1_k, r, B) + dd_pair<R>(p2_i, q2_k, r, B) +
                   dd_pair<R>(q2_i, p2_k, r, B);
        gsum = gsum - dEdr;
        tsum = tsum + t1;
        // potential of the dipoles vbar_k at i (d/p channels coincide here)
        Mpole<R> Dk;
        Dk.q = 0;
        Dk.d = vb_k;
        Dk.Q = Sym<R>{0, 0, 0, 0, 0, 0};
        R pd_[10];
        mpole_potential10<R>(Dk, R(-1) * r, B, pd_);
        // damping derivatives: the same pair energies with dB
        R bare[6], dBd[6], dBa[6];
        const R rinv = R(1) / rr;
        bare_terms<R, 6>(rinv, rinv * rinv, bare);
        thole_radial_derivs<R>(rr, damp, a, R(1), bare, dBd, dBa);
        auto Gwith = [&](const R (&D)[6]) {
            R e = md_energy<R>(Mi, si, vb_k, r, D) + dm_energy<R>(vb_i, Mk, sk, r, D);
            if (mutual)
                e += dd_energy<R>(p1_i, q1_k, r, D) + dd_energy<R>(q1_i, p1_k, r, D) + dd_energy<R>(p2_i, q2_k, r, D) +
                     dd_energy<R>(q2_i, p2_k, r, D);
            return e;
        };
        const R gd = Gwith(dBd) * Aj.e.y;  // d damp / d pdamp_i = pdamp_k
        const R ga = Gwith(dBa);
        const R ti_ = Ai.e.z, tk_ = Aj.e.z;
        const R lo = fmin(ti_, tk_);
        const R own = (lo == R(0)) ? (ti_ > tk_ ? R(1) : ti_ == tk_ ? R(0.5) : R(0))
                                   : (ti_ < tk_ ? R(1) : ti_ == tk_ ? R(0.5) : R(0));
        acc[0] += gsum.x; acc[1] += gsum.y; acc[2] += gsum.z;
        acc[3] += tsum.x; acc[4] += tsum.y; acc[5] += tsum.z;
        acc[6] += gd;
        acc[7] += own * ga;
        for (int k = 0; k < 10; k++) acc[8 + k] += cmr * pm[k] + pd_[k];
    }
#pragma unroll
    for (int k = 0; k < 18; k++) acc[k] = group_sum<LPA>(acc[k]);
    if (lane == 0 && g < n) {
        for (int c = 0; c < 3; c++) {
            grad[3 * i + c] += acc[c];
            trq[3 * i + c] += acc[3 + c];
        }
        dpd[i] += acc[6];
        dth[i] += acc[7];
        for (int k = 0; k < 10; k++) pot[10 * (size_t)i + k] += acc[8 + k];
    }
}

// scaled pairs: the same quantities with each channel's own scale (FP64,
// both sites, atomics)
__global__ void k_adjoint_scaled(int np, const ScaledPair* __restrict__ sp, const double* __restrict__ xyz,
                                 const double* __restrict__ rp10, const double* __restrict__ pdamp,
                                 const double* __restrict__ thole, Box bx, double cut2, double aewald,
                                 const double* __restrict__ bd, const double* __restrict__ bp,
                                 const double* __restrict__ P1, const double* __restrict__ Q1,
                                 const double* __restrict__ P2, const double* __restrict__ Q2, int mutual, double cm,
                                 double* __restrict__ grad, double* __restrict__ trq, double* __restrict__ pot,
                                 double* __restrict__ dpd, double* __restrict__ dth) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= np) return;
    ScaledPair P = sp[t];
    ScaledGeom G = scaled_geom(P, xyz, pdamp, thole, bx, cut2, aewald);
    if (!G.inside) return;
    const int i = P.i, k = P.k;
    const V3<double> r = G.r, mr = (-1.0) * G.r;
    const double rr = sqrt(dot(r, r));
    Mpole<double> Mi = mpole64(rp10 + 10 * i), Mk = mpole64(rp10 + 10 * k);
    double Bm[6], Bd[6], Bp[6], Bu[6];
    scaled_radial(G, P.m, false, aewald > 0, Bm);
    scaled_radial(G, P.d, true, aewald > 0, Bd);
    scaled_radial(G, P.p, true, aewald > 0, Bp);
    scaled_radial(G, P.u, true, aewald > 0, Bu);
    // em
    double E, E2;
    V3<double> gi, ti, gk, tk;
    mm_pair_i<double>(Mi, Mk, r, Bm, E, gi, ti);
    mm_pair_i<double>(Mk, Mi, mr, Bm, E2, gk, tk);
    add3(grad, i, cm * gi);
    add3(grad, k, cm * gk);
    add3(trq, i, cm * ti);
    add3(trq, k, cm * tk);
    double pim[10], pkm[10];
    mpole_potential10(Mk, mr, Bm, pim);  // at i from M_k
    mpole_potential10(Mi, r, Bm, pkm);   // at k from M_i
    // polarization
    V3<double> bdi = ld3(bd, i), bdk = ld3(bd, k), bpi = ld3(bp, i), bpk = ld3(bp, k);
    SiteInv<double> si = invariants(Mi, r), sk_m = invariants(Mk, mr), sk = invariants(Mk, r);
    V3<double> dEdr = v3<double>(0, 0, 0), tqi = v3<double>(0, 0, 0), tqk = v3<double>(0, 0, 0), d1, t1;
    md_pair<double>(Mi, si, bdk, r, Bd, d1, t1);           // U_d(b_d,k ; M_i)
    dEdr = dEdr + d1; tqi = tqi + t1;
    md_pair<double>(Mk, sk_m, bdi, mr, Bd, d1, t1);        // U_d(b_d,i ; M_k)
    dEdr = dEdr - d1; tqk = tqk + t1;
    md_pair<double>(Mi, si, bpk, r, Bp, d1, t1);           // U_p(b_p,k ; M_i)
    dEdr = dEdr + d1; tqi = tqi + t1;
    md_pair<double>(Mk, sk_m, bpi, mr, Bp, d1, t1);        // U_p(b_p,i ; M_k)
    dEdr = dEdr - d1; tqk = tqk + t1;
    V3<double> p1i = ld3(P1, i), p1k = ld3(P1, k), q1i = ld3(Q1, i), q1k = ld3(Q1, k);
    V3<double> p2i = ld3(P2, i), p2k = ld3(P2, k), q2i = ld3(Q2, i), q2k = ld3(Q2, k);
    if (mutual)
        dEdr = dEdr + dd_pair<double>(p1i, q1k, r, Bu) + dd_pair<double>(q1i, p1k, r, Bu) +
               dd_pair<double>(p2i, q2k, r, Bu) + dd_pair<double>(q2i, p2k, r, Bu);
    add3(grad, i, (-1.0) * dEdr);
    add3(grad, k, dEdr);
    add3(trq, i, tqi);
    add3(trq, k, tqk);
    // potentials at i and k from the other site's dipoles (d and p channels)
    auto dip = [](V3<double> v) {
        Mpole<double> D;
        D.q = 0;
        D.d = v;
        D.Q = Sym<double>{0, 0, 0, 0, 0, 0};
        return D;
    };
    double a1[10], a2[10], b1[10], b2[10];
    mpole_potential10(dip(bdk), mr, Bd, a1);
    mpole_potential10(dip(bpk), mr, Bp, a2);
    mpole_potential10(dip(bdi), r, Bd, b1);
    mpole_potential10(dip(bpi), r, Bp, b2);
    for (int q = 0; q < 10; q++) {
        atomicAdd(pot + 10 * (size_t)i + q, cm * pim[q] + a1[q] + a2[q]);
        atomicAdd(pot + 10 * (size_t)k + q, cm * pkm[q] + b1[q] + b2[q]);
    }
    // damping derivatives
    const double damp = pdamp[i] * pdamp[k];
    const double a = pair_thole<double>(thole[i], thole[k]);
    double dBd_d[6], dBd_a[6], dBp_d[6], dBp_a[6], dBu_d[6], dBu_a[6];
    thole_radial_derivs(rr, damp, a, P.d, G.bare, dBd_d, dBd_a);
    thole_radial_derivs(rr, damp, a, P.p, G.bare, dBp_d, dBp_a);
    thole_radial_derivs(rr, damp, a, P.u, G.bare, dBu_d, dBu_a);
    auto Gwith = [&](const double (&Dd)[6], const double (&Dp)[6], const double (&Du)[6]) {
        double e = md_energy(Mi, si, bdk, r, Dd) + dm_energy(bdi, Mk, sk, r, Dd) + md_energy(Mi, si, bpk, r, Dp) +
                   dm_energy(bpi, Mk, sk, r, Dp);
        if (mutual)
            e += dd_energy(p1i, q1k, r, Du) + dd_energy(q1i, p1k, r, Du) + dd_energy(p2i, q2k, r, Du) +
                 dd_energy(q2i, p2k, r, Du);
        return e;
    };
    double gdamp = Gwith(dBd_d, dBp_d, dBu_d), ga = Gwith(dBd_a, dBp_a, dBu_a);
    atomicAdd(dpd + i, gdamp * pdamp[k]);
    atomicAdd(dpd + k, gdamp * pdamp[i]);
    double ti_ = thole[i], tk_ = thole[k], lo = fmin(ti_, tk_);
    double own_i = (lo == 0.0) ? (ti_ > tk_ ? 1.0 : ti_ == tk_ ? 0.5 : 0.0) : (ti_ < tk_ ? 1.0 : ti_ == tk_ ? 0.5 : 0.0);
    atomicAdd(dth + i, own_i * ga);
    atomicAdd(dth + k, (1.0 - own_i) * ga);
}

// reciprocal + self parts of the adjoint:
//   grad_k += vbar_k.gg(phiM) + M_k.g(phi_vbar) + P1_k.gg(phi_Q1) + Q1_k.gg(phi_P1)
//             + P2_k.gg(phi_Q2) + Q2_k.gg(phi_P2)
//   torque  = torque(M_k, phi_vbar) + selfc d_k x vbar_k
//   pot    += c f (phiM + M self) + phi_vbar - selfc vbar (dipole slots)
__global__ void k_adjoint_recip(int n, const double* __restrict__ rp10, const double* __restrict__ phiM,
                                const double* __restrict__ phv, const double* __restrict__ ph1,
                                const double* __restrict__ phq1, const double* __restrict__ ph2,
                                const double* __restrict__ phq2, const double* __restrict__ vbar,
                                const double* __restrict__ P1, const double* __restrict__ Q1,
                                const double* __restrict__ P2, const double* __restrict__ Q2, int mutual,
                                double selfc, double alpha, double cm, double* __restrict__ grad,
                                double* __restrict__ trq, double* __restrict__ pot) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double* m = rp10 + 10 * i;
    const double* pm = phiM + 20 * (size_t)i;
    const double* pv = phv + 20 * (size_t)i;
    V3<double> vb = ld3(vbar, i);
    V3<double> g = cm * site_gradient(m, pm) + dipole_gradient(vb, pm) + site_gradient(m, pv);
    if (mutual) {
        g = g + dipole_gradient(ld3(P1, i), phq1 + 20 * (size_t)i) + dipole_gradient(ld3(Q1, i), ph1 + 20 * (size_t)i) +
            dipole_gradient(ld3(P2, i), phq2 + 20 * (size_t)i) + dipole_gradient(ld3(Q2, i), ph2 + 20 * (size_t)i);
    }
    V3<double> d = v3<double>(m[1], m[2], m[3]);
    V3<double> t = cm * site_torque(m, pm) + site_torque(m, pv) + selfc * cross(d, vb);
    for (int c = 0; c < 3; c++) {
        grad[3 * i + c] += c == 0 ? g.x : c == 1 ? g.y : g.z;
        trq[3 * i + c] += c == 0 ? t.x : c == 1 ? t.y : t.z;
    }
    // potentials: recip of multipoles and of vbar; self of the multipoles
    // (-T_erf(0) M) and of the induced-permanent coupling (-selfc vbar on d)
    const double a2 = alpha * alpha, sp = 1.0 / kSqrtPi;
    double self[10] = {-2 * alpha * sp * m[0],
                       -(4 * a2 * alpha / 3) * sp * m[1], -(4 * a2 * alpha / 3) * sp * m[2],
                       -(4 * a2 * alpha / 3) * sp * m[3],
                       -(16 * a2 * a2 * alpha / 5) * sp * m[4], -(16 * a2 * a2 * alpha / 5) * sp * m[7],
                       -(16 * a2 * a2 * alpha / 5) * sp * m[9], -(16 * a2 * a2 * alpha / 5) * sp * m[5],
                       -(16 * a2 * a2 * alpha / 5) * sp * m[6], -(16 * a2 * a2 * alpha / 5) * sp * m[8]};
    for (int k = 0; k < 10; k++) pot[10 * (size_t)i + k] += cm * (pm[k] + self[k]) + pv[k];
    pot[10 * (size_t)i + 1] -= selfc * vb.x;
    pot[10 * (size_t)i + 2] -= selfc * vb.y;
    pot[10 * (size_t)i + 3] -= selfc * vb.z;
}

// ---------------------------------------------------------------- OPT
// Adjoint of the OPT dipoles u = S E, S = sum_k c_k (alpha T)^k alpha
// (c_k the mixed coefficients copm_k; S is symmetric).  With w^(a) =
// (alpha T)^a alpha g and u^(b) = (alpha T)^b alpha E the orders of the
// cotangents and of the fields (u^(b) kept by the forward), the part of
// dL/dtheta through S is
//   X1^T dS E_d + X2^T dS E_p,  X1 = g_d - c f/2 E_p, X2 = g_p,
// whose orders are X1~_a = w_d^(a) - c f/2 u_p^(a), X2~_a = w_p^(a).  From
// d[(alpha T)^k alpha] = sum_{a+b=k-1} (alpha T)^a alpha dT (alpha T)^b alpha
// + sum_{a+b=k} (alpha T)^a d(alpha) (T alpha)^b it splits into
//   dipole-dipole terms  sum_b V_b^T dT u^(b),
//     V_b = sum_a c_{a+b+1} X~_a   (the pairs (-V_b, u^(b)) of U_u),
//   diagonal terms       dL/dalpha_i += sum_k c_k sum_{a+b=k} X~_a,i . u^(b)_i / alpha_i^2.
// Orders are stored [K+1][2][3n] (d set, then p set, per order).

// w = sum_k c_k w^(k) for both sets
__global__ void k_opt_combine(int n3, int K, OptCoef c, const double* __restrict__ orders, double* __restrict__ wd,
                              double* __restrict__ wp) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n3) return;
    double d = 0, p = 0;
    for (int k = 0; k <= K; k++) {
        d += c.c[k] * orders[(size_t)(2 * k) * n3 + t];
        p += c.c[k] * orders[(size_t)(2 * k + 1) * n3 + t];
    }
    wd[t] = d;
    wp[t] = p;
}

// the dipole-dipole partners of u_d^(b) and u_p^(b): P1 = -V1_b, P2 = -V2_b
__global__ void k_opt_adj_cross(int n3, int K, int b, OptCoef c, double cf, const double* __restrict__ w,
                                const double* __restrict__ u, double* __restrict__ P1, double* __restrict__ P2) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n3) return;
    double v1 = 0, v2 = 0;
    for (int a = 0; a + b + 1 <= K; a++) {
        const double ck = c.c[a + b + 1];
        v1 += ck * (w[(size_t)(2 * a) * n3 + t] - 0.5 * cf * u[(size_t)(2 * a + 1) * n3 + t]);
        v2 += ck * w[(size_t)(2 * a + 1) * n3 + t];
    }
    P1[t] = -v1;
    P2[t] = -v2;
}

// the diagonal terms of dL/dalpha (they replace the mutual model's)
__global__ void k_opt_adj_diag(int n, int K, OptCoef c, double cf, const double* __restrict__ pol,
                               const double* __restrict__ w, const double* __restrict__ u, double* __restrict__ dpol) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const size_t n3 = 3 * (size_t)n;
    double s = 0;
    for (int k = 0; k <= K; k++) {
        double sk = 0;
        for (int a = 0; a <= k; a++) {
            const int b = k - a;
            for (int q = 3 * i; q < 3 * i + 3; q++) {
                const double x1 = w[(2 * a) * n3 + q] - 0.5 * cf * u[(2 * a + 1) * n3 + q];
                const double x2 = w[(2 * a + 1) * n3 + q];
                sk += x1 * u[(2 * b) * n3 + q] + x2 * u[(2 * b + 1) * n3 + q];
            }
        }
        s += c.c[k] * sk;
    }
    dpol[i] = pol[i] > 0 ? s / (pol[i] * pol[i]) : 0.0;
}

// dL/d(local pole): chain the global-frame potentials through the rotation
// (d_g = A^T d_l, Q_g = A^T Q_l A on the upper triangle), the chirality sign
// and the planar rule.  pot: [n][10] = dL/dq, dL/dd (3), and the potential
// second derivatives xx yy zz xy xz yz that multiply Q_g element-wise.
__global__ void k_pole_grad_local(int n, const double* __restrict__ xyz, const double* __restrict__ pole13,
                                  const int* __restrict__ zax, const int* __restrict__ xax,
                                  const int* __restrict__ yax, const int* __restrict__ axe,
                                  const double* __restrict__ pot, double* __restrict__ dpole) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double a[3][3];
    bool flip, planar;
    frame_matrix(i, xyz, zax, xax, yax, axe, a, flip, planar);
    const double* p = pot + 10 * (size_t)i;
    // the rotation uses the upper triangle of Q_g (p <= q), as the
    // reference's rotsite; the compact off-diagonal derivative is 2 phi_pq
    double G[3][3] = {{p[4], 2 * p[7], 2 * p[8]}, {0, p[5], 2 * p[9]}, {0, 0, p[6]}};
    double out[13];
    out[0] = p[0];
    for (int r = 0; r < 3; r++) out[1 + r] = a[r][0] * p[1] + a[r][1] * p[2] + a[r][2] * p[3];
    for (int r = 0; r < 3; r++)
        for (int t = 0; t < 3; t++) {
            double v = 0;
            for (int pp = 0; pp < 3; pp++)
                for (int q = 0; q < 3; q++) v += a[r][pp] * a[t][q] * G[pp][q];
            out[4 + 3 * r + t] = v;
        }
    // AMOEBA quadrupoles are traceless and the pair formulas assume it (as the
    // reference's include/md/pairMpole.h does): report the gradient restricted
    // to traceless quadrupoles
    {
        double tr = (out[4] + out[8] + out[12]) / 3.0;
        out[4] -= tr; out[8] -= tr; out[12] -= tr;
    }
    if (planar) {  // sp[1] = sp[6] = sp[10] = 0; sp[4] = sp[8] = (sp[4] + sp[8]) / 2
        out[1] = out[6] = out[10] = 0;
        double m = 0.5 * (out[4] + out[8]);
        out[4] = out[8] = m;
    }
    if (flip) {
        out[2] = -out[2]; out[5] = -out[5]; out[7] = -out[7]; out[9] = -out[9]; out[11] = -out[11];
    }
    for (int k = 0; k < 13; k++) dpole[13 * (size_t)i + k] = out[k];
}

// the net-charge term's share of each monopole gradient and the chain
// through pdamp = alpha^(1/6) (dpdamp/dalpha = pdamp / (6 alpha)), in place:
// dpole[13 i] += dq, dpol[i] <- dpol + dpd * chain (0 without polarization)
__global__ void k_adj_finish(int n, double dq, int has_pol, const double* __restrict__ pol,
                             const double* __restrict__ pdamp, const double* __restrict__ dpd, double* __restrict__ dth,
                             double* __restrict__ dpol, double* __restrict__ dpole) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    dpole[13 * (size_t)i] += dq;
    if (!has_pol) {
        dpol[i] = 0;
        dth[i] = 0;
        return;
    }
    const double chain = pol[i] > 0 ? pdamp[i] / (6.0 * pol[i]) : 0.0;
    dpol[i] += dpd[i] * chain;
}

}  // namespace amg
