// kernels_pair.cuh -- real-space pair kernels (a lane group per site over
// its exact neighbour list, both directions of every pair, warp-shuffle
// reductions, no atomics) and the FP64 scaled-pair kernels.
#pragma once
#include "kernels.cuh"

namespace amg {

// All bulk pair kernels below give each site a group of LPA consecutive
// lanes (LPA = 4, 8, 16 or 32); sites are taken in cell order (order = sids,
// g the position in that order, i = order[g] the site).  The lanes stride
// through the site's neighbour slots nbr[i * cap + s] -- here the partners'
// positions in cell order (the lists' cnb) -- and gather the packed sites
// `at` and dipoles u4 stored in cell order; results go to site i.  Partial
// sums are combined with warp shuffles (group_sum).  Sites past n run with an
// empty list so every lane takes part in the shuffles.

// Permanent field at every site from all neighbours' multipoles, bulk
// (scale 1, Thole damped, Ewald or bare).  Writes Ed = Ep (the d/p
// differences come only from the scaled pairs).  With COEF the same radial
// factors also fill the PCG's stored coefficient rows (see k_tu_coeffs: c0 =
// pack_tensor(x_i - x_j, B1, B2)) and the sparse preconditioner's rows (pairs
// within usolvcut, compacted in row order, when cu0 is given), so the solve's
// set-up recomputes nothing.
template <class R, bool EWALD, int LPA, bool COEF, bool CELLS = false>
__global__ void __launch_bounds__(128) k_perm_field(int n, const int* __restrict__ order, const AtomR<R>* __restrict__ at, Box bx, R aewald,
                                                    const int* __restrict__ nbr, int cap,
                                                    const int* __restrict__ nnb, double* __restrict__ Ed,
                                                    double* __restrict__ Ep, R4<R>* __restrict__ c0,
                                                    R usolv2, int* __restrict__ nbru, R4<R>* __restrict__ cu0,
                                                    int* __restrict__ nnbu) {
    const int g = (blockIdx.x * blockDim.x + threadIdx.x) / LPA, lane = threadIdx.x % LPA;
    const int gs = min(g, n - 1), i = order[gs];
    const int cnt = g < n ? nnb[i] : 0;
    AtomR<R> Ai = at[gs];
    V3<R> xi = v3<R>(Ai.a.x, Ai.a.y, Ai.a.z);
    R pdi = Ai.e.y, thi = Ai.e.z;
    double fx = 0, fy = 0, fz = 0;
    const size_t base = (size_t)i * cap;
    const int* row = nbr + base;
    // lanes of this group within the warp, and the lanes below this one
    const unsigned gmask = LPA == 32 ? 0xffffffffu : ((1u << LPA) - 1u) << ((threadIdx.x & 31) / LPA * LPA);
    const unsigned below = (1u << (threadIdx.x & 31)) - 1u;
    int nu = 0;  // preconditioner entries of this row so far
    for (int s0 = 0; s0 < cnt; s0 += LPA) {  // all lanes of a group take the same trips
        const int s = s0 + lane;
        const bool ok = s < cnt;
        int j = 0;
        V3<R> r = v3<R>(0, 0, 0);
        R P1 = 0, P2 = 0, r2 = 0;
        if (ok) {
            j = row[s];
            AtomR<R> Aj = ld_atom(at, j);
            r = min_image<R, !EWALD || CELLS>(xi - v3<R>(Aj.a.x, Aj.a.y, Aj.a.z), bx);  // target i - source j
            r2 = dot(r, r);
            R B[6];
            if (COEF) {
                bulk_radial_prec<R, EWALD>(r2, aewald, pdi * Aj.e.y, pair_thole<R>(thi, Aj.e.z), B, P1, P2);
                c0[base + s] = pack_tensor<R>(r.x, r.y, r.z, B[1], B[2]);
            } else {
                bulk_radial<R, EWALD, true>(r2, aewald, pdi * Aj.e.y, pair_thole<R>(thi, Aj.e.z), B);
            }
            V3<R> E = field_of_mpole<R>(load_mpole(Aj), r, B[1], B[2], B[3]);
            fx += E.x; fy += E.y; fz += E.z;
        }
        if (COEF && cu0) {
            const bool take = ok && r2 <= usolv2;
            const unsigned b = __ballot_sync(gmask, take) & gmask;
            if (take) {
                const size_t q = base + nu + __popc(b & below);
                nbru[q] = j;
                cu0[q] = pack_tensor<R>(r.x, r.y, r.z, P1, P2);
            }
            nu += __popc(b);
        }
    }
    if (COEF && cu0 && lane == 0 && g < n) nnbu[i] = nu;
    fx = group_sum<LPA>(fx); fy = group_sum<LPA>(fy); fz = group_sum<LPA>(fz);
    if (lane == 0 && g < n) {
        Ed[3 * i] = fx; Ed[3 * i + 1] = fy; Ed[3 * i + 2] = fz;
        Ep[3 * i] = fx; Ep[3 * i + 1] = fy; Ep[3 * i + 2] = fz;
    }
}

// Mutual field T u for two dipole sets (bulk, u-scale 1), computing the
// pair tensors on the fly (used by the FP64 correction sweep).  u4: [n][2]
// R4 (ux,uy,uz,0), d set then p set per site.  Writes Fd, Fp.
template <class R, bool EWALD, int LPA, bool CELLS = false>
__global__ void __launch_bounds__(128) k_Tu(int n, const int* __restrict__ order, const AtomR<R>* __restrict__ at, const R4<R>* __restrict__ u4,
                                            Box bx, R aewald, const int* __restrict__ nbr, int cap,
                                            const int* __restrict__ nnb, double* __restrict__ Fd,
                                            double* __restrict__ Fp) {
    const int g = (blockIdx.x * blockDim.x + threadIdx.x) / LPA, lane = threadIdx.x % LPA;
    const int i = order[min(g, n - 1)];
    const int cnt = g < n ? nnb[i] : 0;
    R4<R> pi = at[i].a, ei = at[i].e;
    V3<R> xi = v3<R>(pi.x, pi.y, pi.z);
    R ax = 0, ay = 0, az = 0, bx_ = 0, by = 0, bz = 0;
    const int* row = nbr + (size_t)i * cap;
    for (int s = lane; s < cnt; s += LPA) {
        int j = row[s];
        R4<R> pj = at[j].a, ej = at[j].e;
        V3<R> r = min_image<R, !EWALD || CELLS>(xi - v3<R>(pj.x, pj.y, pj.z), bx);
        R r2 = dot(r, r);
        R rinv = rsqrt_<R>(r2);
        R rr = r2 * rinv, rinv2 = rinv * rinv;
        R B1, B2;
        {
            R b1 = rinv * rinv2, b2 = 3 * b1 * rinv2;
            if (EWALD) {
                R eb[3];
                ewald_terms<R, 3>(rr, rinv2, aewald, eb);
                B1 = eb[1]; B2 = eb[2];
            } else {
                B1 = b1; B2 = b2;
            }
            R damp = ei.y * ej.y;
            if (damp != R(0)) {
                R t = ratio_<R>(rr, damp);
                R x = pair_thole<R>(ei.z, ej.z) * t * t * t;
                R e = exp_<R>(-x);
                B1 -= e * b1;                 // (1 - lambda3) = e
                B2 -= (R(1) + x) * e * b2;    // (1 - lambda5) = (1 + x) e
            }
        }
        R4<R> ud = u4[2 * j], up = u4[2 * j + 1];
        R ad = ud.x * r.x + ud.y * r.y + ud.z * r.z;
        R ap = up.x * r.x + up.y * r.y + up.z * r.z;
        ax += ad * B2 * r.x - B1 * ud.x; ay += ad * B2 * r.y - B1 * ud.y; az += ad * B2 * r.z - B1 * ud.z;
        bx_ += ap * B2 * r.x - B1 * up.x; by += ap * B2 * r.y - B1 * up.y; bz += ap * B2 * r.z - B1 * up.z;
    }
    // FP32 partial sums over a few neighbours, combined in FP64
    double sx = group_sum<LPA>((double)ax), sy = group_sum<LPA>((double)ay), sz = group_sum<LPA>((double)az);
    double tx = group_sum<LPA>((double)bx_), ty = group_sum<LPA>((double)by), tz = group_sum<LPA>((double)bz);
    if (lane == 0 && g < n) {
        Fd[3 * i] = sx; Fd[3 * i + 1] = sy; Fd[3 * i + 2] = sz;
        Fp[3 * i] = tx; Fp[3 * i + 1] = ty; Fp[3 * i + 2] = tz;
    }
}

// The same T u in FP64 with every gathered array in cell order (the FP64
// correction sweep): positions spos (x, y, z), damping sdt (pdamp, thole), the
// dipoles u4 [2n] and the rows' partners cnb (positions in cell order, bulk
// slots only), so the gathers of a warp's sites read contiguous runs.
// (7 blocks per SM: 71 registers, no spills; 6 at 75 registers was 8% slower)
template <bool EWALD, int LPA, bool CELLS = false>
__global__ void __launch_bounds__(128, 7) k_Tu_cells(int n, const int* __restrict__ order,
                                                  const double4* __restrict__ spos, const double2* __restrict__ sdt,
                                                  const double4* __restrict__ u4, Box bx, double aewald,
                                                  const int* __restrict__ cnb, int cap, const int* __restrict__ nnb,
                                                  double* __restrict__ Fd, double* __restrict__ Fp) {
    const int g = (blockIdx.x * blockDim.x + threadIdx.x) / LPA, lane = threadIdx.x % LPA;
    const int gs = min(g, n - 1), i = order[gs];
    const int cnt = g < n ? nnb[i] : 0;
    const double4 pi = spos[gs];
    const double2 di = sdt[gs];
    const V3<double> xi = v3<double>(pi.x, pi.y, pi.z);
    double ax = 0, ay = 0, az = 0, bx_ = 0, by = 0, bz = 0;
    const int* row = cnb + (size_t)i * cap;
    for (int s = lane; s < cnt; s += LPA) {
        const int j = row[s];
        const double4 pj = ld256(spos + j);
        const double2 dj = sdt[j];
        const V3<double> r = min_image<double, !EWALD || CELLS>(xi - v3<double>(pj.x, pj.y, pj.z), bx);
        const double r2 = dot(r, r), rinv = rsqrt(r2), rr = r2 * rinv, rinv2 = rinv * rinv;
        const double b1 = rinv * rinv2, b2 = 3 * b1 * rinv2;
        double B1 = b1, B2 = b2;
        if (EWALD) {
            // the Smith recursion of ewald_terms with erfc(x) = exp(-x^2) erfcx(x),
            // so one exponential serves both (0.5% faster per evaluation)
            const double a2 = aewald * aewald, ex = exp(-a2 * r2);
            double eb[3];
            eb[0] = ex * erfcx(aewald * rr) * (rinv2 * rr);
            double fac = 0.56418958354775628695 / aewald;  // 1/(a sqrt(pi))
#pragma unroll
            for (int m = 1; m < 3; m++) {
                fac *= 2 * a2;
                eb[m] = ((2 * m - 1) * eb[m - 1] + fac * ex) * rinv2;
            }
            B1 = eb[1];
            B2 = eb[2];
        }
        const double damp = di.x * dj.x;
        if (damp != 0.0) {
            const double t = rr / damp;
            const double x = pair_thole<double>(di.y, dj.y) * t * t * t;
            const double e = exp(-x);
            B1 -= e * b1;                 // (1 - lambda3) = e
            B2 -= (1.0 + x) * e * b2;     // (1 - lambda5) = (1 + x) e
        }
        double4 ud, up;
        load_pair(u4, j, ud, up);
        const double ad = (ud.x * r.x + ud.y * r.y + ud.z * r.z) * B2;
        const double ap = (up.x * r.x + up.y * r.y + up.z * r.z) * B2;
        ax += ad * r.x - B1 * ud.x; ay += ad * r.y - B1 * ud.y; az += ad * r.z - B1 * ud.z;
        bx_ += ap * r.x - B1 * up.x; by += ap * r.y - B1 * up.y; bz += ap * r.z - B1 * up.z;
    }
    ax = group_sum<LPA>(ax); ay = group_sum<LPA>(ay); az = group_sum<LPA>(az);
    bx_ = group_sum<LPA>(bx_); by = group_sum<LPA>(by); bz = group_sum<LPA>(bz);
    if (lane == 0 && g < n) {
        Fd[3 * i] = ax; Fd[3 * i + 1] = ay; Fd[3 * i + 2] = az;
        Fp[3 * i] = bx_; Fp[3 * i + 1] = by; Fp[3 * i + 2] = bz;
    }
}

// Multipole energy (half of each directed pair), gradient and torque of site
// i from all its neighbours (bulk, m-scale 1).  f = electric/dielec.
// EXTRA: the outputs of the Analysis and Virial modes, each written when its
// pointer is set -- per-site energy, nonzero pair count (directed) and
// intermolecular energy (aem, npair, mol); the pair virial (vir, six sums),
// half of -g_i (x) r per directed pair.
template <class R, bool EWALD, bool EXTRA, int LPA, bool CELLS = false>
__global__ void __launch_bounds__(128) k_mpole_pair(int n, const int* __restrict__ order, const AtomR<R>* __restrict__ at, Box bx, R aewald,
                                                    const int* __restrict__ nbr, int cap,
                                                    const int* __restrict__ nnb, double f, double* __restrict__ grad,
                                                    double* __restrict__ trq, double* __restrict__ eacc,
                                                    double* __restrict__ aem, const int* __restrict__ mol,
                                                    unsigned long long* __restrict__ npair, double* __restrict__ vir) {
    const int gi_ = (blockIdx.x * blockDim.x + threadIdx.x) / LPA, lane = threadIdx.x % LPA;
    const int gs = min(gi_, n - 1), i = order[gs];
    const int cnt = gi_ < n ? nnb[i] : 0;
    double e_i = 0, einter = 0, w[6] = {0, 0, 0, 0, 0, 0};
    long long cntnz = 0;
    AtomR<R> Ai = at[gs];
    Mpole<R> Mi = load_mpole(Ai);
    V3<R> xi = v3<R>(Ai.a.x, Ai.a.y, Ai.a.z);
    V3<R> g = v3<R>(0, 0, 0), t = v3<R>(0, 0, 0);
    int mi = EXTRA && mol ? mol[i] : 0;
    const int* row = nbr + (size_t)i * cap;
    for (int s = lane; s < cnt; s += LPA) {
        int j = row[s];
        AtomR<R> Aj = ld_atom(at, j);
        V3<R> r = min_image<R, !EWALD || CELLS>(v3<R>(Aj.a.x, Aj.a.y, Aj.a.z) - xi, bx);  // x_k - x_i
        R B[6];
        bulk_radial<R, EWALD, false>(dot(r, r), aewald, R(0), R(0), B);
        R E;
        V3<R> gi, ti;
        mm_pair_i<R>(Mi, load_mpole(Aj), r, B, E, gi, ti);
        e_i += 0.5 * (double)E;
        g = g + gi;
        t = t + ti;
        if (EXTRA) {
            if (E != R(0)) cntnz++;
            if (mol && mol[order[j]] != mi) einter += 0.5 * (double)E;
            vir_outer(w, gi.x, gi.y, gi.z, r.x, r.y, r.z, -0.5 * f);
        }
    }
    double gx = group_sum<LPA>((double)g.x), gy = group_sum<LPA>((double)g.y), gz = group_sum<LPA>((double)g.z);
    double tx = group_sum<LPA>((double)t.x), ty = group_sum<LPA>((double)t.y), tz = group_sum<LPA>((double)t.z);
    double es = group_sum<LPA>(e_i);
    if (lane == 0 && gi_ < n) {
        grad[3 * i] += f * gx; grad[3 * i + 1] += f * gy; grad[3 * i + 2] += f * gz;
        trq[3 * i] += f * tx; trq[3 * i + 1] += f * ty; trq[3 * i + 2] += f * tz;
        if (EXTRA && aem) aem[i] += f * es;
    }
    block_sum_add(f * e_i, eacc);
    if (EXTRA && npair) {
        block_sum_add(f * einter, eacc + 1);
        block_sum_add_ll(cntnz, npair);
    }
    if (EXTRA && vir) block_vir_add(w, vir);
}

// Polarization gradient and torque of site i (bulk, all scales 1):
//   G = E(M_i, ubar_k) + E(ubar_i, M_k) + 1/2 [E(up_i, ud_k) + E(ud_i, up_k)]
// with ubar = (ud + up)/2; dG/dx_i = -dG/dr, torque on M_i from ubar_k.
// u4: [n][2] R4, d set then p set per site.  VIR: the pair virial into
// vir (six sums), half of dG/dr (x) r per directed pair.  DDONLY: only the
// dipole-dipole term 1/2 [E(up_i, ud_k) + E(ud_i, up_k)] (the OPT cross
// terms between perturbation orders; no torques).
template <class R, bool EWALD, int LPA, bool VIR, bool DDONLY = false, bool CELLS = false>
__global__ void __launch_bounds__(128, (sizeof(R) == 4 && !VIR && !DDONLY) ? 6 : 1) k_polar_pair(int n, const int* __restrict__ order, const AtomR<R>* __restrict__ at,
                                                    const R4<R>* __restrict__ u4, Box bx, R aewald,
                                                    const int* __restrict__ nbr, int cap,
                                                    const int* __restrict__ nnb, int mutual, double f,
                                                    double* __restrict__ grad, double* __restrict__ trq,
                                                    double* __restrict__ vir) {
    const int gi_ = (blockIdx.x * blockDim.x + threadIdx.x) / LPA, lane = threadIdx.x % LPA;
    const int gs = min(gi_, n - 1), i = order[gs];
    const int cnt = gi_ < n ? nnb[i] : 0;
    AtomR<R> Ai = at[gs];
    Mpole<R> Mi = load_mpole(Ai);
    V3<R> xi = v3<R>(Ai.a.x, Ai.a.y, Ai.a.z);
    R4<R> udi4 = u4[2 * gs], upi4 = u4[2 * gs + 1];
    V3<R> udi = v3<R>(udi4.x, udi4.y, udi4.z), upi = v3<R>(upi4.x, upi4.y, upi4.z);
    V3<R> ubi = R(0.5) * (udi + upi);
    V3<R> g = v3<R>(0, 0, 0), t = v3<R>(0, 0, 0);
    double w[6] = {0, 0, 0, 0, 0, 0};
    const int* row = nbr + (size_t)i * cap;
    for (int s = lane; s < cnt; s += LPA) {
        int j = row[s];
        AtomR<R> Aj = ld_atom(at, j);
        V3<R> r = min_image<R, !EWALD || CELLS>(v3<R>(Aj.a.x, Aj.a.y, Aj.a.z) - xi, bx);
        R B[6];
        bulk_radial<R, EWALD, true>(dot(r, r), aewald, Ai.e.y * Aj.e.y, pair_thole<R>(Ai.e.z, Aj.e.z), B);
        R4<R> udk4, upk4;
        load_pair(u4, j, udk4, upk4);
        V3<R> udk = v3<R>(udk4.x, udk4.y, udk4.z), upk = v3<R>(upk4.x, upk4.y, upk4.z);
        V3<R> dEdr;
        if constexpr (DDONLY) {
            dEdr = R(0.5) * (dd_pair<R>(upi, udk, r, B) + dd_pair<R>(udi, upk, r, B));
        } else {
            V3<R> ubk = R(0.5) * (udk + upk);
            Mpole<R> Mk = load_mpole(Aj);
            SiteInv<R> si = invariants(Mi, r), sk = invariants(Mk, r);
            V3<R> d1, ti;
            md_pair<R>(Mi, si, ubk, r, B, d1, ti);
            dEdr = d1 + dm_pair<R>(ubi, Mk, sk, r, B);
            if (mutual) dEdr = dEdr + R(0.5) * (dd_pair<R>(upi, udk, r, B) + dd_pair<R>(udi, upk, r, B));
            t = t + ti;
        }
        g = g - dEdr;
        if (VIR) vir_outer(w, dEdr.x, dEdr.y, dEdr.z, r.x, r.y, r.z, 0.5 * f);
    }
    double gx = group_sum<LPA>((double)g.x), gy = group_sum<LPA>((double)g.y), gz = group_sum<LPA>((double)g.z);
    double tx = group_sum<LPA>((double)t.x), ty = group_sum<LPA>((double)t.y), tz = group_sum<LPA>((double)t.z);
    if (lane == 0 && gi_ < n) {
        grad[3 * i] += f * gx; grad[3 * i + 1] += f * gy; grad[3 * i + 2] += f * gz;
        if (!DDONLY) { trq[3 * i] += f * tx; trq[3 * i + 1] += f * ty; trq[3 * i + 2] += f * tz; }
    }
    if (VIR) block_vir_add(w, vir);
}

// ------------------------------------------------------------ stored T
// The dipole interaction tensor does not change during the PCG solve, so its
// pair coefficients are computed once per evaluation and streamed by every
// matvec: per slot one packed R4 (pack_tensor of r = x_i - x_j, B1, B2) and
// the neighbour's position in cell order (cnb, rank[j]).  Rows hold the bulk
// neighbours followed by the scaled partners (filled by k_scaled_coeffs), so
// one kernel applies the whole real-space T.  The PCG's R4 vectors (u4 of the
// first matvec, p4, s4) are stored in cell order too: the neighbours of the
// sites a warp handles then lie in a few contiguous runs of those vectors,
// which the gathers read as whole cache lines, mostly from L1.
template <class R, bool EWALD, int LPA, bool CELLS = false>
__global__ void __launch_bounds__(128) k_tu_coeffs(int n, const int* __restrict__ order, const AtomR<R>* __restrict__ at, Box bx, R aewald,
                                                   const int* __restrict__ nbr, int cap, const int* __restrict__ nnb,
                                                   R4<R>* __restrict__ c0, R usolv2, int* __restrict__ nbru,
                                                   R4<R>* __restrict__ cu0, int* __restrict__ nnbu) {
    const int g = (blockIdx.x * blockDim.x + threadIdx.x) / LPA, lane = threadIdx.x % LPA;
    if (g >= n) return;  // whole lane groups leave together
    const int i = order[g];
    const int cnt = nnb[i];
    R4<R> pi = at[g].a, ei = at[g].e;
    V3<R> xi = v3<R>(pi.x, pi.y, pi.z);
    const size_t base = (size_t)i * cap;
    // lanes of this group within the warp, and the lanes below this one
    const unsigned gmask = LPA == 32 ? 0xffffffffu : ((1u << LPA) - 1u) << ((threadIdx.x & 31) / LPA * LPA);
    const unsigned below = (1u << (threadIdx.x & 31)) - 1u;
    int nu = 0;  // preconditioner entries of this row so far
    for (int s0 = 0; s0 < cnt; s0 += LPA) {
        const int s = s0 + lane;
        const bool ok = s < cnt;
        R r2 = 0, P1 = 0, P2 = 0;
        V3<R> r = v3<R>(0, 0, 0);
        int j = 0;
        if (ok) {
            j = nbr[base + s];
            R4<R> pj = at[j].a, ej = at[j].e;
            r = min_image<R, !EWALD || CELLS>(xi - v3<R>(pj.x, pj.y, pj.z), bx);
            r2 = dot(r, r);
            R rinv = rsqrt_<R>(r2);
            R rr = r2 * rinv, rinv2 = rinv * rinv;
            R b1 = rinv * rinv2, b2 = 3 * b1 * rinv2;
            R B1 = b1, B2 = b2;
            if (EWALD) {
                R eb[3];
                ewald_terms<R, 3>(rr, rinv2, aewald, eb);
                B1 = eb[1]; B2 = eb[2];
            }
            P1 = b1; P2 = b2;
            R damp = ei.y * ej.y;
            if (damp != R(0)) {
                R t = ratio_<R>(rr, damp);
                R x = pair_thole<R>(ei.z, ej.z) * t * t * t;
                R e = exp_<R>(-x);
                B1 -= e * b1;
                B2 -= (R(1) + x) * e * b2;
                P1 -= e * b1;
                P2 -= (R(1) + x) * e * b2;
            }
            c0[base + s] = pack_tensor<R>(r.x, r.y, r.z, B1, B2);
        }
        if (cu0) {  // sparse preconditioner: bare Thole-damped T within usolvcut, compacted in order
            const bool take = ok && r2 <= usolv2;
            const unsigned b = __ballot_sync(gmask, take) & gmask;
            if (take) {
                const size_t q = base + nu + __popc(b & below);
                nbru[q] = j;
                cu0[q] = pack_tensor<R>(r.x, r.y, r.z, P1, P2);
            }
            nu += __popc(b);
        }
    }
    if (cu0 && lane == 0) nnbu[i] = nu;
}

// T v with the stored coefficients (both dipole sets): rows of nnb[i] bulk
// slots plus the site's scaled partners.  u4: [n][2] R4 in cell order.
// With vAv, also adds -v.F of both sets to vAv[0..1] (the real-space share
// of v.Av when the rest of Av is assembled apart, see k_gather_field).
template <class R, int LPA>
__global__ void __launch_bounds__(128) k_tu_stored(int n, const int* __restrict__ order, const int* __restrict__ cnb,
                                                   const R4<R>* __restrict__ c0, int cap,
                                                   const int* __restrict__ nnb, const int* __restrict__ xoff,
                                                   const R4<R>* __restrict__ u4, double* __restrict__ Fd,
                                                   double* __restrict__ Fp, const double* __restrict__ vd = nullptr,
                                                   const double* __restrict__ vp = nullptr,
                                                   double* __restrict__ vAv = nullptr) {
    const int g = (blockIdx.x * blockDim.x + threadIdx.x) / LPA, lane = threadIdx.x % LPA;
    const int gs = min(g, n - 1), i = order[gs];  // gs: the site's position in cell order
    const int cnt = g < n ? nnb[i] + (xoff[i + 1] - xoff[i]) : 0;
    const size_t base = (size_t)i * cap;
    R ax = 0, ay = 0, az = 0, bx_ = 0, by = 0, bz = 0;
    row_apply<R, LPA, sizeof(R) == 4 ? 4 : 2>(cnb, c0, base, cnt, lane, gs, u4, ax, ay, az, bx_, by, bz);
    double sx = group_sum<LPA>((double)ax), sy = group_sum<LPA>((double)ay), sz = group_sum<LPA>((double)az);
    double tx = group_sum<LPA>((double)bx_), ty = group_sum<LPA>((double)by), tz = group_sum<LPA>((double)bz);
    double dd = 0, dp = 0;
    if (lane == 0 && g < n) {
        Fd[3 * i] = sx; Fd[3 * i + 1] = sy; Fd[3 * i + 2] = sz;
        Fp[3 * i] = tx; Fp[3 * i + 1] = ty; Fp[3 * i + 2] = tz;
        if (vAv) {  // this part's share of v.Av (Av holds -F)
            dd = -(vd[3 * i] * sx + vd[3 * i + 1] * sy + vd[3 * i + 2] * sz);
            dp = -(vp[3 * i] * tx + vp[3 * i + 1] * ty + vp[3 * i + 2] * tz);
        }
    }
    if (vAv) {
        block_sum_add(dd, vAv);
        block_sum_add(dp, vAv + 1);
    }
}

// ------------------------------------------------------------ scaled pairs
// Pairs with any scale != 1, from the 1-n and polarization-group lists.
// They are removed from the bulk neighbour lists and evaluated whole here in
// FP64: these are the short intramolecular pairs whose large bare terms would
// otherwise pass through the FP32 bulk kernels and cancel against an FP64
// correction.
struct ScaledPair {
    int i, k;
    int si, sk;  // position of k among i's scaled partners and of i among k's
    double m, p, d, u;
};

struct ScaledGeom {  // FP64 geometry and radial parts of one scaled pair
    V3<double> r;    // x_k - x_i
    bool inside;
    double lam[5];
    double bare[6];
    double ew[6];
};

__device__ __forceinline__ ScaledGeom scaled_geom(const ScaledPair& sp, const double* __restrict__ xyz,
                                                  const double* __restrict__ pdamp, const double* __restrict__ thole,
                                                  Box bx, double cut2, double aewald) {
    ScaledGeom G;
    int i = sp.i, k = sp.k;
    G.r = min_image<double>(v3<double>(xyz[3 * k] - xyz[3 * i], xyz[3 * k + 1] - xyz[3 * i + 1],
                                       xyz[3 * k + 2] - xyz[3 * i + 2]), bx);
    double r2 = dot(G.r, G.r);
    G.inside = r2 <= cut2;
    double rinv = 1.0 / sqrt(r2);
    bare_terms<double, 6>(rinv, rinv * rinv, G.bare);
    if (aewald > 0) ewald_terms<double, 6>(r2 * rinv, rinv * rinv, aewald, G.ew);
    double damp = pdamp ? pdamp[i] * pdamp[k] : 0.0;
    double a = thole ? pair_thole<double>(thole[i], thole[k]) : 0.0;
    thole_lambda<double>(r2 * rinv, damp, a, G.lam);
    return G;
}

// Full radial of a scaled pair (these pairs are left out of the bulk
// neighbour lists and evaluated here, in FP64, with every channel):
//   Ewald: B_n = ewald_n - (1 - s lambda_n) bare_n;  bare: s lambda_n bare_n
__device__ __forceinline__ void scaled_radial(const ScaledGeom& G, double s, bool thole, bool ewald,
                                              double (&B)[6]) {
#pragma unroll
    for (int n = 0; n < 6; n++) {
        double sl = s * (thole && n >= 1 && n <= 4 ? G.lam[n] : 1.0);
        B[n] = ewald ? G.ew[n] - (1.0 - sl) * G.bare[n] : sl * G.bare[n];
    }
}

__device__ __forceinline__ Mpole<double> mpole64(const double* m) {
    Mpole<double> M;
    M.q = m[0];
    M.d = v3<double>(m[1], m[2], m[3]);
    M.Q = Sym<double>{m[4], m[5], m[6], m[7], m[8], m[9]};
    return M;
}
__device__ __forceinline__ V3<double> ld3(const double* p, int i) { return v3<double>(p[3 * i], p[3 * i + 1], p[3 * i + 2]); }
__device__ __forceinline__ void add3(double* p, int i, V3<double> v) {
    atomicAdd(p + 3 * i, v.x);
    atomicAdd(p + 3 * i + 1, v.y);
    atomicAdd(p + 3 * i + 2, v.z);
}

__global__ void k_scaled_field(int np, const ScaledPair* __restrict__ sp, const double* __restrict__ xyz,
                               const double* __restrict__ rp10, const double* __restrict__ pdamp,
                               const double* __restrict__ thole, Box bx, double cut2, double aewald,
                               double* __restrict__ Ed, double* __restrict__ Ep) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= np) return;
    ScaledPair P = sp[t];
    ScaledGeom G = scaled_geom(P, xyz, pdamp, thole, bx, cut2, aewald);
    if (!G.inside) return;
    Mpole<double> Mi = mpole64(rp10 + 10 * P.i), Mk = mpole64(rp10 + 10 * P.k);
    double Bd[6], Bp[6];
    scaled_radial(G, P.d, true, aewald > 0, Bd);
    scaled_radial(G, P.p, true, aewald > 0, Bp);
    V3<double> mr = (-1.0) * G.r;
    add3(Ed, P.k, field_of_mpole<double>(Mi, G.r, Bd[1], Bd[2], Bd[3]));
    add3(Ed, P.i, field_of_mpole<double>(Mk, mr, Bd[1], Bd[2], Bd[3]));
    add3(Ep, P.k, field_of_mpole<double>(Mi, G.r, Bp[1], Bp[2], Bp[3]));
    add3(Ep, P.i, field_of_mpole<double>(Mk, mr, Bp[1], Bp[2], Bp[3]));
}

__global__ void k_scaled_Tu(int np, const ScaledPair* __restrict__ sp, const double* __restrict__ xyz,
                            const double* __restrict__ pdamp, const double* __restrict__ thole, Box bx, double cut2,
                            double aewald, const double* __restrict__ ud, const double* __restrict__ up,
                            double* __restrict__ Fd, double* __restrict__ Fp) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= np) return;
    ScaledPair P = sp[t];
    ScaledGeom G = scaled_geom(P, xyz, pdamp, thole, bx, cut2, aewald);
    if (!G.inside) return;
    double B[6];
    scaled_radial(G, P.u, true, aewald > 0, B);
    V3<double> mr = (-1.0) * G.r;
    add3(Fd, P.k, field_of_dipole<double>(ld3(ud, P.i), G.r, B[1], B[2]));
    add3(Fd, P.i, field_of_dipole<double>(ld3(ud, P.k), mr, B[1], B[2]));
    add3(Fp, P.k, field_of_dipole<double>(ld3(up, P.i), G.r, B[1], B[2]));
    add3(Fp, P.i, field_of_dipole<double>(ld3(up, P.k), mr, B[1], B[2]));
}

// u-channel coefficients of the scaled pairs (FP64 radial, stored in R) in
// the slots after each row's bulk neighbours; pairs beyond the cutoff get
// zero coefficients.
template <class R>
__global__ void k_scaled_coeffs(int np, const ScaledPair* __restrict__ sp, const double* __restrict__ xyz,
                                const double* __restrict__ pdamp, const double* __restrict__ thole, Box bx,
                                double cut2, double aewald, const int* __restrict__ nnb, int cap,
                                const int* __restrict__ rank, int* __restrict__ cnb, R4<R>* __restrict__ c0,
                                double usolv2,
                                const int* __restrict__ nnbu, int* __restrict__ nbru, R4<R>* __restrict__ cu0) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= np) return;
    ScaledPair P = sp[t];
    ScaledGeom G = scaled_geom(P, xyz, pdamp, thole, bx, cut2, aewald);
    double B[6] = {0, 0, 0, 0, 0, 0};
    if (G.inside) scaled_radial(G, P.u, true, aewald > 0, B);
    V3<double> r = G.inside ? G.r : v3<double>(0, 0, 0);
    size_t si = (size_t)P.i * cap + nnb[P.i] + P.si;
    size_t sk = (size_t)P.k * cap + nnb[P.k] + P.sk;
    cnb[si] = rank[P.k];
    cnb[sk] = rank[P.i];
    c0[si] = pack_tensor<R>((R)(-r.x), (R)(-r.y), (R)(-r.z), (R)B[1], (R)B[2]);   // x_i - x_k
    c0[sk] = pack_tensor<R>((R)r.x, (R)r.y, (R)r.z, (R)B[1], (R)B[2]);
    if (cu0) {  // preconditioner slots after the row's compacted bulk entries; zero beyond usolvcut
        double U[6] = {0, 0, 0, 0, 0, 0};
        const bool in = G.inside && dot(G.r, G.r) <= usolv2;
        if (in) scaled_radial(G, P.u, true, false, U);
        size_t ui = (size_t)P.i * cap + nnbu[P.i] + P.si;
        size_t uk = (size_t)P.k * cap + nnbu[P.k] + P.sk;
        nbru[ui] = rank[P.k];
        nbru[uk] = rank[P.i];
        cu0[ui] = pack_tensor<R>((R)(-r.x), (R)(-r.y), (R)(-r.z), (R)U[1], (R)U[2]);
        cu0[uk] = pack_tensor<R>((R)r.x, (R)r.y, (R)r.z, (R)U[1], (R)U[2]);
    }
}

// Sparse preconditioner z = M r for both residuals:
//   z_i = alpha_i (w r_i + sum_j T_ij s_j),  s = alpha r  (packed in s4,
// cell order), T over the rows built by k_tu_coeffs / k_scaled_coeffs (bulk
// pairs within usolvcut, then the scaled partners; nbru holds the partners'
// positions in cell order).  Adds r.z of both sets to scal[RZN_D..RZN_P].
// Blocks stride over the sites (a grid of a few blocks per SM), so each block
// adds its r.z once; the last block to finish (counted in *done, which it
// resets) then rolls the PCG scalars (rz_old <- rz <- r.z) for the direction
// update that follows.
template <class R, int LPA>
__global__ void __launch_bounds__(128) k_precond(int n, const int* __restrict__ order, const int* __restrict__ nbru, const R4<R>* __restrict__ cu0,
                                                 int cap, const int* __restrict__ nnbu,
                                                 const int* __restrict__ xoff, const R4<R>* __restrict__ s4,
                                                 const double* __restrict__ pol, double wdiag,
                                                 const double* __restrict__ rd, const double* __restrict__ rp,
                                                 double* __restrict__ zd, double* __restrict__ zp,
                                                 double* __restrict__ scal, int* __restrict__ done) {
    const int lane = threadIdx.x % LPA, per_block = blockDim.x / LPA;
    double rzd = 0, rzp = 0;
    for (int g0 = blockIdx.x * per_block; g0 < n; g0 += gridDim.x * per_block) {
        const int g = g0 + threadIdx.x / LPA;
        const int gs = min(g, n - 1), i = order[gs];  // gs: the site's position in cell order
        const int cnt = g < n ? nnbu[i] + (xoff[i + 1] - xoff[i]) : 0;
        const size_t base = (size_t)i * cap;
        R ax = 0, ay = 0, az = 0, bx_ = 0, by = 0, bz = 0;
        row_apply<R, LPA, sizeof(R) == 4 ? 4 : 2>(nbru, cu0, base, cnt, lane, gs, s4, ax, ay, az, bx_, by, bz);
        double S[6];
        S[0] = group_sum<LPA>((double)ax); S[1] = group_sum<LPA>((double)ay); S[2] = group_sum<LPA>((double)az);
        S[3] = group_sum<LPA>((double)bx_); S[4] = group_sum<LPA>((double)by); S[5] = group_sum<LPA>((double)bz);
        // the group's lanes finish the six components (k = lane, lane + LPA, ...)
        if (g < n) {
            const double a = pol[i];
            for (int k = lane; k < 6; k += LPA) {
                const int c = k % 3;
                const bool dset = k < 3;
                const double Sv = k == 0 ? S[0] : k == 1 ? S[1] : k == 2 ? S[2] : k == 3 ? S[3] : k == 4 ? S[4] : S[5];
                const int q = 3 * i + c;
                const double rv = dset ? rd[q] : rp[q];
                const double z = a > 0 ? a * (wdiag * rv + Sv) : 0.0;
                (dset ? zd : zp)[q] = z;
                if (dset) rzd += rv * z; else rzp += rv * z;
            }
        }
    }
    block_sum_add(rzd, scal + RZN_D);
    block_sum_add(rzp, scal + RZN_P);
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(done, 1) == (int)gridDim.x - 1) {
            __threadfence();
            *done = 0;
            pcg_roll(scal);
        }
    }
}

// scaled pairs' contribution to em, its gradient and the torques (both
// sites, full pair in FP64); the pair virial g_k (x) r into vir when set
__global__ void k_scaled_mpole(int np, const ScaledPair* __restrict__ sp, const double* __restrict__ xyz,
                               const double* __restrict__ rp10, Box bx, double cut2, double aewald, double f,
                               double* __restrict__ grad, double* __restrict__ trq, double* __restrict__ eacc,
                               double* __restrict__ aem, const int* __restrict__ mol,
                               unsigned long long* __restrict__ npair, double* __restrict__ vir) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    double e = 0, einter = 0, w[6] = {0, 0, 0, 0, 0, 0};
    long long nz = 0;
    if (t < np) {
        ScaledPair P = sp[t];
        {
            ScaledGeom G = scaled_geom(P, xyz, nullptr, nullptr, bx, cut2, aewald);
            if (G.inside) {
                double B[6];
                scaled_radial(G, P.m, false, aewald > 0, B);
                Mpole<double> Mi = mpole64(rp10 + 10 * P.i), Mk = mpole64(rp10 + 10 * P.k);
                double E, E2;
                V3<double> gi, ti, gk, tk;
                mm_pair_i<double>(Mi, Mk, G.r, B, E, gi, ti);
                mm_pair_i<double>(Mk, Mi, (-1.0) * G.r, B, E2, gk, tk);
                e = f * E;
                nz = 2 * (E != 0.0);   // counted as two directed pairs, like the bulk kernel
                add3(grad, P.i, f * gi);
                add3(grad, P.k, f * gk);
                add3(trq, P.i, f * ti);
                add3(trq, P.k, f * tk);
                if (aem) {
                    atomicAdd(aem + P.i, 0.5 * e);
                    atomicAdd(aem + P.k, 0.5 * e);
                }
                if (mol && mol[P.i] != mol[P.k]) einter = e;
                vir_outer(w, gk.x, gk.y, gk.z, G.r.x, G.r.y, G.r.z, f);
            }
        }
    }
    block_sum_add(e, eacc);
    if (mol) block_sum_add(einter, eacc + 1);
    if (npair) block_sum_add_ll(nz, npair);
    if (vir) block_vir_add(w, vir);
}

// scaled pairs' polarization gradient and torques (full pair, FP64):
//  1/2 [E^d(M_i, up_k) + E^d(up_i, M_k) + E^p(M_i, ud_k) + E^p(ud_i, M_k)
//       + E^u(up_i, ud_k) + E^u(ud_i, up_k)]
__device__ __forceinline__ void scaled_polar_pair(const ScaledPair& P, const double* __restrict__ xyz,
                                                  const double* __restrict__ rp10, const double* __restrict__ pdamp,
                                                  const double* __restrict__ thole, Box bx, double cut2, double aewald,
                                                  const double* __restrict__ ud, const double* __restrict__ up,
                                                  int mutual, int ddonly, double f, double* __restrict__ grad,
                                                  double* __restrict__ trq, double (&w)[6]) {
    ScaledGeom G = scaled_geom(P, xyz, pdamp, thole, bx, cut2, aewald);
    if (!G.inside) return;
    double Bd[6], Bp[6], Bu[6];
    scaled_radial(G, P.d, true, aewald > 0, Bd);
    scaled_radial(G, P.p, true, aewald > 0, Bp);
    scaled_radial(G, P.u, true, aewald > 0, Bu);
    const int i = P.i, k = P.k;
    Mpole<double> Mi = mpole64(rp10 + 10 * i), Mk = mpole64(rp10 + 10 * k);
    V3<double> r = G.r, mr = (-1.0) * G.r;
    V3<double> udi = ld3(ud, i), upi = ld3(up, i), udk = ld3(ud, k), upk = ld3(up, k);
    SiteInv<double> si = invariants(Mi, r), sk = invariants(Mk, r);
    SiteInv<double> si_m = invariants(Mi, mr), sk_m = invariants(Mk, mr);
    V3<double> dEdr = v3<double>(0, 0, 0), tqi = v3<double>(0, 0, 0), tqk = v3<double>(0, 0, 0);
    V3<double> d1, t1;
    if (!ddonly) {  // ddonly: only the dipole-dipole term (OPT cross terms)
        // d channel: (M_i, up_k) and (up_i, M_k)
        md_pair<double>(Mi, si, upk, r, Bd, d1, t1);
        dEdr = dEdr + d1;
        tqi = tqi + t1;
        md_pair<double>(Mk, sk_m, upi, mr, Bd, d1, t1);   // E(M_k, up_i) seen from k: dE/d(x_i - x_k)
        dEdr = dEdr - d1;
        tqk = tqk + t1;
        // p channel: (M_i, ud_k) and (ud_i, M_k)
        md_pair<double>(Mi, si, udk, r, Bp, d1, t1);
        dEdr = dEdr + d1;
        tqi = tqi + t1;
        md_pair<double>(Mk, sk_m, udi, mr, Bp, d1, t1);
        dEdr = dEdr - d1;
        tqk = tqk + t1;
    }
    if (mutual) dEdr = dEdr + dd_pair<double>(upi, udk, r, Bu) + dd_pair<double>(udi, upk, r, Bu);
    dEdr = 0.5 * dEdr;
    add3(grad, i, (-f) * dEdr);
    add3(grad, k, f * dEdr);
    add3(trq, i, (0.5 * f) * tqi);
    add3(trq, k, (0.5 * f) * tqk);
    vir_outer(w, dEdr.x, dEdr.y, dEdr.z, r.x, r.y, r.z, f);
}

// The pair virial dG/dr (x) r goes into vir when set.
__global__ void k_scaled_polar(int np, const ScaledPair* __restrict__ sp, const double* __restrict__ xyz,
                               const double* __restrict__ rp10, const double* __restrict__ pdamp,
                               const double* __restrict__ thole, Box bx, double cut2, double aewald,
                               const double* __restrict__ ud, const double* __restrict__ up, int mutual, int ddonly,
                               double f, double* __restrict__ grad, double* __restrict__ trq,
                               double* __restrict__ vir) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    double w[6] = {0, 0, 0, 0, 0, 0};
    if (t < np)
        scaled_polar_pair(sp[t], xyz, rp10, pdamp, thole, bx, cut2, aewald, ud, up, mutual, ddonly, f, grad, trq, w);
    if (vir) block_vir_add(w, vir);
}

}  // namespace amg
