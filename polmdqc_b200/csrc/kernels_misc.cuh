// kernels_misc.cuh -- reciprocal/self finishing steps, the PCG vector
// updates (FP64 vectors, FP64 dot products), energies and torque -> force.
#pragma once
#include "kernels.cuh"
#include "kernels_pme.cuh"

namespace amg {

// Fields from the reciprocal potential (E = -grad phi) and the Ewald self
// field (4 a^3 / (3 sqrt(pi))) d; then the direct dipoles u = alpha E.
__global__ void k_field_finish(int n, const double* __restrict__ phiM, int ewald, const double* __restrict__ rp10,
                               double selfc, const double* __restrict__ pol, double* __restrict__ Ed,
                               double* __restrict__ Ep, double* __restrict__ ud, double* __restrict__ up) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (int a = 0; a < 3; a++) {
        double add = ewald ? -phiM[20 * (size_t)i + 1 + a] + selfc * rp10[10 * i + 1 + a] : 0.0;
        double ed = Ed[3 * i + a] + add, ep = Ep[3 * i + a] + add;
        Ed[3 * i + a] = ed;
        Ep[3 * i + a] = ep;
        ud[3 * i + a] = pol[i] * ed;
        up[3 * i + a] = pol[i] * ep;
    }
}

// FP64 dipole vectors -> R4 copies for the pair kernels ([n][2], d then p),
// at site i or, with rank, at the site's position in cell order (the PCG's
// stored-coefficient matvec)
template <class R>
__global__ void k_pack_u(int n, const double* __restrict__ ud, const double* __restrict__ up, R4<R>* __restrict__ u4,
                         const int* __restrict__ rank = nullptr) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int o = rank ? rank[i] : i;
    u4[2 * o] = make_r4<R>((R)ud[3 * i], (R)ud[3 * i + 1], (R)ud[3 * i + 2], R(0));
    u4[2 * o + 1] = make_r4<R>((R)up[3 * i], (R)up[3 * i + 1], (R)up[3 * i + 2], R(0));
}

// A v = v/alpha - (real + recip + self) field of v, both sets; pol = 0 sites
// give 0.  phi: [2][n][4] reciprocal potentials (0 and first derivatives).
__global__ void k_matvec_finish(int n, const double* __restrict__ vd, const double* __restrict__ vp,
                                const double* __restrict__ Fd, const double* __restrict__ Fp,
                                const double* __restrict__ phi, int ewald, double selfc,
                                const double* __restrict__ pol, double* __restrict__ Ad, double* __restrict__ Ap) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double a = pol[i];
    double ia = a > 0 ? 1.0 / a : 0.0;
    for (int c = 0; c < 3; c++) {
        double fd = Fd[3 * i + c], fp = Fp[3 * i + c];
        if (ewald) {
            fd += -phi[4 * (size_t)i + 1 + c] + selfc * vd[3 * i + c];
            fp += -phi[4 * ((size_t)n + i) + 1 + c] + selfc * vp[3 * i + c];
        }
        Ad[3 * i + c] = a > 0 ? ia * vd[3 * i + c] - fd : 0.0;
        Ap[3 * i + c] = a > 0 ? ia * vp[3 * i + c] - fp : 0.0;
    }
}

// scalar slots of the PCG (device memory)

template <class T>
__global__ void k_zero(T* __restrict__ p, size_t n) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = T(0);
}


__global__ void k_pcg_control(double* __restrict__ scal, int* __restrict__ iter, double thr2, int maxit, int first,
                              int roll, cudaGraphConditionalHandle h, int use_handle, int* __restrict__ cont_out) {
    pcg_decide(scal, iter, thr2, maxit, first, roll, h, use_handle, cont_out);
}

// r = E - A u and rr.  Diagonal preconditioner (s4 null): z = alpha r and
// rz.  Sparse preconditioner: s = alpha r packed into s4 for k_precond, which
// forms z and rz.
template <class R>
__global__ void k_pcg_init(int n, const double* __restrict__ Ed, const double* __restrict__ Ep,
                           const double* __restrict__ Aud, const double* __restrict__ Aup,
                           const double* __restrict__ pol, double* __restrict__ rd, double* __restrict__ rp,
                           double* __restrict__ zd, double* __restrict__ zp, double* __restrict__ scal,
                           R4<R>* __restrict__ s4, const int* __restrict__ rank) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double rzd = 0, rzp = 0, rrd = 0, rrp = 0;
    if (i < n) {
        double a = pol[i];
        double sv[6];
        for (int c = 0; c < 3; c++) {
            int q = 3 * i + c;
            double r1 = a > 0 ? Ed[q] - Aud[q] : 0.0, r2 = a > 0 ? Ep[q] - Aup[q] : 0.0;
            rd[q] = r1; rp[q] = r2;
            double z1 = a * r1, z2 = a * r2;
            sv[c] = z1; sv[3 + c] = z2;
            if (!s4) {
                zd[q] = z1; zp[q] = z2;
                rzd += r1 * z1; rzp += r2 * z2;
            }
            rrd += r1 * r1; rrp += r2 * r2;
        }
        if (s4) {
            s4[2 * rank[i]] = make_r4<R>((R)sv[0], (R)sv[1], (R)sv[2], R(0));
            s4[2 * rank[i] + 1] = make_r4<R>((R)sv[3], (R)sv[4], (R)sv[5], R(0));
        }
    }
    if (!s4) {
        block_sum_add(rzd, scal + RZ_D);
        block_sum_add(rzp, scal + RZ_P);
    }
    block_sum_add(rrd, scal + RR_D);
    block_sum_add(rrp, scal + RR_P);
}

__global__ void k_dot2(int n3, const double* __restrict__ a1, const double* __restrict__ b1,
                       const double* __restrict__ a2, const double* __restrict__ b2, double* __restrict__ o1,
                       double* __restrict__ o2) {
    int q = blockIdx.x * blockDim.x + threadIdx.x;
    double s1 = 0, s2 = 0;
    if (q < n3) { s1 = a1[q] * b1[q]; s2 = a2[q] * b2[q]; }
    block_sum_add(s1, o1);
    block_sum_add(s2, o2);
}

// u += a p; r -= a Ap; rr  (a = rz / pAp per set).  Diagonal
// preconditioner (s4 null): z = alpha r and rz_new; sparse preconditioner:
// s = alpha r packed into s4 for k_precond.  With Fd, Fp the stored Apd, App
// lack the real-space part, and A p = Apd - Fd (see k_gather_field).  The
// last block takes the PCG control decision (pcg_decide).
template <class R>
__global__ void k_pcg_update(int n, const double* __restrict__ pol, const double* __restrict__ pd,
                             const double* __restrict__ pp, const double* __restrict__ Apd,
                             const double* __restrict__ App, double* __restrict__ ud, double* __restrict__ up,
                             double* __restrict__ rd, double* __restrict__ rp, double* __restrict__ zd,
                             double* __restrict__ zp, double* __restrict__ scal, R4<R>* __restrict__ s4,
                             const int* __restrict__ rank, const double* __restrict__ Fd,
                             const double* __restrict__ Fp, int* __restrict__ done, int* __restrict__ iter,
                             double thr2, int maxit, int roll, cudaGraphConditionalHandle h, int use_handle,
                             int* __restrict__ cont_out) {
    // one thread per vector component q = 3i + c (the site loop had too few
    // threads in flight for its chains of dependent loads), blocks striding
    // over the components so that few blocks add to the scalars
    double ad = scal[PAP_D] != 0 ? scal[RZ_D] / scal[PAP_D] : 0.0;
    double ap = scal[PAP_P] != 0 ? scal[RZ_P] / scal[PAP_P] : 0.0;
    double rzd = 0, rzp = 0, rrd = 0, rrp = 0;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < 3 * n; q += gridDim.x * blockDim.x) {
        const int i = q / 3, c = q - 3 * (q / 3);
        const double a = pol[i];
        ud[q] += ad * pd[q];
        up[q] += ap * pp[q];
        const double Aq1 = Fd ? Apd[q] - Fd[q] : Apd[q], Aq2 = Fp ? App[q] - Fp[q] : App[q];
        const double r1 = rd[q] - ad * Aq1, r2 = rp[q] - ap * Aq2;
        rd[q] = r1; rp[q] = r2;
        const double z1 = a * r1, z2 = a * r2;
        if (s4) {  // the scaled residual in cell order, both sets (x, y, z of each R4)
            R* sv = reinterpret_cast<R*>(s4 + 2 * (size_t)rank[i]);
            sv[c] = (R)z1;
            sv[4 + c] = (R)z2;
        } else {
            zd[q] = z1; zp[q] = z2;
            rzd += r1 * z1; rzp += r2 * z2;
        }
        rrd += r1 * r1; rrp += r2 * r2;
    }
    if (!s4) {
        block_sum_add(rzd, scal + RZN_D);
        block_sum_add(rzp, scal + RZN_P);
    }
    block_sum_add(rrd, scal + RR_D);
    block_sum_add(rrp, scal + RR_P);
    // the last block to finish (counted in *done, which it resets) takes the
    // control decision: every block has added its r.r by then
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(done, 1) == (int)gridDim.x - 1) {
            __threadfence();
            *done = 0;
            pcg_decide(scal, iter, thr2, maxit, 0, roll, h, use_handle, cont_out);
        }
    }
}

// beta = rz / rz_old after the scalars were rolled (0 on the first iteration)
__device__ __forceinline__ void pcg_beta(const double* __restrict__ scal, double& bd, double& bp) {
    bd = scal[RZO_D] != 0 ? scal[RZ_D] / scal[RZO_D] : 0.0;
    bp = scal[RZO_P] != 0 ? scal[RZ_P] / scal[RZO_P] : 0.0;
}

// p = z + beta p; p = z when beta = 0 (the first direction, whose old p is
// not defined)
__device__ __forceinline__ double pcg_dir_value(double z, double beta, double p) {
    return beta != 0 ? z + beta * p : z;
}

// p = z + beta p and its R4 copy (after the rz scalars were rolled)
template <class R>
__global__ void k_pcg_dir(int n, const double* __restrict__ zd, const double* __restrict__ zp,
                          double* __restrict__ pd, double* __restrict__ pp, const double* __restrict__ scal,
                          R4<R>* __restrict__ p4, const int* __restrict__ rank) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double bd, bp;
    pcg_beta(scal, bd, bp);
    double a[3], b[3];
    for (int c = 0; c < 3; c++) {
        int q = 3 * i + c;
        a[c] = pcg_dir_value(zd[q], bd, pd[q]);
        b[c] = pcg_dir_value(zp[q], bp, pp[q]);
        pd[q] = a[c];
        pp[q] = b[c];
    }
    p4[2 * rank[i]] = make_r4<R>((R)a[0], (R)a[1], (R)a[2], R(0));
    p4[2 * rank[i] + 1] = make_r4<R>((R)b[0], (R)b[1], (R)b[2], R(0));
}

// p = z + beta p (after the rz scalars were rolled) fused with the spreading of
// p into the complex grid zg for the next matvec (zg holds the cleared grid
// left by the previous transform), in the layout of k_spread_dipoles: FP32,
// kLineSites sites per block of 128 threads and one z-line per thread; FP64,
// one site per block and one stencil point per thread.  The first 6 threads
// per site form p (and its R4 copy).
template <class R, int P>
__global__ void __launch_bounds__(128) k_pcg_dir_spread(int n, const double* __restrict__ zd,
                                                        const double* __restrict__ zp, double* __restrict__ pd,
                                                        double* __restrict__ pp, const double* __restrict__ scal,
                                                        R4<R>* __restrict__ p4, const R* __restrict__ theta,
                                                        const int* __restrict__ k0, int3 K, Frac F,
                                                        typename Cplx<R>::type* __restrict__ zg,
                                                        const int* __restrict__ rank) {
    constexpr int SPB = sizeof(R) == 8 ? 1 : kLineSites;  // sites per block
    __shared__ double pv[SPB][6];
    const int t = threadIdx.x, i0 = blockIdx.x * SPB;
    if (t < 6 * SPB) {
        const int s = t / 6, k = t % 6, i = i0 + s;
        if (i < n) {
            double bd, bp;
            pcg_beta(scal, bd, bp);
            const int q = 3 * i + k % 3;
            const double v = k < 3 ? pcg_dir_value(zd[q], bd, pd[q]) : pcg_dir_value(zp[q], bp, pp[q]);
            (k < 3 ? pd : pp)[q] = v;
            pv[s][k] = v;
        }
    }
    __syncthreads();
    if (t < SPB && i0 + t < n) {
        const double* v = pv[t];
        const int o = rank[i0 + t];  // p4 in cell order
        p4[2 * o] = make_r4<R>((R)v[0], (R)v[1], (R)v[2], R(0));
        p4[2 * o + 1] = make_r4<R>((R)v[3], (R)v[4], (R)v[5], R(0));
    }
    if constexpr (SPB == 1) {
        if (t >= P * P * P || i0 >= n) return;
        spread_site_point<R, P>(i0, t, pv[0], pv[0] + 3, theta, k0, K, F, zg);
    } else {
        const int s = t / (P * P), i = i0 + s;
        if (t >= SPB * P * P || i >= n) return;
        spread_site_line<R, P>(i, t % (P * P), pv[s], pv[s] + 3, theta, k0, K, F, zg);
    }
}

// One preconditioned correction step u += alpha r with the FP64 residual
// r = E - A u, and the norms of that residual.
__global__ void k_correct(int n, const double* __restrict__ Ed, const double* __restrict__ Ep,
                          const double* __restrict__ Aud, const double* __restrict__ Aup,
                          const double* __restrict__ pol, double* __restrict__ ud, double* __restrict__ up,
                          double* __restrict__ resd, double* __restrict__ scal) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double rrd = 0, rrp = 0, urd = 0;
    if (i < n) {
        double a = pol[i];
        for (int c = 0; c < 3; c++) {
            int q = 3 * i + c;
            double r1 = a > 0 ? Ed[q] - Aud[q] : 0.0, r2 = a > 0 ? Ep[q] - Aup[q] : 0.0;
            rrd += r1 * r1; rrp += r2 * r2;
            urd += up[q] * r1;   // up . r_d (before the update) for the stationary energy
            resd[q] = r1;
            ud[q] += a * r1;
            up[q] += a * r2;
        }
    }
    block_sum_add(rrd, scal + RR_D);
    block_sum_add(rrp, scal + RR_P);
    block_sum_add(urd, scal + RZN_D);
}

// ep = -1/2 f sum ud . Ep (per-site aep when requested); nep = sites with
// nonzero energy
__global__ void k_polar_energy(int n, const double* __restrict__ ud, const double* __restrict__ Ep, double f,
                               double* __restrict__ eacc, double* __restrict__ aep,
                               unsigned long long* __restrict__ nep) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double e = 0;
    long long c = 0;
    if (i < n) {
        e = -0.5 * f * (ud[3 * i] * Ep[3 * i] + ud[3 * i + 1] * Ep[3 * i + 1] + ud[3 * i + 2] * Ep[3 * i + 2]);
        if (aep) aep[i] = e;
        c = e != 0.0;
    }
    block_sum_add(e, eacc);
    block_sum_add_ll(c, nep);
}

// ---------------------------------------------------------------- reciprocal
__device__ __forceinline__ double site_energy(const double* m, const double* p) {
    return m[0] * p[0] + m[1] * p[1] + m[2] * p[2] + m[3] * p[3] + m[4] * p[4] + m[7] * p[5] + m[9] * p[6] +
           2 * (m[5] * p[7] + m[6] * p[8] + m[8] * p[9]);
}
// d/dx_site (M . phi): q grad phi + d.grad grad phi + Q:grad^3 phi
__device__ __forceinline__ V3<double> site_gradient(const double* m, const double* p) {
    double q = m[0], dx = m[1], dy = m[2], dz = m[3], Qxx = m[4], Qxy = m[5], Qxz = m[6], Qyy = m[7], Qyz = m[8],
           Qzz = m[9];
    V3<double> g;
    g.x = q * p[1] + dx * p[4] + dy * p[7] + dz * p[8] + Qxx * p[10] + Qyy * p[15] + Qzz * p[17] +
          2 * (Qxy * p[13] + Qxz * p[14] + Qyz * p[19]);
    g.y = q * p[2] + dx * p[7] + dy * p[5] + dz * p[9] + Qxx * p[13] + Qyy * p[11] + Qzz * p[18] +
          2 * (Qxy * p[15] + Qxz * p[19] + Qyz * p[16]);
    g.z = q * p[3] + dx * p[8] + dy * p[9] + dz * p[6] + Qxx * p[14] + Qyy * p[16] + Qzz * p[12] +
          2 * (Qxy * p[19] + Qxz * p[17] + Qyz * p[18]);
    return g;
}
// dipole-only version (v . grad grad phi)
__device__ __forceinline__ V3<double> dipole_gradient(V3<double> v, const double* p) {
    return v3<double>(v.x * p[4] + v.y * p[7] + v.z * p[8], v.x * p[7] + v.y * p[5] + v.z * p[9],
                      v.x * p[8] + v.y * p[9] + v.z * p[6]);
}
// torque -dE/dtheta of E = M . phi
__device__ __forceinline__ V3<double> site_torque(const double* m, const double* p) {
    V3<double> d = v3<double>(m[1], m[2], m[3]);
    V3<double> t = (-1.0) * cross(d, v3<double>(p[1], p[2], p[3]));
    Sym<double> Q{m[4], m[5], m[6], m[7], m[8], m[9]};
    Sym<double> H{p[4], p[7], p[8], p[5], p[9], p[6]};
    return t - 2.0 * axial_prod(Q, H);
}

// Multipole term of the reciprocal virial: at fixed fractional coordinates a
// strain acts on the structure factor as if each source were deformed,
// d -> (1 - eps) d, Q -> Q - eps Q - Q eps^T; with phi the derivative of the
// energy with respect to the source, v += s sym(-(grad phi) (x) d - 2 H Q),
// H = grad grad phi.  Q is skipped for a dipole-only source (m[4] unused).
__device__ __forceinline__ void vir_source(double (&v)[6], const double* m, bool quad, const double* p, double s) {
    vir_outer(v, p[1], p[2], p[3], m[1], m[2], m[3], -s);
    if (!quad) return;
    const double Q[3][3] = {{m[4], m[5], m[6]}, {m[5], m[7], m[8]}, {m[6], m[8], m[9]}};
    const double H[3][3] = {{p[4], p[7], p[8]}, {p[7], p[5], p[9]}, {p[8], p[9], p[6]}};
    double HQ[3][3];
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) HQ[a][b] = H[a][0] * Q[0][b] + H[a][1] * Q[1][b] + H[a][2] * Q[2][b];
    v[0] -= 2 * s * HQ[0][0];
    v[1] -= 2 * s * HQ[1][1];
    v[2] -= 2 * s * HQ[2][2];
    v[3] -= s * (HQ[0][1] + HQ[1][0]);
    v[4] -= s * (HQ[0][2] + HQ[2][0]);
    v[5] -= s * (HQ[1][2] + HQ[2][1]);
}

__device__ __forceinline__ void vir_dipole(double (&v)[6], V3<double> u, const double* p, double s) {
    const double m[4] = {0, u.x, u.y, u.z};
    vir_source(v, m, false, p, s);
}

// permanent reciprocal energy 1/2 M.phi, gradient, torque; self energy;
// per-site energies on request; the multipole term of the reciprocal virial
// into vir when set
__global__ void k_recip_mpole(int n, const double* __restrict__ rp10, const double* __restrict__ phiM, double f,
                              double alpha, double* __restrict__ grad, double* __restrict__ trq,
                              double* __restrict__ eacc, double* __restrict__ aem, double* __restrict__ qsum,
                              double* __restrict__ vir) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double e = 0, q = 0, w[6] = {0, 0, 0, 0, 0, 0};
    if (i < n) {
        const double* m = rp10 + 10 * i;
        const double* p = phiM + 20 * (size_t)i;
        double er = 0.5 * site_energy(m, p);
        double d2 = m[1] * m[1] + m[2] * m[2] + m[3] * m[3];
        double qq = m[4] * m[4] + m[7] * m[7] + m[9] * m[9] + 2 * (m[5] * m[5] + m[6] * m[6] + m[8] * m[8]);
        double a2 = alpha * alpha;
        double es = -(alpha / kSqrtPi) * (m[0] * m[0] + (2 * a2 / 3) * d2 + (8 * a2 * a2 / 5) * qq);
        e = f * (er + es);
        q = m[0];
        V3<double> g = site_gradient(m, p), t = site_torque(m, p);
        grad[3 * i] += f * g.x; grad[3 * i + 1] += f * g.y; grad[3 * i + 2] += f * g.z;
        trq[3 * i] += f * t.x; trq[3 * i + 1] += f * t.y; trq[3 * i + 2] += f * t.z;
        if (aem) aem[i] += e;
        if (vir) vir_source(w, m, true, p, f);
    }
    block_sum_add(e, eacc);
    block_sum_add(q, qsum);
    if (vir) block_vir_add(w, vir);
}

// reciprocal + self part of the polarization gradient and torques:
//   dG/dx_i = 1/2 [(up+ud)_i . grad grad phiM + M_i . grad(phi_p + phi_d)
//                  + up_i . grad grad phi_d + ud_i . grad grad phi_p]
//   torque  = torque(M_i, (phi_d + phi_p)/2) + (selfc/2) d_i x (ud + up)_i
// and, into vir when set, the multipole terms of the reciprocal virial of
//   G = 1/2 [U(up, M) + U(ud, M) + U(up, ud)].
// ddonly: the dipole-dipole part alone, 1/2 U(up, ud) (the OPT cross terms).
__global__ void k_recip_polar(int n, const double* __restrict__ rp10, const double* __restrict__ phiM,
                              const double* __restrict__ phid, const double* __restrict__ phip,
                              const double* __restrict__ ud, const double* __restrict__ up, int mutual,
                              int ddonly, double selfc, double f, double* __restrict__ grad,
                              double* __restrict__ trq, double* __restrict__ vir) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double w[6] = {0, 0, 0, 0, 0, 0};
    if (i < n && ddonly) {
        const double* pd = phid + 20 * (size_t)i;
        const double* pp = phip + 20 * (size_t)i;
        V3<double> udi = ld3(ud, i), upi = ld3(up, i);
        V3<double> g = (0.5 * f) * (dipole_gradient(upi, pd) + dipole_gradient(udi, pp));
        grad[3 * i] += g.x; grad[3 * i + 1] += g.y; grad[3 * i + 2] += g.z;
        if (vir) {
            vir_dipole(w, upi, pd, 0.5 * f);
            vir_dipole(w, udi, pp, 0.5 * f);
        }
    } else if (i < n) {
        const double* m = rp10 + 10 * i;
        const double* pm = phiM + 20 * (size_t)i;
        const double* pd = phid + 20 * (size_t)i;
        const double* pp = phip + 20 * (size_t)i;
        V3<double> udi = ld3(ud, i), upi = ld3(up, i);
        double avg[20];
        for (int j = 0; j < 20; j++) avg[j] = pd[j] + pp[j];
        V3<double> g = dipole_gradient(udi + upi, pm) + site_gradient(m, avg);
        if (mutual) g = g + dipole_gradient(upi, pd) + dipole_gradient(udi, pp);
        g = (0.5 * f) * g;
        for (int j = 0; j < 20; j++) avg[j] *= 0.5;
        V3<double> t = site_torque(m, avg) + (0.5 * selfc) * cross(v3<double>(m[1], m[2], m[3]), udi + upi);
        t = f * t;
        grad[3 * i] += g.x; grad[3 * i + 1] += g.y; grad[3 * i + 2] += g.z;
        trq[3 * i] += t.x; trq[3 * i + 1] += t.y; trq[3 * i + 2] += t.z;
        if (vir) {
            const double h = 0.5 * f;
            vir_dipole(w, upi + udi, pm, h);   // U(up, M) + U(ud, M): dipoles in phiM
            vir_source(w, m, true, avg, f);    // ... and M in phi_p + phi_d (avg holds half the sum)
            if (mutual) {                      // U(up, ud)
                vir_dipole(w, upi, pd, h);
                vir_dipole(w, udi, pp, h);
            }
        }
    }
    if (vir) block_vir_add(w, vir);
}

// ---------------------------------------------------------------- OPT
// Extrapolated perturbation theory: u^(0) = alpha E, u^(k) = alpha T u^(k-1),
// u = sum_k copm_k u^(k) for both sets.  uo: [K+1][2][3n] (d then p).
struct OptCoef {
    double c[8];
};

// u^(0) from the direct dipoles (ud, up), which become copm_0 u^(0)
__global__ void k_opt_init(int n3, double c0, double* __restrict__ ud, double* __restrict__ up,
                           double* __restrict__ u0d, double* __restrict__ u0p) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n3) return;
    u0d[t] = ud[t];
    u0p[t] = up[t];
    ud[t] *= c0;
    up[t] *= c0;
}

// u^(k) = alpha T v = v - alpha (A v), A v = v/alpha - T v; u += c u^(k)
__global__ void k_opt_step(int n3, const double* __restrict__ pol, const double* __restrict__ vd,
                           const double* __restrict__ vp, const double* __restrict__ Ad, const double* __restrict__ Ap,
                           double c, double* __restrict__ od, double* __restrict__ op, double* __restrict__ ud,
                           double* __restrict__ up) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n3) return;
    const double a = pol[t / 3];
    const double d = vd[t] - a * Ad[t], p = vp[t] - a * Ap[t];
    od[t] = d;
    op[t] = p;
    ud[t] += c * d;
    up[t] += c * p;
}

// V_b = sum_{a + b + 1 <= K} copm_{a+b+1} up^(a): the p-side partner of
// ud^(b) in the dipole-dipole force terms
__global__ void k_opt_cross(int n3, int K, int b, OptCoef cm, const double* __restrict__ uo, double* __restrict__ out) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n3) return;
    double v = 0;
    for (int a = 0; a + b + 1 <= K; a++) v += cm.c[a + b + 1] * uo[(size_t)(2 * a + 1) * n3 + t];
    out[t] = v;
}

// ---------------------------------------------------------------- torque
// Site torques -> gradients on the frame atoms, restating the reference's
// torque (src/md/torque.cpp:42-397; Popelier & Stone 1994, Sagui et al.
// 2004).  Gradients are accumulated with FP64 atomics (frame atoms are shared).
// With vir set, the frame atoms' share of the virial: each frame atom's
// gradient times its offset from the site (src/md/torque.cpp:360-395).
__device__ __forceinline__ void torque_site(int i, const double* __restrict__ xyz, const int* __restrict__ zax,
                                            const int* __restrict__ xax, const int* __restrict__ yax,
                                            const int* __restrict__ axe, const double* __restrict__ trq,
                                            double* __restrict__ grad, double (*vacc)[6]);

__global__ void k_torque(int n, const double* __restrict__ xyz, const int* __restrict__ zax,
                         const int* __restrict__ xax, const int* __restrict__ yax, const int* __restrict__ axe,
                         const double* __restrict__ trq, double* __restrict__ grad, double* __restrict__ vir) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double w[6] = {0, 0, 0, 0, 0, 0};
    if (i < n && axe[i] != AMG_FRAME_NONE) torque_site(i, xyz, zax, xax, yax, axe, trq, grad, vir ? &w : nullptr);
    if (vir) block_vir_add(w, vir);
}

__device__ __forceinline__ void torque_site(int i, const double* __restrict__ xyz, const int* __restrict__ zax,
                                            const int* __restrict__ xax, const int* __restrict__ yax,
                                            const int* __restrict__ axe, const double* __restrict__ trq,
                                            double* __restrict__ grad, double (*vacc)[6]) {
    const int ft = axe[i];
    using D = double;
    auto P = [&](int a) { return v3<D>(xyz[3 * a], xyz[3 * a + 1], xyz[3 * a + 2]); };
    auto unit = [](V3<D> v) { D s = 1.0 / sqrt(dot(v, v)); return s * v; };
    int ia = zax[i] - 1, ib = i, ic = xax[i] - 1, id = abs(yax[i]) - 1;
    V3<D> t = v3<D>(trq[3 * i], trq[3 * i + 1], trq[3 * i + 2]);
    V3<D> u = P(ia) - P(ib);
    D us = sqrt(dot(u, u));
    V3<D> v;
    D vs;
    if (ft != AMG_FRAME_ZONLY) {
        v = P(ic) - P(ib);
        vs = sqrt(dot(v, v));
    } else {
        v = fabs(u.x / us) > 0.866 ? v3<D>(0, 1, 0) : v3<D>(1, 0, 0);
        vs = 1;
    }
    V3<D> w = (ft == AMG_FRAME_ZBISECT || ft == AMG_FRAME_THREEFOLD) ? P(id) - P(ib) : cross(u, v);
    D ws = sqrt(dot(w, w));
    u = (1.0 / us) * u;
    v = (1.0 / vs) * v;
    w = (1.0 / ws) * w;
    D dpu = -dot(t, u), dpv = -dot(t, v), dpw = -dot(t, w);
    V3<D> uv = unit(cross(v, u)), uw = unit(cross(w, u)), vw = unit(cross(w, v));
    D uvc = dot(u, v), uvsn = sqrt(1 - uvc * uvc);
    auto add = [&](int at, V3<D> g) {
        atomicAdd(grad + 3 * at, g.x);
        atomicAdd(grad + 3 * at + 1, g.y);
        atomicAdd(grad + 3 * at + 2, g.z);
        if (vacc && at != ib) {
            V3<D> o = P(at) - P(ib);
            vir_outer(*vacc, g.x, g.y, g.z, o.x, o.y, o.z, 1.0);
        }
    };
    if (ft == AMG_FRAME_ZONLY) {
        V3<D> du = (dpv / (us * uvsn)) * uv + (dpw / us) * uw;
        add(ia, du);
        add(ib, (-1.0) * du);
    } else if (ft == AMG_FRAME_ZTHENX) {
        V3<D> du = (dpv / (us * uvsn)) * uv + (dpw / us) * uw;
        V3<D> dv = (-dpu / (vs * uvsn)) * uv;
        add(ia, du);
        add(ic, dv);
        add(ib, (-1.0) * (du + dv));
    } else if (ft == AMG_FRAME_BISECTOR) {
        V3<D> du = (dpv / (us * uvsn)) * uv + (0.5 * dpw / us) * uw;
        V3<D> dv = (-dpu / (vs * uvsn)) * uv + (0.5 * dpw / vs) * vw;
        add(ia, du);
        add(ic, dv);
        add(ib, (-1.0) * (du + dv));
    } else if (ft == AMG_FRAME_ZBISECT) {
        V3<D> r = unit(v + w);
        V3<D> s = unit(cross(u, r));
        D dpr = -dot(t, r), dps = -dot(t, s);
        V3<D> ur = unit(cross(r, u)), us_ = unit(cross(s, u));
        D urc = dot(u, r), ursn = sqrt(1 - urc * urc);
        D vsc = dot(v, s), vssn = sqrt(1 - vsc * vsc);
        D wsc = dot(w, s), wssn = sqrt(1 - wsc * wsc);
        V3<D> t1 = unit(v - vsc * s), t2 = unit(w - wsc * s);
        D ut1c = dot(u, t1), ut1s = sqrt(1 - ut1c * ut1c);
        D ut2c = dot(u, t2), ut2s = sqrt(1 - ut2c * ut2c);
        V3<D> du = (dpr / (us * ursn)) * ur + (dps / us) * us_;
        V3<D> dv = (dpu / (vs * (ut1s + ut2s))) * (vssn * s - vsc * t1);
        V3<D> dw = (dpu / (ws * (ut1s + ut2s))) * (wssn * s - wsc * t2);
        add(ia, du);
        add(ic, dv);
        add(id, dw);
        add(ib, (-1.0) * (du + dv + dw));
    } else if (ft == AMG_FRAME_THREEFOLD) {
        V3<D> sum = u + v + w;
        D ps = sqrt(dot(sum, sum));
        V3<D> p = (1.0 / ps) * sum;
        D wpc = dot(w, p), upc = dot(u, p), vpc = dot(v, p);
        auto leg = [&](V3<D> a1, V3<D> a2, V3<D> self, D selfsiz, D selfpc, int atom) {
            V3<D> rr = unit(a1 + a2);
            D c = dot(rr, self), sn = sqrt(1 - c * c);
            D dpr_ = -dot(t, rr);
            V3<D> del = unit(cross(rr, self));
            D dpd = -dot(t, del);
            V3<D> eps = cross(del, self);
            V3<D> g = (dpr_ / (selfsiz * sn)) * del + (dpd * selfpc / (selfsiz * ps)) * eps;
            add(atom, g);
            add(ib, (-1.0) * g);
        };
        leg(u, v, w, ws, wpc, id);
        leg(v, w, u, us, upc, ia);
        leg(u, w, v, vs, vpc, ic);
    }
}

// ------------------------------------------------------------ predictor
// History of converged dipoles: slots [kPredSteps][2][3n] (u_d then u_p),
// state[0] = the slot the next evaluation writes, state[1] = filled slots.
constexpr int kPredSteps = 6;
struct PredCoef {
    double b[kPredSteps];  // b[j-1] multiplies the dipoles of evaluation n-j
};

// starting dipoles sum_j b_j u(n-j) once the history is full (else the
// direct dipoles already in ud/up stay)
__global__ void k_predict(int n3, const double* __restrict__ hist, const int* __restrict__ state, PredCoef c,
                          double* __restrict__ ud, double* __restrict__ up) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n3 || state[1] < kPredSteps) return;
    const int next = state[0];
    double vd = 0, vp = 0;
#pragma unroll
    for (int j = 1; j <= kPredSteps; j++) {
        const int slot = (next - j + kPredSteps) % kPredSteps;
        const double* h = hist + (size_t)slot * 2 * n3;
        vd += c.b[j - 1] * h[t];
        vp += c.b[j - 1] * h[n3 + t];
    }
    ud[t] = vd;
    up[t] = vp;
}

// the converged dipoles into the next slot
__global__ void k_pred_store(int n3, double* __restrict__ hist, const int* __restrict__ state,
                             const double* __restrict__ ud, const double* __restrict__ up) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n3) return;
    double* h = hist + (size_t)state[0] * 2 * n3;
    h[t] = ud[t];
    h[n3 + t] = up[t];
}

__global__ void k_pred_advance(int* __restrict__ state) {
    state[0] = (state[0] + 1) % kPredSteps;
    state[1] = min(state[1] + 1, kPredSteps);
}

}  // namespace amg
