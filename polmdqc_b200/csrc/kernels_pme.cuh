// kernels_pme.cuh -- smooth PME for multipoles and induced dipoles
// (Essmann et al. 1995; multipoles as Sagui, Pedersen & Darden 2004):
// fractional multipoles spread with order-P B-splines, R2C FFT (cuFFT),
// a hand-written convolution with the influence function, C2R, and gathers
// of up to 20 potential derivatives per site.
#pragma once
#include "kernels.cuh"

namespace amg {

template <class R>
struct Cplx;
template <>
struct Cplx<float> {
    using type = float2;
};
template <>
struct Cplx<double> {
    using type = double2;
};

__device__ __forceinline__ int gidx(int a, int b, int c, int3 K) { return (a * K.y + b) * K.z + c; }

// Spread the permanent multipoles (global frame, FP64 rp10) as fractional
// multipoles: grid(g) += q t0u0v0 + sum_a d'_a (first derivative in a) +
// sum_ab Q'_ab (second derivatives), with d' = (K/L) d, Q' = (K/L)(K/L) Q.
template <class R, int P>
__global__ void k_spread_mpole(int n, const double* __restrict__ rp10, const R* __restrict__ theta,
                               const int* __restrict__ k0, int3 K, R sc0, R sc1, R sc2, R* __restrict__ grid) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double* m = rp10 + 10 * i;
    R q = (R)m[0];
    R d1 = (R)m[1] * sc0, d2 = (R)m[2] * sc1, d3 = (R)m[3] * sc2;
    R q11 = (R)m[4] * sc0 * sc0, q22 = (R)m[7] * sc1 * sc1, q33 = (R)m[9] * sc2 * sc2;
    R q12 = 2 * (R)m[5] * sc0 * sc1, q13 = 2 * (R)m[6] * sc0 * sc2, q23 = 2 * (R)m[8] * sc1 * sc2;
    const R* t1 = theta + ((size_t)i * 3 + 0) * 4 * P;
    const R* t2 = theta + ((size_t)i * 3 + 1) * 4 * P;
    const R* t3 = theta + ((size_t)i * 3 + 2) * 4 * P;
    int a0 = k0[3 * i], b0 = k0[3 * i + 1], c0 = k0[3 * i + 2];
    for (int c = 0; c < P; c++) {
        R v0 = t3[c], v1 = t3[P + c], v2 = t3[2 * P + c];
        int gc = c0 + c; if (gc >= K.z) gc -= K.z;
        for (int b = 0; b < P; b++) {
            R u0 = t2[b], u1 = t2[P + b], u2 = t2[2 * P + b];
            int gb = b0 + b; if (gb >= K.y) gb -= K.y;
            // coefficients of t0, t1, t2 (x derivatives) for this (b, c)
            R w0 = q * u0 * v0 + d2 * u1 * v0 + d3 * u0 * v1 + q22 * u2 * v0 + q33 * u0 * v2 + q23 * u1 * v1;
            R w1 = d1 * u0 * v0 + q12 * u1 * v0 + q13 * u0 * v1;
            R w2 = q11 * u0 * v0;
            for (int a = 0; a < P; a++) {
                int ga = a0 + a; if (ga >= K.x) ga -= K.x;
                R val = t1[a] * w0 + t1[P + a] * w1 + t1[2 * P + a] * w2;
                atomicAdd(grid + gidx(ga, gb, gc, K), val);
            }
        }
    }
}

// Spread two sets of dipoles (FP64 [3n] each) onto two grids.
template <class R, int P>
__global__ void k_spread_dipoles(int n, const double* __restrict__ ud, const double* __restrict__ up,
                                 const R* __restrict__ theta, const int* __restrict__ k0, int3 K, R sc0, R sc1,
                                 R sc2, R* __restrict__ grid, size_t gstride) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    R da[3] = {(R)ud[3 * i] * sc0, (R)ud[3 * i + 1] * sc1, (R)ud[3 * i + 2] * sc2};
    R pa[3] = {(R)up[3 * i] * sc0, (R)up[3 * i + 1] * sc1, (R)up[3 * i + 2] * sc2};
    const R* t1 = theta + ((size_t)i * 3 + 0) * 4 * P;
    const R* t2 = theta + ((size_t)i * 3 + 1) * 4 * P;
    const R* t3 = theta + ((size_t)i * 3 + 2) * 4 * P;
    int a0 = k0[3 * i], b0 = k0[3 * i + 1], c0 = k0[3 * i + 2];
    for (int c = 0; c < P; c++) {
        R v0 = t3[c], v1 = t3[P + c];
        int gc = c0 + c; if (gc >= K.z) gc -= K.z;
        for (int b = 0; b < P; b++) {
            R u0 = t2[b], u1 = t2[P + b];
            int gb = b0 + b; if (gb >= K.y) gb -= K.y;
            R wd0 = da[1] * u1 * v0 + da[2] * u0 * v1, wd1 = da[0] * u0 * v0;
            R wp0 = pa[1] * u1 * v0 + pa[2] * u0 * v1, wp1 = pa[0] * u0 * v0;
            for (int a = 0; a < P; a++) {
                int ga = a0 + a; if (ga >= K.x) ga -= K.x;
                int g = gidx(ga, gb, gc, K);
                atomicAdd(grid + g, t1[a] * wd0 + t1[P + a] * wd1);
                atomicAdd(grid + gstride + g, t1[a] * wp0 + t1[P + a] * wp1);
            }
        }
    }
}

// Point-parallel spreading of two dipole sets: one block of 128 threads per
// site, thread t < P^3 owns stencil point (a,b,c) = (t / P^2, t / P % P, t % P)
// and issues one fire-and-forget atomic add per grid; consecutive threads
// write consecutive z addresses.
template <class R, int P>
__global__ void __launch_bounds__(128) k_spread_dipoles_pt(int n, const double* __restrict__ ud,
                                                           const double* __restrict__ up,
                                                           const R* __restrict__ theta, const int* __restrict__ k0,
                                                           int3 K, R sc0, R sc1, R sc2, R* __restrict__ grid,
                                                           size_t gstride) {
    const int i = blockIdx.x, t = threadIdx.x;
    if (t >= P * P * P) return;
    const int a = t / (P * P), b = (t / P) % P, c = t % P;
    const R* th = theta + (size_t)i * 3 * 4 * P;
    R t0 = th[a], t1 = th[P + a];
    R u0 = th[4 * P + b], u1 = th[5 * P + b];
    R v0 = th[8 * P + c], v1 = th[9 * P + c];
    R d0 = (R)ud[3 * i] * sc0, d1 = (R)ud[3 * i + 1] * sc1, d2 = (R)ud[3 * i + 2] * sc2;
    R p0 = (R)up[3 * i] * sc0, p1 = (R)up[3 * i + 1] * sc1, p2 = (R)up[3 * i + 2] * sc2;
    R w100 = t1 * u0 * v0, w010 = t0 * u1 * v0, w001 = t0 * u0 * v1;
    int ga = k0[3 * i] + a; if (ga >= K.x) ga -= K.x;
    int gb = k0[3 * i + 1] + b; if (gb >= K.y) gb -= K.y;
    int gc = k0[3 * i + 2] + c; if (gc >= K.z) gc -= K.z;
    const int g = gidx(ga, gb, gc, K);
    atomicAdd(grid + g, d0 * w100 + d1 * w010 + d2 * w001);
    atomicAdd(grid + gstride + g, p0 * w100 + p1 * w010 + p2 * w001);
}

// Point-parallel gather of the field of two dipole grids (first derivatives
// only) fused with the matvec assembly:
//   A v = v/alpha - (F_real + F_recip + selfc v),  F_recip = -grad phi
// One block per site; the P^3 stencil points are reduced with shuffles and
// shared memory.
template <class R, int P>
__global__ void __launch_bounds__(128) k_gather_field_pt(int n, const R* __restrict__ phigrid, size_t gstride,
                                                         const R* __restrict__ theta, const int* __restrict__ k0,
                                                         int3 K, double sc0, double sc1, double sc2,
                                                         const double* __restrict__ vd,
                                                         const double* __restrict__ vp,
                                                         const double* __restrict__ Fd,
                                                         const double* __restrict__ Fp, double selfc,
                                                         const double* __restrict__ pol, double* __restrict__ Ad,
                                                         double* __restrict__ Ap) {
    const int i = blockIdx.x, t = threadIdx.x;
    R f[6] = {0, 0, 0, 0, 0, 0};
    if (t < P * P * P) {
        const int a = t / (P * P), b = (t / P) % P, c = t % P;
        const R* th = theta + (size_t)i * 3 * 4 * P;
        R t0 = th[a], t1 = th[P + a];
        R u0 = th[4 * P + b], u1 = th[5 * P + b];
        R v0 = th[8 * P + c], v1 = th[9 * P + c];
        int ga = k0[3 * i] + a; if (ga >= K.x) ga -= K.x;
        int gb = k0[3 * i + 1] + b; if (gb >= K.y) gb -= K.y;
        int gc = k0[3 * i + 2] + c; if (gc >= K.z) gc -= K.z;
        const int g = gidx(ga, gb, gc, K);
        R qd = phigrid[g], qp = phigrid[gstride + g];
        R w100 = t1 * u0 * v0, w010 = t0 * u1 * v0, w001 = t0 * u0 * v1;
        f[0] = w100 * qd; f[1] = w010 * qd; f[2] = w001 * qd;
        f[3] = w100 * qp; f[4] = w010 * qp; f[5] = w001 * qp;
    }
    __shared__ R part[4][6];
#pragma unroll
    for (int k = 0; k < 6; k++) f[k] = warp_sum(f[k]);
    if ((t & 31) == 0)
        for (int k = 0; k < 6; k++) part[t >> 5][k] = f[k];
    __syncthreads();
    if (t < 6) {
        double v = (double)part[0][t] + (double)part[1][t] + (double)part[2][t] + (double)part[3][t];
        double scv = t % 3 == 0 ? sc0 : t % 3 == 1 ? sc1 : sc2;
        const int c = t % 3;
        const bool dset = t < 3;
        const double* vv = dset ? vd : vp;
        const double* FF = dset ? Fd : Fp;
        double* AA = dset ? Ad : Ap;
        double alpha = pol[i];
        double field = FF[3 * i + c] - v * scv + selfc * vv[3 * i + c];
        AA[3 * i + c] = alpha > 0 ? vv[3 * i + c] / alpha - field : 0.0;
    }
}

// Multiply the transformed grids by the influence function
//   G(m) = exp(-pi^2 |h|^2 / alpha^2) / (pi V |h|^2 bsmod1 bsmod2 bsmod3)
// precomputed in FP64 on the host (half-complex layout, G(0) = 0).
// The same kernel clears the real spreading grids ([batch][nreal], already
// consumed by the forward FFT) for the next spreading pass.
template <class R>
__global__ void k_convolve(size_t ncomplex, int batch, const R* __restrict__ infl,
                           typename Cplx<R>::type* __restrict__ cg, R* __restrict__ spread, size_t nreal) {
    size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < ncomplex) {
        R g = infl[t];
        for (int b = 0; b < batch; b++) {
            auto v = cg[b * ncomplex + t];
            v.x *= g;
            v.y *= g;
            cg[b * ncomplex + t] = v;
        }
    }
    if (spread)
        for (size_t q = t; q < (size_t)batch * nreal; q += (size_t)gridDim.x * blockDim.x) spread[q] = R(0);
}

// Gather NC (4, 10 or 20) Cartesian potential derivatives per site from
// a convolved grid: phi_tuv = (K1/L1)^t (K2/L2)^u (K3/L3)^v sum_g theta...
// Output order: 0; x y z; xx yy zz xy xz yz; xxx yyy zzz xxy xxz xyy yyz xzz yzz xyz
template <class R, int P, int NC>
__global__ void k_gather(int n, const R* __restrict__ grid, const R* __restrict__ theta, const int* __restrict__ k0,
                         int3 K, double sc0, double sc1, double sc2, double* __restrict__ phi) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const R* t1 = theta + ((size_t)i * 3 + 0) * 4 * P;
    const R* t2 = theta + ((size_t)i * 3 + 1) * 4 * P;
    const R* t3 = theta + ((size_t)i * 3 + 2) * 4 * P;
    int a0 = k0[3 * i], b0 = k0[3 * i + 1], c0 = k0[3 * i + 2];
    R f[20];
#pragma unroll
    for (int j = 0; j < 20; j++) f[j] = 0;
    for (int c = 0; c < P; c++) {
        R v0 = t3[c], v1 = t3[P + c], v2 = t3[2 * P + c], v3 = t3[3 * P + c];
        int gc = c0 + c; if (gc >= K.z) gc -= K.z;
        for (int b = 0; b < P; b++) {
            R u0 = t2[b], u1 = t2[P + b], u2 = t2[2 * P + b], u3 = t2[3 * P + b];
            int gb = b0 + b; if (gb >= K.y) gb -= K.y;
            // x-sums: s_k = sum_a t1^(k)[a] grid
            R s0 = 0, s1 = 0, s2 = 0, s3 = 0;
            for (int a = 0; a < P; a++) {
                int ga = a0 + a; if (ga >= K.x) ga -= K.x;
                R g = grid[gidx(ga, gb, gc, K)];
                s0 += t1[a] * g;
                s1 += t1[P + a] * g;
                if (NC >= 10) s2 += t1[2 * P + a] * g;
                if (NC >= 20) s3 += t1[3 * P + a] * g;
            }
            f[0] += s0 * u0 * v0;
            f[1] += s1 * u0 * v0;
            f[2] += s0 * u1 * v0;
            f[3] += s0 * u0 * v1;
            if (NC >= 10) {
                f[4] += s2 * u0 * v0;
                f[5] += s0 * u2 * v0;
                f[6] += s0 * u0 * v2;
                f[7] += s1 * u1 * v0;
                f[8] += s1 * u0 * v1;
                f[9] += s0 * u1 * v1;
            }
            if (NC >= 20) {
                f[10] += s3 * u0 * v0;
                f[11] += s0 * u3 * v0;
                f[12] += s0 * u0 * v3;
                f[13] += s2 * u1 * v0;
                f[14] += s2 * u0 * v1;
                f[15] += s1 * u2 * v0;
                f[16] += s0 * u2 * v1;
                f[17] += s1 * u0 * v2;
                f[18] += s0 * u1 * v2;
                f[19] += s1 * u1 * v1;
            }
        }
    }
    const int ex[20][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {2, 0, 0}, {0, 2, 0}, {0, 0, 2},
                           {1, 1, 0}, {1, 0, 1}, {0, 1, 1}, {3, 0, 0}, {0, 3, 0}, {0, 0, 3}, {2, 1, 0},
                           {2, 0, 1}, {1, 2, 0}, {0, 2, 1}, {1, 0, 2}, {0, 1, 2}, {1, 1, 1}};
    double p0[4] = {1, sc0, sc0 * sc0, sc0 * sc0 * sc0};
    double p1[4] = {1, sc1, sc1 * sc1, sc1 * sc1 * sc1};
    double p2[4] = {1, sc2, sc2 * sc2, sc2 * sc2 * sc2};
#pragma unroll
    for (int j = 0; j < NC; j++) phi[(size_t)NC * i + j] = (double)f[j] * p0[ex[j][0]] * p1[ex[j][1]] * p2[ex[j][2]];
}

}  // namespace amg
