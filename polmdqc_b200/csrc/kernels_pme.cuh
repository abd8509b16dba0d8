// kernels_pme.cuh -- smooth PME for multipoles and induced dipoles
// (Essmann et al. 1995; multipoles as Sagui, Pedersen & Darden 2004):
// fractional multipoles spread with order-P B-splines and gathers of up to
// 20 potential derivatives per site.  The permanent multipoles use one real
// grid (library R2C/C2R transform and k_convolve).  The two induced-dipole
// sets are spread into one complex grid g = Q_d + i Q_p: the influence
// function G is real and even (G(m) = G(-m)), so
//   IFFT(G . FFT(Q_d + i Q_p)) = (G * Q_d) + i (G * Q_p)
// and one in-place complex transform pair (library C2C, unnormalised both
// ways as in smooth PME) convolves both sets.
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

// fractional dipole d'_j = sum_i d_i m[i][j]
template <class R>
__device__ __forceinline__ void frac_dipole(const Frac& F, double x, double y, double z, R& a, R& b, R& c) {
    if (!F.general) {
        a = (R)x * (R)F.m[0][0];
        b = (R)y * (R)F.m[1][1];
        c = (R)z * (R)F.m[2][2];
        return;
    }
    a = (R)(x * F.m[0][0] + y * F.m[1][0] + z * F.m[2][0]);
    b = (R)(x * F.m[0][1] + y * F.m[1][1] + z * F.m[2][1]);
    c = (R)(x * F.m[0][2] + y * F.m[1][2] + z * F.m[2][2]);
}

// Exponents (x, y, z) of the 20 potential derivatives in output order:
// 0; x y z; xx yy zz xy xz yz; xxx yyy zzz xxy xxz xyy yyz xzz yzz xyz
__constant__ int kDerEx[20][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {2, 0, 0}, {0, 2, 0}, {0, 0, 2},
                                  {1, 1, 0}, {1, 0, 1}, {0, 1, 1}, {3, 0, 0}, {0, 3, 0}, {0, 0, 3}, {2, 1, 0},
                                  {2, 0, 1}, {1, 2, 0}, {0, 2, 1}, {1, 0, 2}, {0, 1, 2}, {1, 1, 1}};

// Cartesian derivative j of the potential from the grid-unit derivatives f[]
// (same ordering) in a general cell: the grid-unit tensor contracted with m
// on every index.  Called only for non-orthogonal cells.
__device__ __noinline__ double cart_deriv(const Frac F, const double* f, int nc, int j) {
    int ax[3], n = 0;
    for (int a = 0; a < 3; a++)
        for (int r = 0; r < kDerEx[j][a]; r++) ax[n++] = a;
    if (n == 0) return f[0];
    const int tuples = n == 1 ? 3 : n == 2 ? 9 : 27;
    double v = 0;
    for (int t = 0; t < tuples; t++) {
        int cnt[3] = {0, 0, 0};
        double w = 1;
        int r = t;
        for (int k = 0; k < n; k++) {
            const int q = r % 3;
            r /= 3;
            cnt[q]++;
            w *= F.m[ax[k]][q];
        }
        for (int q = 0; q < nc; q++)
            if (kDerEx[q][0] == cnt[0] && kDerEx[q][1] == cnt[1] && kDerEx[q][2] == cnt[2]) v += w * f[q];
    }
    return v;
}

// Spread the permanent multipoles (global frame, FP64 rp10) as fractional
// multipoles: grid(g) += q t0u0v0 + sum_a d'_a (first derivative in a) +
// sum_ab Q'_ab (second derivatives), with d' = m^T d, Q' = m^T Q m.
template <class R, int P>
__global__ void k_spread_mpole(int n, const double* __restrict__ rp10, const R* __restrict__ theta,
                               const int* __restrict__ k0, int3 K, Frac F, R* __restrict__ grid) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double* m = rp10 + 10 * i;
    R q = (R)m[0];
    R d1, d2, d3, q11, q22, q33, q12, q13, q23;
    frac_dipole<R>(F, m[1], m[2], m[3], d1, d2, d3);
    if (!F.general) {
        const R sc0 = (R)F.m[0][0], sc1 = (R)F.m[1][1], sc2 = (R)F.m[2][2];
        q11 = (R)m[4] * sc0 * sc0; q22 = (R)m[7] * sc1 * sc1; q33 = (R)m[9] * sc2 * sc2;
        q12 = 2 * (R)m[5] * sc0 * sc1; q13 = 2 * (R)m[6] * sc0 * sc2; q23 = 2 * (R)m[8] * sc1 * sc2;
    } else {
        const double Qc[3][3] = {{m[4], m[5], m[6]}, {m[5], m[7], m[8]}, {m[6], m[8], m[9]}};
        double Qf[3][3];
        for (int j = 0; j < 3; j++)
            for (int k = 0; k < 3; k++) {
                double v = 0;
                for (int a = 0; a < 3; a++)
                    for (int b = 0; b < 3; b++) v += F.m[a][j] * Qc[a][b] * F.m[b][k];
                Qf[j][k] = v;
            }
        q11 = (R)Qf[0][0]; q22 = (R)Qf[1][1]; q33 = (R)Qf[2][2];
        q12 = (R)(2 * Qf[0][1]); q13 = (R)(2 * Qf[0][2]); q23 = (R)(2 * Qf[1][2]);
    }
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

// Line-parallel spreading of two dipole sets (FP64 [3n] each) into the
// complex grid zg = Q_d + i Q_p.  A block of 128 threads takes
// kLineSites = 5 sites (sites in the order `order`); thread t < 5 P^2 owns the
// z-line (a, b) = (l / P, l % P), l = t % P^2, of site t / P^2: the P grid
// points (a, b, c0 .. c0 + P - 1) that are consecutive in memory.  In FP32
// with an even K3 the line is added as aligned pairs of complex points (one
// 16-byte vector atomic each: 3 atomics for P = 5 instead of 5); otherwise
// point by point.  zg must start at zero.
constexpr int kLineSites = 5;

template <class R>
__device__ __forceinline__ void add_cplx(typename Cplx<R>::type* p, R x, R y);
template <>
__device__ __forceinline__ void add_cplx<float>(float2* p, float x, float y) {
    atomicAdd(p, make_float2(x, y));
}
template <>
__device__ __forceinline__ void add_cplx<double>(double2* p, double x, double y) {
    atomicAdd(&p->x, x);
    atomicAdd(&p->y, y);
}

// add the P values (vx + i vy) of one z-line starting at c0 (wrapping at K3)
template <class R, int P>
__device__ __forceinline__ void add_line(typename Cplx<R>::type* line, int c0, int K3, const R (&vx)[P],
                                         const R (&vy)[P]) {
    if constexpr (sizeof(R) == 4) {
        if ((K3 & 1) == 0) {
            // with K3 even a pair starting at an even index never straddles
            // the wrap, and the line start (a multiple of K3 points of 8 B)
            // keeps even indices 16-byte aligned
            auto pair = [&](int cc) {  // points cc, cc + 1 (cc a compile-time index after unrolling)
                int gc = c0 + cc;
                if (gc >= K3) gc -= K3;
                atomicAdd(reinterpret_cast<float4*>(line + gc), make_float4(vx[cc], vy[cc], vx[cc + 1], vy[cc + 1]));
            };
            if (c0 & 1) {  // odd start: a single point, then pairs
                add_cplx<R>(line + c0, vx[0], vy[0]);
#pragma unroll
                for (int q = 0; q < (P - 1) / 2; q++) pair(1 + 2 * q);
            } else {       // even start: pairs, then a single point
#pragma unroll
                for (int q = 0; q < (P - 1) / 2; q++) pair(2 * q);
                int gc = c0 + P - 1;
                if (gc >= K3) gc -= K3;
                add_cplx<R>(line + gc, vx[P - 1], vy[P - 1]);
            }
            return;
        }
    }
#pragma unroll
    for (int c = 0; c < P; c++) {
        int gc = c0 + c;
        if (gc >= K3) gc -= K3;
        add_cplx<R>(line + gc, vx[c], vy[c]);
    }
}

// spread stencil point t = (a, b, c) = (t / P^2, t / P % P, t % P) of site i
// (FP64, where one point per thread measured faster than whole lines: without
// vector atomics a line is P dependent pairs of atomics in one thread)
template <class R, int P>
__device__ __forceinline__ void spread_site_point(int i, int t, const double* pd, const double* pq,
                                                  const R* __restrict__ theta, const int* __restrict__ k0, int3 K,
                                                  const Frac& F, typename Cplx<R>::type* __restrict__ zg) {
    const int a = t / (P * P), b = (t / P) % P, c = t % P;
    const R* th = theta + (size_t)i * 3 * 4 * P;
    const R t0 = th[a], t1 = th[P + a];
    const R u0 = th[4 * P + b], u1 = th[5 * P + b];
    const R v0 = th[8 * P + c], v1 = th[9 * P + c];
    R d0, d1, d2, p0, p1, p2;
    frac_dipole<R>(F, pd[0], pd[1], pd[2], d0, d1, d2);
    frac_dipole<R>(F, pq[0], pq[1], pq[2], p0, p1, p2);
    const R w100 = t1 * u0 * v0, w010 = t0 * u1 * v0, w001 = t0 * u0 * v1;
    int ga = k0[3 * i] + a; if (ga >= K.x) ga -= K.x;
    int gb = k0[3 * i + 1] + b; if (gb >= K.y) gb -= K.y;
    int gc = k0[3 * i + 2] + c; if (gc >= K.z) gc -= K.z;
    add_cplx<R>(zg + gidx(ga, gb, gc, K), d0 * w100 + d1 * w010 + d2 * w001, p0 * w100 + p1 * w010 + p2 * w001);
}

// spread the line (a, b) of site i with Cartesian dipoles pd (d set) and pq
// (p set), converted to fractional dipoles here
template <class R, int P>
__device__ __forceinline__ void spread_site_line(int i, int l, const double* pd, const double* pq,
                                                 const R* __restrict__ theta, const int* __restrict__ k0, int3 K,
                                                 const Frac& F, typename Cplx<R>::type* __restrict__ zg) {
    static_assert(P % 2 == 1, "the pairing of line points assumes an odd order");
    const int a = l / P, b = l % P;
    const R* th = theta + (size_t)i * 3 * 4 * P;
    const R t0 = th[a], t1 = th[P + a];
    const R u0 = th[4 * P + b], u1 = th[5 * P + b];
    R d0, d1, d2, p0, p1, p2;
    frac_dipole<R>(F, pd[0], pd[1], pd[2], d0, d1, d2);
    frac_dipole<R>(F, pq[0], pq[1], pq[2], p0, p1, p2);
    // value at z weight (v0, v1): (d0 t1 u0 + d1 t0 u1) v0 + d2 t0 u0 v1
    const R ad = d0 * t1 * u0 + d1 * t0 * u1, bd = d2 * t0 * u0;
    const R ap = p0 * t1 * u0 + p1 * t0 * u1, bp = p2 * t0 * u0;
    R vx[P], vy[P];
#pragma unroll
    for (int c = 0; c < P; c++) {
        const R v0 = th[8 * P + c], v1 = th[9 * P + c];
        vx[c] = ad * v0 + bd * v1;
        vy[c] = ap * v0 + bp * v1;
    }
    int ga = k0[3 * i] + a; if (ga >= K.x) ga -= K.x;
    int gb = k0[3 * i + 1] + b; if (gb >= K.y) gb -= K.y;
    add_line<R, P>(zg + ((size_t)ga * K.y + gb) * K.z, k0[3 * i + 2], K.z, vx, vy);
}

template <class R, int P>
__global__ void __launch_bounds__(128) k_spread_dipoles(int n, const int* __restrict__ order,
                                                        const double* __restrict__ ud,
                                                        const double* __restrict__ up,
                                                        const R* __restrict__ theta, const int* __restrict__ k0,
                                                        int3 K, Frac F,
                                                        typename Cplx<R>::type* __restrict__ zg) {
    static_assert(kLineSites * P * P <= 128, "lines of a block");
    const int t = threadIdx.x;
    if constexpr (sizeof(R) == 8) {  // FP64: one site per block, one stencil point per thread
        if (t >= P * P * P) return;
        const int i = order[blockIdx.x];
        spread_site_point<R, P>(i, t, ud + 3 * i, up + 3 * i, theta, k0, K, F, zg);
    } else {
        const int g = blockIdx.x * kLineSites + t / (P * P);
        if (t >= kLineSites * P * P || g >= n) return;
        const int i = order[g];
        spread_site_line<R, P>(i, t % (P * P), ud + 3 * i, up + 3 * i, theta, k0, K, F, zg);
    }
}

// blocks of k_spread_dipoles / k_pcg_dir_spread for n sites
template <class R>
inline unsigned spread_blocks(int n) {
    return sizeof(R) == 8 ? (unsigned)n : (unsigned)((n + kLineSites - 1) / kLineSites);
}

// The P grid values z = c0 .. c0+P-1 (periodic in Kz) of one z-line of the
// complex dipole grid.  With the line's z-range inside the grid and Kz even,
// from three aligned loads of two values each (16 bytes in FP32, 32 in FP64)
// and a select by the parity of c0, instead of one load per value: 6 values
// cover any 5 consecutive ones; else value by value.  (Two 256-bit FP32
// loads of 8 values were slower: 64 bytes through L1 for 40 used.)  The grid
// is read-only in the gathers.
template <int P>
__device__ __forceinline__ void load_line(const float2* __restrict__ line, int c0, int Kz, float2 (&q)[P]) {
    static_assert(P <= 5, "a line of at most 5 values fits 6 loaded ones");
    const int zb = c0 & ~1, o = c0 & 1;
    if ((Kz & 1) == 0 && zb + 6 <= Kz) {
        float4 w[3];
#pragma unroll
        for (int h = 0; h < 3; h++) w[h] = __ldg(reinterpret_cast<const float4*>(line + zb) + h);
        const float2 v[6] = {make_float2(w[0].x, w[0].y), make_float2(w[0].z, w[0].w), make_float2(w[1].x, w[1].y),
                             make_float2(w[1].z, w[1].w), make_float2(w[2].x, w[2].y), make_float2(w[2].z, w[2].w)};
#pragma unroll
        for (int c = 0; c < P; c++) q[c] = o ? v[c + 1] : v[c];
        return;
    }
#pragma unroll
    for (int c = 0; c < P; c++) {
        int gc = c0 + c;
        if (gc >= Kz) gc -= Kz;
        q[c] = line[gc];
    }
}
template <int P>
__device__ __forceinline__ void load_line(const double2* __restrict__ line, int c0, int Kz, double2 (&q)[P]) {
    static_assert(P <= 5, "a line of at most 5 values fits 6 loaded ones");
    const int zb = c0 & ~1, o = c0 & 1;
    if ((Kz & 1) == 0 && zb + 6 <= Kz) {
        double w[12];
#pragma unroll
        for (int h = 0; h < 3; h++)
            asm("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];"
                : "=d"(w[4 * h]), "=d"(w[4 * h + 1]), "=d"(w[4 * h + 2]), "=d"(w[4 * h + 3])
                : "l"(line + zb + 2 * h));
#pragma unroll
        for (int c = 0; c < P; c++) {
            q[c].x = o ? w[2 * c + 2] : w[2 * c];
            q[c].y = o ? w[2 * c + 3] : w[2 * c + 1];
        }
        return;
    }
#pragma unroll
    for (int c = 0; c < P; c++) {
        int gc = c0 + c;
        if (gc >= Kz) gc -= Kz;
        q[c] = line[gc];
    }
}

// Gather of the field of two dipole potential grids (interleaved as the
// real and imaginary parts of zg; first derivatives only) fused with the
// matvec assembly:
//   A v = v/alpha - (F_real + F_recip + selfc v),  F_recip = -grad phi
// and, when vAv is given, the PCG dot products v.Av of both sets added to
// vAv[0], vAv[1].  G consecutive lanes per site; each lane takes whole
// z-lines (a, b) of the P^3 stencil (P grid values per line), the per-lane
// sums are combined with shuffles and lanes 0..5 write the six components.
// Blocks stride over the sites, so each block adds its dot products once.
// With Fd, Fp null the real-space field is left out (A v without -F_real,
// and its dot products): the real-space kernel then runs beside this one and
// adds its own share (k_tu_stored with vAv), and k_pcg_update subtracts F.
template <class R, int P, int G>
__global__ void __launch_bounds__(128) k_gather_field(int n, const typename Cplx<R>::type* __restrict__ zg,
                                                      const R* __restrict__ theta, const int* __restrict__ k0,
                                                      int3 K, Frac F,
                                                      const double* __restrict__ vd, const double* __restrict__ vp,
                                                      const double* __restrict__ Fd, const double* __restrict__ Fp,
                                                      double selfc, const double* __restrict__ pol,
                                                      double* __restrict__ Ad, double* __restrict__ Ap,
                                                      double* __restrict__ vAv) {
    const int lane = threadIdx.x % G, per_block = blockDim.x / G;
    double dotd = 0, dotp = 0;  // v.Av of this thread's components
    for (int g0 = blockIdx.x * per_block; g0 < n; g0 += gridDim.x * per_block) {
        const int g = g0 + threadIdx.x / G;
        const int i = min(g, n - 1);
        const R* th = theta + (size_t)i * 3 * 4 * P;
        const int a0 = k0[3 * i], b0 = k0[3 * i + 1], c0 = k0[3 * i + 2];
        R v0[P], v1[P];
#pragma unroll
        for (int c = 0; c < P; c++) {
            v0[c] = th[8 * P + c];
            v1[c] = th[9 * P + c];
        }
        R f[6] = {0, 0, 0, 0, 0, 0};
        for (int l = lane; l < P * P; l += G) {
            const int a = l / P, b = l - (l / P) * P;
            int ga = a0 + a; if (ga >= K.x) ga -= K.x;
            int gb = b0 + b; if (gb >= K.y) gb -= K.y;
            const typename Cplx<R>::type* line = zg + ((size_t)ga * K.y + gb) * K.z;
            typename Cplx<R>::type qv[P];
            load_line<P>(line, c0, K.z, qv);
            R sd0 = 0, sd1 = 0, sp0 = 0, sp1 = 0;
#pragma unroll
            for (int c = 0; c < P; c++) {
                const R qd = qv[c].x, qp = qv[c].y;
                sd0 += v0[c] * qd; sd1 += v1[c] * qd;
                sp0 += v0[c] * qp; sp1 += v1[c] * qp;
            }
            const R t0 = th[a], t1 = th[P + a], u0 = th[4 * P + b], u1 = th[5 * P + b];
            const R w100 = t1 * u0, w010 = t0 * u1, w001 = t0 * u0;
            f[0] += w100 * sd0; f[1] += w010 * sd0; f[2] += w001 * sd1;
            f[3] += w100 * sp0; f[4] += w010 * sp0; f[5] += w001 * sp1;
        }
        double sum[6];
#pragma unroll
        for (int k = 0; k < 6; k++) sum[k] = group_sum<G>((double)f[k]);
        if (g < n && lane < 6) {
            const int t = lane, c = t % 3;
            const bool dset = t < 3;
            // d phi / dx_c from the grid-unit first derivatives of this set
            const double s0 = dset ? sum[0] : sum[3], s1 = dset ? sum[1] : sum[4], s2 = dset ? sum[2] : sum[5];
            const double dphi = F.general ? F.m[c][0] * s0 + F.m[c][1] * s1 + F.m[c][2] * s2
                                          : F.m[c][c] * (c == 0 ? s0 : c == 1 ? s1 : s2);
            const double* vv = dset ? vd : vp;
            const double* FF = dset ? Fd : Fp;
            double* AA = dset ? Ad : Ap;
            const double alpha = pol[i];
            const double field = (FF ? FF[3 * i + c] : 0.0) - dphi + selfc * vv[3 * i + c];
            const double av = alpha > 0 ? vv[3 * i + c] / alpha - field : 0.0;
            AA[3 * i + c] = av;
            if (dset) dotd += vv[3 * i + c] * av;
            else dotp += vv[3 * i + c] * av;
        }
    }
    if (vAv) {
        block_sum_add(dotd, vAv);
        block_sum_add(dotp, vAv + 1);
    }
}

// out = G . g on the transformed complex dipole grid (G real, on the full
// grid), and g cleared for the next spreading
template <class R>
__global__ void k_scale_grid(size_t npts, const R* __restrict__ G, typename Cplx<R>::type* __restrict__ g,
                             typename Cplx<R>::type* __restrict__ out) {
    size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= npts) return;
    auto v = g[t];
    const R w = G[t];
    v.x *= w;
    v.y *= w;
    out[t] = v;
    v.x = v.y = R(0);
    g[t] = v;
}

// Reciprocal virial through the influence function.  A strain eps moves the
// reciprocal vectors h -> (1 - eps^T) h and the volume V -> V (1 + tr eps) at
// fixed fractional coordinates, so for an energy term e(m) = g(m) X(m)
// (X a product of structure factors)
//   de/deps_ab = e (2 (1/h^2 + pi^2/alpha^2) h_a h_b - delta_ab)
// (the reciprocal virial of Essmann et al., J. Chem. Phys. 103, 8577 (1995),
// in dE/d(strain) form).  `c2` = pi^2/alpha^2; h = sum_j m_j b_j with the
// reciprocal vectors b_j = (column j of F.m) / K_j.
__device__ __forceinline__ void kvir_point(double (&v)[6], int ma, int mb, int mc, const Frac& F, int3 K, double c2,
                                           double e) {
    const double fa = (double)ma / K.x, fb = (double)mb / K.y, fc = (double)mc / K.z;
    const double hx = F.m[0][0] * fa + F.m[0][1] * fb + F.m[0][2] * fc;
    const double hy = F.m[1][0] * fa + F.m[1][1] * fb + F.m[1][2] * fc;
    const double hz = F.m[2][0] * fa + F.m[2][1] * fb + F.m[2][2] * fc;
    const double h2 = hx * hx + hy * hy + hz * hz;
    const double t = 2.0 * (1.0 / h2 + c2) * e;
    v[0] += t * hx * hx - e;
    v[1] += t * hy * hy - e;
    v[2] += t * hz * hz - e;
    v[3] += t * hx * hy;
    v[4] += t * hx * hz;
    v[5] += t * hy * hz;
}

// Permanent multipoles: e(m) = f/2 g(m) |S(m)|^2 over the half-complex
// transform cg (before the convolution); points 0 < c < K3/2 stand for m and
// -m.  Saves the transform into `save` for the polarization cross terms.
template <class R>
__global__ void k_kvir_mpole(size_t ncomplex, int3 K, Frac F, double c2, double f, const R* __restrict__ infl,
                             const typename Cplx<R>::type* __restrict__ cg, typename Cplx<R>::type* __restrict__ save,
                             double* __restrict__ vir) {
    const int K3h = K.z / 2 + 1;
    double v[6] = {0, 0, 0, 0, 0, 0};
    for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < ncomplex; t += (size_t)gridDim.x * blockDim.x) {
        const auto S = cg[t];
        if (save) save[t] = S;
        if (t == 0) continue;
        const int c = (int)(t % K3h);
        const int b = (int)((t / K3h) % K.y);
        const int a = (int)(t / ((size_t)K3h * K.y));
        const int ma = a <= K.x / 2 ? a : a - K.x, mb = b <= K.y / 2 ? b : b - K.y;
        const double wgt = (c == 0 || 2 * c == K.z) ? 1.0 : 2.0;
        const double e = 0.5 * f * wgt * (double)infl[t] * ((double)S.x * S.x + (double)S.y * S.y);
        kvir_point(v, ma, mb, c, F, K, c2, e);
    }
    block_vir_add(v, vir);
}

// Polarization, G = 1/2 [U(up, M) + U(ud, M) + mutual U(up, ud)] with
//   U(X, Y) = sum_m g(m) Re[S_X(m) conj S_Y(m)],
// over the full grid: z is the transform of the dipole grid Q_d + i Q_p (so
// S_d(m) = (z(m) + conj z(-m))/2, S_p(m) = (z(m) - conj z(-m))/(2i)), sM the
// saved half-complex transform of the permanent grid, G the influence
// function on the full grid.  mterms 0: the U(up, ud) term alone (OPT cross
// terms).
template <class R>
__global__ void k_kvir_polar(size_t npts, int3 K, Frac F, double c2, double f, int mutual, int mterms,
                             const R* __restrict__ G, const typename Cplx<R>::type* __restrict__ z,
                             const typename Cplx<R>::type* __restrict__ sM, double* __restrict__ vir) {
    const int K3h = K.z / 2 + 1;
    double v[6] = {0, 0, 0, 0, 0, 0};
    for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < npts; t += (size_t)gridDim.x * blockDim.x) {
        if (t == 0) continue;
        const int c = (int)(t % K.z);
        const int b = (int)((t / K.z) % K.y);
        const int a = (int)(t / ((size_t)K.z * K.y));
        const int an = a ? K.x - a : 0, bn = b ? K.y - b : 0, cn = c ? K.z - c : 0;
        const auto zp = z[t];
        const auto zn = z[((size_t)an * K.y + bn) * K.z + cn];
        const double dx = 0.5 * ((double)zp.x + zn.x), dy = 0.5 * ((double)zp.y - zn.y);
        const double px = 0.5 * ((double)zp.y + zn.y), py = -0.5 * ((double)zp.x - zn.x);
        double mx, my;
        if (c < K3h) {
            const auto m = sM[((size_t)a * K.y + b) * K3h + c];
            mx = m.x;
            my = m.y;
        } else {  // S_M(m) = conj S_M(-m), held at (an, bn, K3 - c)
            const auto m = sM[((size_t)an * K.y + bn) * K3h + cn];
            mx = m.x;
            my = -(double)m.y;
        }
        double x = mterms ? mx * (px + dx) + my * (py + dy) : 0.0;
        if (mutual) x += px * dx + py * dy;
        // frequency of the point, or past the half-complex range that of its
        // partner (-a, -b, K3 - c): G is the even extension of the
        // half-complex influence function, so its strain derivative follows
        // the partner's reciprocal vector (different on the Nyquist planes)
        const int ea = c < K3h ? a : an, eb = c < K3h ? b : bn, ec = c < K3h ? c : cn;
        const int ma = ea <= K.x / 2 ? ea : ea - K.x, mb = eb <= K.y / 2 ? eb : eb - K.y;
        kvir_point(v, ma, mb, ec, F, K, c2, 0.5 * f * (double)G[t] * x);
    }
    block_vir_add(v, vir);
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

// Gather NC (4, 10 or 20) Cartesian potential derivatives per site:
//   phi_tuv = (K1/L1)^t (K2/L2)^u (K3/L3)^v sum_abc theta1^(t)_a theta2^(u)_b theta3^(v)_c grid
// from a real grid (NS = 1: grid[g]) or from both parts of the complex
// dipole grid at once (NS = 2: zg[g].x into phi, zg[g].y into phi + NC n).
// G consecutive lanes per site; each lane takes whole z-lines (a, b) of the
// P^3 stencil, contracts the line's P values with the z weights of orders
// 0..3 and adds them with the x and y weights; the lanes' sums are combined
// with shuffles.  Output order: 0; x y z; xx yy zz xy xz yz;
// xxx yyy zzz xxy xxz xyy yyz xzz yzz xyz.
template <class R, int NC>
__device__ __forceinline__ void add_derivs(R (&f)[NC], const R (&x)[4], const R (&y)[4], const R (&z)[4]) {
    f[0] += x[0] * y[0] * z[0];
    f[1] += x[1] * y[0] * z[0];
    f[2] += x[0] * y[1] * z[0];
    f[3] += x[0] * y[0] * z[1];
    if constexpr (NC >= 10) {
        f[4] += x[2] * y[0] * z[0];
        f[5] += x[0] * y[2] * z[0];
        f[6] += x[0] * y[0] * z[2];
        f[7] += x[1] * y[1] * z[0];
        f[8] += x[1] * y[0] * z[1];
        f[9] += x[0] * y[1] * z[1];
    }
    if constexpr (NC >= 20) {
        f[10] += x[3] * y[0] * z[0];
        f[11] += x[0] * y[3] * z[0];
        f[12] += x[0] * y[0] * z[3];
        f[13] += x[2] * y[1] * z[0];
        f[14] += x[2] * y[0] * z[1];
        f[15] += x[1] * y[2] * z[0];
        f[16] += x[0] * y[2] * z[1];
        f[17] += x[1] * y[0] * z[2];
        f[18] += x[0] * y[1] * z[2];
        f[19] += x[1] * y[1] * z[1];
    }
}

template <class R, int P, int NC, int G, int NS>
__global__ void __launch_bounds__(128) k_gather(int n, const void* __restrict__ gridv, const R* __restrict__ theta,
                                                const int* __restrict__ k0, int3 K, Frac F,
                                                double* __restrict__ phi) {
    constexpr int ND = NC == 4 ? 2 : NC == 10 ? 3 : 4;  // derivative orders per axis
    using C = typename Cplx<R>::type;
    const int g = (blockIdx.x * blockDim.x + threadIdx.x) / G, lane = threadIdx.x % G;
    const int i = min(g, n - 1);
    const R* t1 = theta + ((size_t)i * 3 + 0) * 4 * P;
    const R* t2 = theta + ((size_t)i * 3 + 1) * 4 * P;
    const R* t3 = theta + ((size_t)i * 3 + 2) * 4 * P;
    const int a0 = k0[3 * i], b0 = k0[3 * i + 1], c0 = k0[3 * i + 2];
    int zc[P];
#pragma unroll
    for (int c = 0; c < P; c++) {
        int gc = c0 + c;
        if (gc >= K.z) gc -= K.z;
        zc[c] = gc;
    }
    R f[NS][NC];
#pragma unroll
    for (int s = 0; s < NS; s++)
#pragma unroll
        for (int j = 0; j < NC; j++) f[s][j] = 0;
    for (int l = lane; l < P * P; l += G) {
        const int a = l / P, b = l - (l / P) * P;
        int ga = a0 + a; if (ga >= K.x) ga -= K.x;
        int gb = b0 + b; if (gb >= K.y) gb -= K.y;
        const size_t line = ((size_t)ga * K.y + gb) * K.z;
        R z[NS][4], x[4], y[4];
#pragma unroll
        for (int d = 0; d < 4; d++) {
            x[d] = d < ND ? t1[d * P + a] : R(0);
            y[d] = d < ND ? t2[d * P + b] : R(0);
#pragma unroll
            for (int s = 0; s < NS; s++) z[s][d] = 0;
        }
        C qv[P];
        if constexpr (NS == 2) load_line<P>(static_cast<const C*>(gridv) + line, c0, K.z, qv);
#pragma unroll
        for (int c = 0; c < P; c++) {
            R q[NS];
            if constexpr (NS == 2) {
                q[0] = qv[c].x;
                q[NS - 1] = qv[c].y;
            } else {
                q[0] = static_cast<const R*>(gridv)[line + zc[c]];
            }
#pragma unroll
            for (int d = 0; d < ND; d++) {
                const R w = t3[d * P + c];
#pragma unroll
                for (int s = 0; s < NS; s++) z[s][d] += w * q[s];
            }
        }
#pragma unroll
        for (int s = 0; s < NS; s++) add_derivs<R, NC>(f[s], x, y, z[s]);
    }
    double sum[NS][NC];
#pragma unroll
    for (int s = 0; s < NS; s++)
#pragma unroll
        for (int j = 0; j < NC; j++) sum[s][j] = group_sum<G>((double)f[s][j]);
    if (g >= n) return;
    const int ex[20][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {2, 0, 0}, {0, 2, 0}, {0, 0, 2},
                           {1, 1, 0}, {1, 0, 1}, {0, 1, 1}, {3, 0, 0}, {0, 3, 0}, {0, 0, 3}, {2, 1, 0},
                           {2, 0, 1}, {1, 2, 0}, {0, 2, 1}, {1, 0, 2}, {0, 1, 2}, {1, 1, 1}};
    if (F.general) {
#pragma unroll
        for (int s = 0; s < NS; s++) {
            double fs[NC];
#pragma unroll
            for (int j = 0; j < NC; j++) fs[j] = sum[s][j];
            for (int j = lane; j < NC; j += G) phi[(size_t)s * NC * n + (size_t)NC * i + j] = cart_deriv(F, fs, NC, j);
        }
        return;
    }
    const double sc0 = F.m[0][0], sc1 = F.m[1][1], sc2 = F.m[2][2];
    const double p0[4] = {1, sc0, sc0 * sc0, sc0 * sc0 * sc0};
    const double p1[4] = {1, sc1, sc1 * sc1, sc1 * sc1 * sc1};
    const double p2[4] = {1, sc2, sc2 * sc2, sc2 * sc2 * sc2};
#pragma unroll
    for (int s = 0; s < NS; s++)
#pragma unroll
        for (int j = 0; j < NC; j++)
            if (j % G == lane)
                phi[(size_t)s * NC * n + (size_t)NC * i + j] = sum[s][j] * p0[ex[j][0]] * p1[ex[j][1]] * p2[ex[j][2]];
}

}  // namespace amg
