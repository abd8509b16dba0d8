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

// ------------------------------------------------ spreading by bricks
// The grid is cut into bricks of B grid points per axis (the last brick of an
// axis may be shorter, but not shorter than P-1); sites are sorted by the
// brick holding their stencil start k0.  Phase 1: one block per brick adds
// its sites' P^3 stencils into a shared-memory region of E = B + P - 1 points
// per axis (the brick plus the P-1 points its stencils reach beyond it) and
// stores the region with plain writes.  Phase 2: every grid point sums the
// one to eight regions that cover it (its own brick's and, within P-1 points
// of a brick's low faces, the preceding bricks', periodically) and writes the
// grid.  No global atomics; the grid needs no clearing.
struct Bricks {
    int3 B;   // brick edge per axis
    int3 nb;  // bricks per axis
    int3 E;   // region edge per axis, B + P - 1
};

__device__ __forceinline__ int brick_len(int b, int B, int nb, int K) { return b == nb - 1 ? K - b * B : B; }

__global__ void k_brick_keys(int n, const int* __restrict__ k0, Bricks bk, unsigned* __restrict__ keys,
                             int* __restrict__ ids) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int bx = min(k0[3 * i] / bk.B.x, bk.nb.x - 1);
    const int by = min(k0[3 * i + 1] / bk.B.y, bk.nb.y - 1);
    const int bz = min(k0[3 * i + 2] / bk.B.z, bk.nb.z - 1);
    keys[i] = (unsigned)((bx * bk.nb.y + by) * bk.nb.z + bz);
    ids[i] = i;
}

// start/end of every non-empty brick in the sorted keys (others stay 0/0)
__global__ void k_brick_bounds(int n, const unsigned* __restrict__ skeys, int* __restrict__ start,
                               int* __restrict__ end) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const unsigned k = skeys[i];
    if (i == 0 || skeys[i - 1] != k) start[k] = i;
    if (i == n - 1 || skeys[i + 1] != k) end[k] = i + 1;
}

// Phase 1 for two dipole sets (FP64 [3n] each); regions [brick][2][E^3].
// The brick's sites are staged in shared memory (up to MAXA at a time: the
// ten stencil weights per axis that a dipole needs, the scaled dipoles and
// the stencil start inside the region), then consecutive threads take
// consecutive z points of one site's stencil and add into the region.
// Dynamic shared memory: 2 E^3 + MAXA (6P + 6) values of R + MAXA ints.
template <class R, int P, int MAXA>
__global__ void __launch_bounds__(256) k_spread_dipoles_brick(Bricks bk, const int* __restrict__ sids,
                                                              const int* __restrict__ bstart,
                                                              const int* __restrict__ bend,
                                                              const double* __restrict__ ud,
                                                              const double* __restrict__ up,
                                                              const R* __restrict__ theta,
                                                              const int* __restrict__ k0, R sc0, R sc1, R sc2,
                                                              R* __restrict__ regions) {
    extern __shared__ __align__(16) unsigned char brick_smem[];
    const int RE = bk.E.x * bk.E.y * bk.E.z;
    R* reg = reinterpret_cast<R*>(brick_smem);
    R* wts = reg + 2 * RE;          // [MAXA][6P]: t0 t1 u0 u1 v0 v1
    R* dip = wts + MAXA * 6 * P;    // [MAXA][6]: scaled d, p
    int* org = reinterpret_cast<int*>(dip + MAXA * 6);  // [MAXA]: region offset of the stencil start
    const int b = blockIdx.x;
    const int bz = b % bk.nb.z, by = (b / bk.nb.z) % bk.nb.y, bx = b / (bk.nb.z * bk.nb.y);
    const int lox = bx * bk.B.x, loy = by * bk.B.y, loz = bz * bk.B.z;
    for (int t = threadIdx.x; t < 2 * RE; t += blockDim.x) reg[t] = R(0);
    constexpr int P3 = P * P * P;
    const int s0 = bstart[b], s1 = bend[b];
    for (int a0 = s0; a0 < s1; a0 += MAXA) {
        const int na = min(MAXA, s1 - a0);
        __syncthreads();  // region cleared / previous batch consumed
        for (int t = threadIdx.x; t < na * 6 * P; t += blockDim.x) {
            const int ia = t / (6 * P), w = t - ia * 6 * P;
            const int i = sids[a0 + ia];
            const int dim = w / (2 * P), rest = w - dim * 2 * P;  // rest: derivative order 0/1 times P + point
            wts[t] = theta[(size_t)i * 3 * 4 * P + dim * 4 * P + rest];
        }
        for (int t = threadIdx.x; t < na * 6; t += blockDim.x) {
            const int ia = t / 6, c = t - ia * 6;
            const int i = sids[a0 + ia];
            const double v = c < 3 ? ud[3 * i + c] : up[3 * i + c - 3];
            const int ax = c % 3;
            dip[t] = (R)v * (ax == 0 ? sc0 : ax == 1 ? sc1 : sc2);
        }
        for (int t = threadIdx.x; t < na; t += blockDim.x) {
            const int i = sids[a0 + t];
            org[t] = ((k0[3 * i] - lox) * bk.E.y + (k0[3 * i + 1] - loy)) * bk.E.z + (k0[3 * i + 2] - loz);
        }
        __syncthreads();
        for (int t = threadIdx.x; t < na * P3; t += blockDim.x) {
            const int ia = t / P3, pt = t - ia * P3;
            const int a = pt / (P * P), bb = (pt / P) % P, c = pt % P;
            const R* w = wts + ia * 6 * P;
            const R t0 = w[a], t1 = w[P + a], u0 = w[2 * P + bb], u1 = w[3 * P + bb], v0 = w[4 * P + c],
                    v1 = w[5 * P + c];
            const R w100 = t1 * u0 * v0, w010 = t0 * u1 * v0, w001 = t0 * u0 * v1;
            const R* d = dip + ia * 6;
            const int q = org[ia] + (a * bk.E.y + bb) * bk.E.z + c;
            atomicAdd(reg + q, d[0] * w100 + d[1] * w010 + d[2] * w001);
            atomicAdd(reg + RE + q, d[3] * w100 + d[4] * w010 + d[5] * w001);
        }
    }
    __syncthreads();
    R* out = regions + (size_t)b * 2 * RE;
    for (int t = threadIdx.x; t < 2 * RE; t += blockDim.x) out[t] = reg[t];
}

// Phase 2: grid[set][g] = sum of the regions covering g, for two sets.
template <class R, int P>
__global__ void k_sum_bricks(Bricks bk, int3 K, const R* __restrict__ regions, R* __restrict__ grid,
                             size_t gstride) {
    const size_t g = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= gstride) return;
    const int z = (int)(g % K.z), y = (int)((g / K.z) % K.y), x = (int)(g / ((size_t)K.z * K.y));
    const int bx = min(x / bk.B.x, bk.nb.x - 1), by = min(y / bk.B.y, bk.nb.y - 1), bz = min(z / bk.B.z, bk.nb.z - 1);
    const int lx = x - bx * bk.B.x, ly = y - by * bk.B.y, lz = z - bz * bk.B.z;
    const int RE = bk.E.x * bk.E.y * bk.E.z;
    R sd = 0, sp = 0;
    for (int dx = 0; dx < 2; dx++) {
        if (dx && lx >= P - 1) break;
        const int rbx = dx ? (bx == 0 ? bk.nb.x - 1 : bx - 1) : bx;
        const int rx = dx ? lx + brick_len(rbx, bk.B.x, bk.nb.x, K.x) : lx;
        for (int dy = 0; dy < 2; dy++) {
            if (dy && ly >= P - 1) break;
            const int rby = dy ? (by == 0 ? bk.nb.y - 1 : by - 1) : by;
            const int ry = dy ? ly + brick_len(rby, bk.B.y, bk.nb.y, K.y) : ly;
            for (int dz = 0; dz < 2; dz++) {
                if (dz && lz >= P - 1) break;
                const int rbz = dz ? (bz == 0 ? bk.nb.z - 1 : bz - 1) : bz;
                const int rz = dz ? lz + brick_len(rbz, bk.B.z, bk.nb.z, K.z) : lz;
                const R* r = regions + (size_t)((rbx * bk.nb.y + rby) * bk.nb.z + rbz) * 2 * RE;
                const int q = (rx * bk.E.y + ry) * bk.E.z + rz;
                sd += r[q];
                sp += r[RE + q];
            }
        }
    }
    grid[g] = sd;
    grid[gstride + g] = sp;
}

// Gather of the field of two dipole grids (first derivatives only) fused
// with the matvec assembly:
//   A v = v/alpha - (F_real + F_recip + selfc v),  F_recip = -grad phi
// G consecutive lanes per site; each lane takes whole z-lines (a, b) of the
// P^3 stencil (P grid values per line and grid), the per-lane sums are
// combined with shuffles and lanes 0..5 write the six components.
template <class R, int P, int G>
__global__ void __launch_bounds__(128) k_gather_field(int n, const R* __restrict__ phigrid, size_t gstride,
                                                      const R* __restrict__ theta, const int* __restrict__ k0,
                                                      int3 K, double sc0, double sc1, double sc2,
                                                      const double* __restrict__ vd, const double* __restrict__ vp,
                                                      const double* __restrict__ Fd, const double* __restrict__ Fp,
                                                      double selfc, const double* __restrict__ pol,
                                                      double* __restrict__ Ad, double* __restrict__ Ap) {
    const int g = (blockIdx.x * blockDim.x + threadIdx.x) / G, lane = threadIdx.x % G;
    const int i = min(g, n - 1);
    const R* th = theta + (size_t)i * 3 * 4 * P;
    const int a0 = k0[3 * i], b0 = k0[3 * i + 1], c0 = k0[3 * i + 2];
    R v0[P], v1[P];
    int zc[P];
#pragma unroll
    for (int c = 0; c < P; c++) {
        v0[c] = th[8 * P + c];
        v1[c] = th[9 * P + c];
        int gc = c0 + c;
        if (gc >= K.z) gc -= K.z;
        zc[c] = gc;
    }
    R f[6] = {0, 0, 0, 0, 0, 0};
    for (int l = lane; l < P * P; l += G) {
        const int a = l / P, b = l - (l / P) * P;
        int ga = a0 + a; if (ga >= K.x) ga -= K.x;
        int gb = b0 + b; if (gb >= K.y) gb -= K.y;
        const R* line = phigrid + ((size_t)ga * K.y + gb) * K.z;
        R sd0 = 0, sd1 = 0, sp0 = 0, sp1 = 0;
#pragma unroll
        for (int c = 0; c < P; c++) {
            const R qd = line[zc[c]], qp = line[gstride + zc[c]];
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
        const double v = t == 0 ? sum[0] : t == 1 ? sum[1] : t == 2 ? sum[2] : t == 3 ? sum[3] : t == 4 ? sum[4] : sum[5];
        const double scv = c == 0 ? sc0 : c == 1 ? sc1 : sc2;
        const bool dset = t < 3;
        const double* vv = dset ? vd : vp;
        const double* FF = dset ? Fd : Fp;
        double* AA = dset ? Ad : Ap;
        const double alpha = pol[i];
        const double field = FF[3 * i + c] - v * scv + selfc * vv[3 * i + c];
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
