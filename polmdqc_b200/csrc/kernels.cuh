// kernels.cuh -- the sm_100a kernels of the electrostatics path.
//
// Data layout in HBM (per atom, original atom order):
//   AtomR<R> : 4 x R4  = (x,y,z,q) (dx,dy,dz,Qxx) (Qxy,Qxz,Qyy,Qyz)
//              (Qzz, pdamp, thole, polarity)   -- 64 B per atom in FP32
//   induced dipoles (and PCG vectors) as double[3n]; R4 copies for the
//   pair kernels; neighbour rows site-major (nbr[i*cap + slot]), read by a
//   lane group per site.
#pragma once
#include "device_util.cuh"
#include "pair_math.cuh"

namespace amg {

constexpr double kPi = 3.141592653589793238462643383279502884;
constexpr double kSqrt2 = 1.414213562373095048801688724209698079;
constexpr double kSqrtPi = 1.772453850905516027298167483341145183;

template <class R>
struct AtomR {
    R4<R> a, b, c, e;
};

struct Box {
    double L[3];       // box lengths (0: no periodic wrapping on that axis)
    double iL[3];
    // cell shape: 0 orthogonal, 1 monoclinic, 2 triclinic, 3 truncated
    // octahedron, 4 rhombic dodecahedron; lattice terms of the reference's
    // lattice (src/md/lattice.cpp:80-110)
    int shape;
    double bsin, bcos, gsin, gcos, bterm, gterm;
};

// Cartesian -> grid units of the PME: u_j = sum_i x_i m[i][j] (m = inverse
// lattice times K_j), so d/dx_i = sum_j m[i][j] d/du_j.  For an orthogonal
// box m is diagonal (K/L) and `general` is 0: the kernels then take the
// diagonal scalings alone.
struct Frac {
    double m[3][3];
    int general;
};

template <class R>
__device__ __forceinline__ Mpole<R> load_mpole(const AtomR<R>& A) {
    Mpole<R> M;
    M.q = A.a.w;
    M.d = v3<R>(A.b.x, A.b.y, A.b.z);
    M.Q = Sym<R>{A.b.w, A.c.x, A.c.y, A.c.z, A.c.w, A.e.x};
    return M;
}

// Minimum image of the non-orthogonal cells, restating the reference's
// image() (src/md/image.cpp:37-124): wrap along the cell axes in scaled
// fractional coordinates (monoclinic, triclinic), or wrap in the enclosing
// box and remove the corner images (truncated octahedron, rhombic
// dodecahedron with zbox = sqrt(2) xbox).
template <class R>
__device__ __noinline__ V3<R> image_cell(V3<R> d, const Box bx) {
    const R L0 = (R)bx.L[0], L1 = (R)bx.L[1], L2 = (R)bx.L[2];
    const R i0 = (R)bx.iL[0], i1 = (R)bx.iL[1], i2 = (R)bx.iL[2];
    if (bx.shape == 1) {
        const R bs = (R)bx.bsin, bc = (R)bx.bcos;
        R z = d.z / bs, x = d.x - z * bc;
        x = wrap1<R>(x, L0, i0);
        const R y = wrap1<R>(d.y, L1, i1);
        z = wrap1<R>(z, L2, i2);
        return v3<R>(x + z * bc, y, z * bs);
    }
    if (bx.shape == 2) {
        const R gs = (R)bx.gsin, gc = (R)bx.gcos, bc = (R)bx.bcos, bt = (R)bx.bterm, gt = (R)bx.gterm;
        R z = d.z / gt, y = (d.y - z * bt) / gs, x = d.x - y * gc - z * bc;
        x = wrap1<R>(x, L0, i0);
        y = wrap1<R>(y, L1, i1);
        z = wrap1<R>(z, L2, i2);
        return v3<R>(x + y * gc + z * bc, y * gs + z * bt, z * gt);
    }
    V3<R> r;
    if (bx.shape == 3) {
        r = v3<R>(wrap1<R>(d.x, L0, i0), wrap1<R>(d.y, L1, i1), wrap1<R>(d.z, L2, i2));
        if (fabs(r.x) + fabs(r.y) + fabs(r.z) > R(0.75) * L0) {
            r.x -= copysign(R(0.5) * L0, r.x);
            r.y -= copysign(R(0.5) * L1, r.y);
            r.z -= copysign(R(0.5) * L2, r.z);
        }
        return r;
    }
    // rhombic dodecahedron
    const R r2 = (R)1.41421356237309504880;
    r = v3<R>(wrap1<R>(d.x, L0, i0), wrap1<R>(d.y, L1, i1), d.z - r2 * L2 * round(d.z / (L2 * r2)));
    const R corr = R(0.5) * L0 * (R)(int)(fabs(r.x * i0) + fabs(r.y * i1) + fabs(r2 * r.z * i2));
    r.x -= copysign(corr, r.x);
    r.y -= copysign(corr, r.y);
    r.z -= copysign(corr, r.z) * r2;
    return r;
}

// CELLS false: the box is orthogonal (or absent) by construction, as in
// the default instances of the Ewald pair kernels; true: any cell shape, the
// non-orthogonal ones through image_cell (the pair kernels' CELLS instances,
// launched for Ewald in a monoclinic or triclinic cell).
template <class R, bool CELLS = true>
__device__ __forceinline__ V3<R> min_image(V3<R> d, const Box& bx) {
    if (CELLS && bx.shape != 0) return image_cell<R>(d, bx);
    return v3<R>(wrap1<R>(d.x, (R)bx.L[0], (R)bx.iL[0]), wrap1<R>(d.y, (R)bx.L[1], (R)bx.iL[1]),
                 wrap1<R>(d.z, (R)bx.L[2], (R)bx.iL[2]));
}

// pair Thole value: the smaller, or the larger when the smaller is zero
// (src/md/kpolar.cpp:514-517)
template <class R>
__device__ __forceinline__ R pair_thole(R ti, R tk) {
    R a = fmin(ti, tk);
    return a == R(0) ? fmax(ti, tk) : a;
}

// Radial hierarchy of the bulk (unscaled) pair: Ewald (or bare) minus the
// part removed by Thole damping, B_n = ewald_n - (1 - lam_n) bare_n.
template <class R, bool EWALD, bool THOLE>
__device__ __forceinline__ void bulk_radial(R r2, R aewald, R damp, R thl, R (&B)[6]) {
    R rinv = rsqrt_<R>(r2);
    R r = r2 * rinv;
    R rinv2 = rinv * rinv;
    R bare[6];
    bare_terms<R, 6>(rinv, rinv2, bare);
    if (EWALD) {
        ewald_terms<R, 6>(r, rinv2, aewald, B);
    } else {
#pragma unroll
        for (int n = 0; n < 6; n++) B[n] = bare[n];
    }
    if (THOLE) {
        R lam[5];
        thole_lambda<R>(r, damp, thl, lam);
#pragma unroll
        for (int n = 1; n < 5; n++) B[n] -= (R(1) - lam[n]) * bare[n];
    }
}

// bulk_radial with Thole damping that also returns the bare Thole-damped
// lambda_3 b_1 and lambda_5 b_2 (the sparse preconditioner's tensor)
template <class R, bool EWALD>
__device__ __forceinline__ void bulk_radial_prec(R r2, R aewald, R damp, R thl, R (&B)[6], R& P1, R& P2) {
    R rinv = rsqrt_<R>(r2);
    R r = r2 * rinv;
    R rinv2 = rinv * rinv;
    R bare[6];
    bare_terms<R, 6>(rinv, rinv2, bare);
    if (EWALD) {
        ewald_terms<R, 6>(r, rinv2, aewald, B);
    } else {
#pragma unroll
        for (int n = 0; n < 6; n++) B[n] = bare[n];
    }
    R lam[5];
    thole_lambda<R>(r, damp, thl, lam);
#pragma unroll
    for (int n = 1; n < 5; n++) B[n] -= (R(1) - lam[n]) * bare[n];
    P1 = lam[1] * bare[1];
    P2 = lam[2] * bare[2];
}

// Stored dipole-tensor coefficients of one directed pair, T = B2 r r^T - B1 I,
// packed in one R4: w = sqrt(|B2|) r and B1, with the sign of B2 kept in the
// lowest mantissa bit of B1 (a change of one unit in the last place of B1), so
//   T u = s (w.u) w - B1 u,  s = sign(B2).
// 16 bytes per pair in FP32 instead of 20 for (r, B1) and B2.
__device__ __forceinline__ float flag_lsb(float v, bool f) {
    return __uint_as_float((__float_as_uint(v) & ~1u) | (f ? 1u : 0u));
}
__device__ __forceinline__ double flag_lsb(double v, bool f) {
    return __longlong_as_double((__double_as_longlong(v) & ~1ll) | (f ? 1ll : 0ll));
}
__device__ __forceinline__ bool lsb_of(float v) { return __float_as_uint(v) & 1u; }
__device__ __forceinline__ bool lsb_of(double v) { return __double_as_longlong(v) & 1ll; }

template <class R>
__device__ __forceinline__ R4<R> pack_tensor(R rx, R ry, R rz, R B1, R B2) {
    const R sq = sqrt(fabs(B2));
    return make_r4<R>(sq * rx, sq * ry, sq * rz, flag_lsb(B1, B2 < R(0)));
}

// accumulate T v for the packed coefficient c into (fx, fy, fz)
template <class R>
__device__ __forceinline__ void apply_tensor(const R4<R>& c, const R4<R>& v, R& fx, R& fy, R& fz) {
    R a = v.x * c.x + v.y * c.y + v.z * c.z;
    a = lsb_of(c.w) ? -a : a;
    fx += a * c.x - c.w * v.x;
    fy += a * c.y - c.w * v.y;
    fz += a * c.z - c.w * v.z;
}

// streaming (evict-first) load of one packed coefficient: the rows are read
// once per launch and would otherwise push the gathered vectors out of L2
template <class R>
__device__ __forceinline__ R4<R> load_stream(const R4<R>* p) {
    if constexpr (sizeof(R) == 4) {
        return __ldcs(reinterpret_cast<const float4*>(p));
    } else {
        const double2 a = __ldcs(reinterpret_cast<const double2*>(p));
        const double2 b = __ldcs(reinterpret_cast<const double2*>(p) + 1);
        return make_r4<R>(a.x, a.y, b.x, b.y);
    }
}

// The two vectors v4[2j], v4[2j+1] of partner j (adjacent, 32-byte aligned:
// the arrays come from cudaMalloc) with 256-bit loads: one request for both
// FP32 vectors, two for the FP64 ones, instead of one per 16 bytes.  Read
// through the non-coherent path: the kernels using it never write v4.
__device__ __forceinline__ void load_pair(const float4* __restrict__ v4, int j, float4& d, float4& p) {
    asm("ld.global.nc.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
        : "=f"(d.x), "=f"(d.y), "=f"(d.z), "=f"(d.w), "=f"(p.x), "=f"(p.y), "=f"(p.z), "=f"(p.w)
        : "l"(v4 + 2 * (size_t)j));
}
__device__ __forceinline__ void load_pair(const double4* __restrict__ v4, int j, double4& d, double4& p) {
    asm("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];"
        : "=d"(d.x), "=d"(d.y), "=d"(d.z), "=d"(d.w)
        : "l"(v4 + 2 * (size_t)j));
    asm("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];"
        : "=d"(p.x), "=d"(p.y), "=d"(p.z), "=d"(p.w)
        : "l"(v4 + 2 * (size_t)j + 1));
}

// one 32-byte aligned FP64 vector with a single 256-bit load (read-only data)
__device__ __forceinline__ double4 ld256(const double4* __restrict__ p) {
    double4 v;
    asm("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];" : "=d"(v.x), "=d"(v.y), "=d"(v.z), "=d"(v.w) : "l"(p));
    return v;
}

// One site's packed data (64 bytes in FP32, 128 in FP64; 32-byte aligned)
// with 256-bit loads, for the pair kernels' partner gathers (read-only there).
__device__ __forceinline__ AtomR<float> ld_atom(const AtomR<float>* __restrict__ at, int j) {
    AtomR<float> A;
    const float4* p = reinterpret_cast<const float4*>(at + j);
    load_pair(p, 0, A.a, A.b);
    load_pair(p, 1, A.c, A.e);
    return A;
}
__device__ __forceinline__ AtomR<double> ld_atom(const AtomR<double>* __restrict__ at, int j) {
    AtomR<double> A;
    const double4* p = reinterpret_cast<const double4*>(at + j);
    load_pair(p, 0, A.a, A.b);
    load_pair(p, 1, A.c, A.e);
    return A;
}

// Sum of T v over one stored row (cnt slots from `base`; partner indices and
// packed coefficients side by side) for two vector sets v4[2j], v4[2j+1],
// the row's LPA lanes taking every LPA-th slot.  Software-pipelined: the next
// batch of U indices and coefficients is requested before the current batch's
// partner vectors are consumed, so a lane keeps two memory round trips in
// flight (the kernels using it are bound by memory latency).  Empty slots
// point at `self` with a zero coefficient.
template <class R, int LPA, int U>
__device__ __forceinline__ void row_apply(const int* __restrict__ idx, const R4<R>* __restrict__ coef, size_t base,
                                          int cnt, int lane, int self, const R4<R>* __restrict__ v4, R& ax, R& ay,
                                          R& az, R& bx, R& by, R& bz) {
    int jn[U];
    R4<R> cn[U];
    auto fetch = [&](int s0) {
#pragma unroll
        for (int q = 0; q < U; q++) {
            const int s = s0 + q * LPA;
            const bool ok = s < cnt;
            jn[q] = ok ? __ldcs(idx + base + s) : self;
            cn[q] = ok ? load_stream<R>(coef + base + s) : make_r4<R>(0, 0, 0, 0);
        }
    };
    fetch(lane);
    for (int s0 = lane; s0 < cnt; s0 += U * LPA) {
        int j[U];
        R4<R> c[U];
#pragma unroll
        for (int q = 0; q < U; q++) {
            j[q] = jn[q];
            c[q] = cn[q];
        }
        R4<R> vd[U], vp[U];
#pragma unroll
        for (int q = 0; q < U; q++) load_pair(v4, j[q], vd[q], vp[q]);
        fetch(s0 + U * LPA);
#pragma unroll
        for (int q = 0; q < U; q++) {
            apply_tensor<R>(c[q], vd[q], ax, ay, az);
            apply_tensor<R>(c[q], vp[q], bx, by, bz);
        }
    }
}

// PCG scalars: rz (current), p.Ap, rz of the next iteration, r.r, and the
// previous rz for the direction update
enum Scal { RZ_D = 0, RZ_P, PAP_D, PAP_P, RZN_D, RZN_P, RR_D, RR_P, RZO_D, RZO_P, NSCAL };

// rz_old <- rz, rz <- rz_new (cleared): the scalars of the direction update
// p = z + (rz / rz_old) p that follows (rz_old = 0 on the first iteration
// gives p = z)
__device__ __forceinline__ void pcg_roll(double* __restrict__ scal) {
    scal[RZO_D] = scal[RZ_D];
    scal[RZO_P] = scal[RZ_P];
    scal[RZ_D] = scal[RZN_D];
    scal[RZ_P] = scal[RZN_P];
    scal[RZN_D] = scal[RZN_P] = 0;
}

// PCG control (one thread), after the residual update: counts the iteration,
// decides whether to continue (residual above threshold and fewer than
// politer iterations) and, inside a captured graph, sets the WHILE node's
// condition.  `first` marks the decision taken right after the initial
// residual; `roll` rolls the rz scalars here (diagonal preconditioner, whose
// z comes with the update; the sparse preconditioner rolls them itself).
// The loop body starts with the preconditioner and the direction update, so
// an iteration that meets the threshold ends the loop without them.
__device__ __forceinline__ void pcg_decide(double* __restrict__ scal, int* __restrict__ iter, double thr2, int maxit,
                                           int first, int roll, cudaGraphConditionalHandle h, int use_handle,
                                           int* __restrict__ cont_out) {
    int it = first ? 0 : *iter + 1;
    *iter = it;
    if (!first && roll) pcg_roll(scal);
    double e2 = fmax(scal[RR_D], scal[RR_P]);
    int cont = (e2 > thr2) && (it < maxit);
    *cont_out = cont;
    if (cont) {  // accumulators of the next iteration
        scal[PAP_D] = scal[PAP_P] = 0;
        scal[RR_D] = scal[RR_P] = 0;
    }
    if (use_handle) cudaGraphSetConditional(h, cont ? 1u : 0u);
}

}  // namespace amg
