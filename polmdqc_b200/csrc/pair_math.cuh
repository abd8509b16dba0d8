// pair_math.cuh -- pair interactions of the AMOEBA electrostatics path in
// invariant form, for one precision R (float for the mixed path, double for
// the FP64 path and for the scaled-pair corrections).
//
// Every interaction is written with a generic radial hierarchy
//   B_n(r) = (-1/r d/dr)^n psi(r),   n = 0..5,
// so one formula serves all channels:
//   bare Coulomb     psi = 1/r           B_n = (2n-1)!!/r^(2n+1)
//   Ewald real space psi = erfc(a r)/r   (Smith recursion)
//   Thole damping    B_n = lambda_(2n+1)(r) (2n-1)!!/r^(2n+1)
//   scaled pairs     (s - 1) lambda B_n^bare, added to the s = 1 bulk value.
//
// Multipole energy of sites i and k (r = x_k - x_i, multipoles [q, d, Q] with
// Q pre-divided by 3 as in the reference, src/md/kmpole.cpp:547-550):
//   E = sum_n c_n B_n,  with  a = d.r, b = r.Q.r, Qr = Q r and
//   c0 = qi qk
//   c1 = qk ai - qi ak + di.dk
//   c2 = qi bk + qk bi - ai ak + 2 (dk.Qri - di.Qrk + Qi:Qk)
//   c3 = ai bk - ak bi - 4 Qri.Qrk
//   c4 = bi bk
// which is the Cartesian multipole expansion the reference evaluates with
// undamped radial factors in include/md/pairMpole.h:21-175.  The gradient
// and the torques below are derived from these invariants (dB_n/dr_vec =
// -r B_{n+1}; torque = -(d x dE/dd) - 2 axial(Q dE/dQ)).
#pragma once
#include <cuda_runtime.h>

namespace amg {

template <class R>
struct V3 {
    R x, y, z;
};
template <class R>
__host__ __device__ __forceinline__ V3<R> v3(R x, R y, R z) { return {x, y, z}; }
template <class R>
__host__ __device__ __forceinline__ V3<R> operator+(V3<R> a, V3<R> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class R>
__host__ __device__ __forceinline__ V3<R> operator-(V3<R> a, V3<R> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class R>
__host__ __device__ __forceinline__ V3<R> operator*(R s, V3<R> a) { return {s * a.x, s * a.y, s * a.z}; }
template <class R>
__host__ __device__ __forceinline__ R dot(V3<R> a, V3<R> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class R>
__host__ __device__ __forceinline__ V3<R> cross(V3<R> a, V3<R> b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}

// symmetric 3x3 (quadrupole), stored xx xy xz yy yz zz
template <class R>
struct Sym {
    R xx, xy, xz, yy, yz, zz;
};
template <class R>
__host__ __device__ __forceinline__ V3<R> mul(const Sym<R>& Q, V3<R> v) {
    return {Q.xx * v.x + Q.xy * v.y + Q.xz * v.z, Q.xy * v.x + Q.yy * v.y + Q.yz * v.z,
            Q.xz * v.x + Q.yz * v.y + Q.zz * v.z};
}
template <class R>
__host__ __device__ __forceinline__ R ddot(const Sym<R>& A, const Sym<R>& B) {
    return A.xx * B.xx + A.yy * B.yy + A.zz * B.zz + 2 * (A.xy * B.xy + A.xz * B.xz + A.yz * B.yz);
}
// axial vector of the product A B: (axial)_c = eps_cda (A B)_da
template <class R>
__host__ __device__ __forceinline__ V3<R> axial_prod(const Sym<R>& A, const Sym<R>& B) {
    // (AB)_yz - (AB)_zy, (AB)_zx - (AB)_xz, (AB)_xy - (AB)_yx
    R ab_yz = A.xy * B.xz + A.yy * B.yz + A.yz * B.zz;
    R ab_zy = A.xz * B.xy + A.yz * B.yy + A.zz * B.yz;
    R ab_zx = A.xz * B.xx + A.yz * B.xy + A.zz * B.xz;
    R ab_xz = A.xx * B.xz + A.xy * B.yz + A.xz * B.zz;
    R ab_xy = A.xx * B.xy + A.xy * B.yy + A.xz * B.yz;
    R ab_yx = A.xy * B.xx + A.yy * B.xy + A.yz * B.xz;
    return {ab_yz - ab_zy, ab_zx - ab_xz, ab_xy - ab_yx};
}

template <class R>
struct Mpole {
    R q;
    V3<R> d;
    Sym<R> Q;
};

// ------------------------------------------------------------ radial parts
template <class R>
__device__ __forceinline__ R rsqrt_(R x);
template <>
__device__ __forceinline__ float rsqrt_<float>(float x) { return rsqrtf(x); }
template <>
__device__ __forceinline__ double rsqrt_<double>(double x) { return rsqrt(x); }

template <class R>
__device__ __forceinline__ R exp_(R x);
template <>
__device__ __forceinline__ float exp_<float>(float x) { return __expf(x); }
template <>
__device__ __forceinline__ double exp_<double>(double x) { return exp(x); }

// quotient for the damping ratio r / damp: the fast FP32 division (a few
// ulp, within the FP32 pair arithmetic's error) or the exact FP64 one
template <class R>
__device__ __forceinline__ R ratio_(R a, R b);
template <>
__device__ __forceinline__ float ratio_<float>(float a, float b) { return __fdividef(a, b); }
template <>
__device__ __forceinline__ double ratio_<double>(double a, double b) { return a / b; }

template <class R>
__device__ __forceinline__ R erfc_(R x);
template <>
__device__ __forceinline__ float erfc_<float>(float x) { return erfcf(x); }
template <>
__device__ __forceinline__ double erfc_<double>(double x) { return erfc(x); }

// bare B_n = (2n-1)!!/r^(2n+1), n = 0..N-1
template <class R, int N>
__device__ __forceinline__ void bare_terms(R rinv, R rinv2, R (&b)[N]) {
    b[0] = rinv;
#pragma unroll
    for (int n = 1; n < N; n++) b[n] = b[n - 1] * rinv2 * R(2 * n - 1);
}

// Ewald B_n from erfc(a r)/r by the Smith recursion
//   B_n = ((2n-1) B_{n-1} + (2a^2)^n/(a sqrt(pi)) exp(-a^2 r^2)) / r^2
template <class R, int N>
__device__ __forceinline__ void ewald_terms(R r, R rinv2, R aewald, R (&b)[N]) {
    const R a2 = aewald * aewald;
    const R ex = exp_<R>(-a2 * r * r);
    R fac = R(0.56418958354775628695) / aewald;  // 1/(a sqrt(pi))
    b[0] = erfc_<R>(aewald * r) * (rinv2 * r);
#pragma unroll
    for (int n = 1; n < N; n++) {
        fac *= 2 * a2;
        b[n] = (R(2 * n - 1) * b[n - 1] + fac * ex) * rinv2;
    }
}

// AMOEBA Thole factors lambda_3,5,7,9 (index n = 1..4 multiplies bare B_n);
// x = a (r/damp)^3 with damp = pdamp_i pdamp_k, a = pair Thole value.
template <class R>
__device__ __forceinline__ void thole_lambda(R r, R damp, R a, R (&lam)[5]) {
    lam[0] = lam[1] = lam[2] = lam[3] = lam[4] = R(1);
    if (damp != R(0)) {
        R t = ratio_<R>(r, damp);
        R x = a * t * t * t;
        R e = exp_<R>(-x);
        lam[1] = R(1) - e;
        lam[2] = R(1) - (R(1) + x) * e;
        lam[3] = R(1) - (R(1) + x + R(0.6) * x * x) * e;
        lam[4] = R(1) - (R(1) + x + (R(18) / R(35)) * x * x + (R(9) / R(35)) * x * x * x) * e;
    }
}

// ------------------------------------------------------------ site helpers
template <class R>
struct SiteInv {  // invariants of one site against the pair vector
    R a, b;       // d.r, r.Q.r
    V3<R> Qr;     // Q r
};
template <class R>
__device__ __forceinline__ SiteInv<R> invariants(const Mpole<R>& M, V3<R> r) {
    SiteInv<R> s;
    s.a = dot(M.d, r);
    s.Qr = mul(M.Q, r);
    s.b = dot(s.Qr, r);
    return s;
}

// ---------------------------------------------------------------- mm pair
// Full multipole pair seen from site i (r = x_k - x_i): energy E (whole
// pair), gradient dE/dx_i and torque on i.  B[0..5].
template <class R>
__device__ __forceinline__ void mm_pair_i(const Mpole<R>& Mi, const Mpole<R>& Mk, V3<R> r, const R (&B)[6],
                                          R& E, V3<R>& gi, V3<R>& ti) {
    SiteInv<R> si = invariants(Mi, r), sk = invariants(Mk, r);
    R dik = dot(Mi.d, Mk.d);
    R dkQri = dot(Mk.d, si.Qr), diQrk = dot(Mi.d, sk.Qr);
    R QiQk = ddot(Mi.Q, Mk.Q);
    R QriQrk = dot(si.Qr, sk.Qr);
    R c0 = Mi.q * Mk.q;
    R c1 = Mk.q * si.a - Mi.q * sk.a + dik;
    R c2 = Mi.q * sk.b + Mk.q * si.b - si.a * sk.a + 2 * (dkQri - diQrk + QiQk);
    R c3 = si.a * sk.b - sk.a * si.b - 4 * QriQrk;
    R c4 = si.b * sk.b;
    E = c0 * B[0] + c1 * B[1] + c2 * B[2] + c3 * B[3] + c4 * B[4];
    R G = c0 * B[1] + c1 * B[2] + c2 * B[3] + c3 * B[4] + c4 * B[5];
    R s_di = Mk.q * B[1] - sk.a * B[2] + sk.b * B[3];
    R s_dk = -Mi.q * B[1] - si.a * B[2] - si.b * B[3];
    R s_qi2 = Mk.q * B[2] - sk.a * B[3] + sk.b * B[4];  // half of s_qi
    R s_qk2 = Mi.q * B[2] + si.a * B[3] + si.b * B[4];
    V3<R> Qi_dk = mul(Mi.Q, Mk.d), Qk_di = mul(Mk.Q, Mi.d);
    V3<R> Qi_Qrk = mul(Mi.Q, sk.Qr), Qk_Qri = mul(Mk.Q, si.Qr);
    // dE/dr
    V3<R> dEdr = (-G) * r + s_di * Mi.d + s_dk * Mk.d + (2 * s_qi2) * si.Qr + (2 * s_qk2) * sk.Qr +
                 (2 * B[2]) * (Qi_dk - Qk_di) + (-4 * B[3]) * (Qi_Qrk + Qk_Qri);
    gi = (R(-1)) * dEdr;
    // torque on i
    V3<R> dEddi = s_di * r + B[1] * Mk.d + (-2 * B[2]) * sk.Qr;
    V3<R> t = cross(Mi.d, dEddi);
    t = t + (2 * s_qi2) * cross(si.Qr, r);
    t = t + (2 * B[2]) * (cross(Qi_dk, r) + cross(si.Qr, Mk.d));
    t = t + (-4 * B[3]) * (cross(Qi_Qrk, r) + cross(si.Qr, sk.Qr));
    t = t + (4 * B[2]) * axial_prod(Mi.Q, Mk.Q);
    ti = (R(-1)) * t;
}

// ---------------------------------------------------------------- fields
// Field at site k from multipole i (r = x_k - x_i), B[1..3]:
//   E_k = r (qi B1 + ai B2 + bi B3) - di B1 - 2 Qri B2
template <class R>
__device__ __forceinline__ V3<R> field_of_mpole(const Mpole<R>& Mi, V3<R> r, R B1, R B2, R B3) {
    SiteInv<R> si = invariants(Mi, r);
    return (Mi.q * B1 + si.a * B2 + si.b * B3) * r - B1 * Mi.d - (2 * B2) * si.Qr;
}

// Field at site k from a dipole u at site i: E_k = r (u.r) B2 - u B1
template <class R>
__device__ __forceinline__ V3<R> field_of_dipole(V3<R> u, V3<R> r, R B1, R B2) {
    return (dot(u, r) * B2) * r - B1 * u;
}

// ---------------------------------------------------------------- polarization
// Gradient dE/dr of E(M_i, v_k): multipole at i, dipole v at k (r = x_k - x_i),
// and the torque on M_i.  B[1..4].
template <class R>
__device__ __forceinline__ void md_pair(const Mpole<R>& Mi, const SiteInv<R>& si, V3<R> v, V3<R> r,
                                        const R (&B)[6], V3<R>& dEdr, V3<R>& ti) {
    R av = dot(v, r);
    R c1 = -Mi.q * av + dot(Mi.d, v);
    R c2 = -si.a * av + 2 * dot(v, si.Qr);
    R c3 = -av * si.b;
    R G = c1 * B[2] + c2 * B[3] + c3 * B[4];
    R s_di = -av * B[2];
    R s_dk = -Mi.q * B[1] - si.a * B[2] - si.b * B[3];
    R s_qi = -2 * av * B[3];
    V3<R> Qiv = mul(Mi.Q, v);
    dEdr = (-G) * r + s_di * Mi.d + s_dk * v + s_qi * si.Qr + (2 * B[2]) * Qiv;
    V3<R> dEddi = s_di * r + B[1] * v;
    V3<R> t = cross(Mi.d, dEddi) + s_qi * cross(si.Qr, r) + (2 * B[2]) * (cross(Qiv, r) + cross(si.Qr, v));
    ti = (R(-1)) * t;
}

// Gradient dE/dr of E(w_i, M_k): dipole w at i, multipole at k (r = x_k - x_i).
template <class R>
__device__ __forceinline__ V3<R> dm_pair(V3<R> w, const Mpole<R>& Mk, const SiteInv<R>& sk, V3<R> r,
                                         const R (&B)[6]) {
    R aw = dot(w, r);
    R c1 = Mk.q * aw + dot(w, Mk.d);
    R c2 = -aw * sk.a - 2 * dot(w, sk.Qr);
    R c3 = aw * sk.b;
    R G = c1 * B[2] + c2 * B[3] + c3 * B[4];
    R s_di = Mk.q * B[1] - sk.a * B[2] + sk.b * B[3];
    R s_dk = -aw * B[2];
    R s_qk = 2 * aw * B[3];
    return (-G) * r + s_di * w + s_dk * Mk.d + s_qk * sk.Qr + (-2 * B[2]) * mul(Mk.Q, w);
}

// Gradient dE/dr of the dipole-dipole energy E(a_i, b_k) = (a.b) B1 - (a.r)(b.r) B2.
template <class R>
__device__ __forceinline__ V3<R> dd_pair(V3<R> a, V3<R> b, V3<R> r, const R (&B)[6]) {
    R aa = dot(a, r), ab = dot(b, r);
    R G = dot(a, b) * B[2] - aa * ab * B[3];
    return (-G) * r + (-ab * B[2]) * a + (-aa * B[2]) * b;
}

}  // namespace amg
