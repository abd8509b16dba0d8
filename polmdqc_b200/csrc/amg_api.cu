// amg_api.cu -- host side of libamoeba_gpu.so: the C ABI of
// include/amoeba_gpu.h, device buffers, cuFFT plans and the evaluation
// pipeline (frames -> lists -> permanent field -> PCG -> energies/forces).
//
// One context = one device, one stream.  Everything between amg_set_coords
// and the result copy stays on the device; the PCG convergence test reads
// two FP64 scalars per iteration.
#include "../../include/amoeba_gpu.h"
#include "kernels_setup.cuh"
#include "kernels_pme.cuh"
#include "kernels_pair.cuh"
#include "kernels_misc.cuh"
#include "kernels_adjoint.cuh"
#include "kernels_cp.cuh"

#include <cub/device/device_radix_sort.cuh>
#include <cufft.h>

#include <algorithm>
#include <climits>
#include <initializer_list>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

using namespace amg;

namespace {

constexpr int kOrder = 5;        // B-spline order compiled in (pme.h bseorder default)
constexpr int kGatherLanes = 8;  // lanes per site in the PME derivative gathers
constexpr int kThreads = 128;
constexpr int kRbChunks = 8;  // pieces of the gradient read-back
// FP64 accumulators (eacc): em real 0, einter 1, em reciprocal 2, net charge
// 3, ep 4; the virial's six sums (xx yy zz xy xz yz) of em from kVir and of
// ep from kVirP
constexpr int kVir = 8;
constexpr int kVirP = 14;
constexpr int kEacc = 20;

inline unsigned nblk(size_t n, int t = kThreads) { return (unsigned)((n + t - 1) / t); }

// lanes per site of the bulk pair kernels (runtime choice among compiled 8/16/32)
#define LPA_DISPATCH(lpa, ...)                      \
    do {                                            \
        if ((lpa) == 32) {                          \
            constexpr int L = 32;                   \
            __VA_ARGS__                             \
        } else if ((lpa) == 16) {                   \
            constexpr int L = 16;                   \
            __VA_ARGS__                             \
        } else {                                    \
            constexpr int L = 8;                    \
            __VA_ARGS__                             \
        }                                           \
    } while (0)

template <class R>
struct CufftTypes;
template <>
struct CufftTypes<float> {
    static constexpr cufftType r2c = CUFFT_R2C, c2r = CUFFT_C2R, c2c = CUFFT_C2C;
    static cufftResult fwd(cufftHandle p, float* i, cufftComplex* o) { return cufftExecR2C(p, i, o); }
    static cufftResult inv(cufftHandle p, cufftComplex* i, float* o) { return cufftExecC2R(p, i, o); }
    static cufftResult cc(cufftHandle p, cufftComplex* g, int dir) { return cufftExecC2C(p, g, g, dir); }
    using C = cufftComplex;
};
template <>
struct CufftTypes<double> {
    static constexpr cufftType r2c = CUFFT_D2Z, c2r = CUFFT_Z2D, c2c = CUFFT_Z2Z;
    static cufftResult fwd(cufftHandle p, double* i, cufftDoubleComplex* o) { return cufftExecD2Z(p, i, o); }
    static cufftResult inv(cufftHandle p, cufftDoubleComplex* i, double* o) { return cufftExecZ2D(p, i, o); }
    static cufftResult cc(cufftHandle p, cufftDoubleComplex* g, int dir) { return cufftExecZ2Z(p, g, g, dir); }
    using C = cufftDoubleComplex;
};

template <class R>
struct Pme {
    bool ready = false;
    R* grid = nullptr;                       // [2][K1 K2 K3] spreading grids (kept zeroed)
    R* phig = nullptr;                       // [2][K1 K2 K3] convolved potential grids
    typename CufftTypes<R>::C* cgrid = nullptr;  // [2][K1 K2 (K3/2+1)]
    R* infl = nullptr;                       // [K1 K2 (K3/2+1)]
    R* theta = nullptr;                      // [n][3][4][P]
    int* k0 = nullptr;                       // [n][3]
    cufftHandle f1 = 0, i1 = 0, zplan = 0;
    // dipole grids: d + i p interleaved, transformed in place
    typename Cplx<R>::type* zg = nullptr;    // [K1 K2 K3] spreading grid, zero between uses
    typename Cplx<R>::type* zq = nullptr;    // [K1 K2 K3] convolved potentials (d + i p)
    R* Gfull = nullptr;                      // [K1 K2 K3] influence function on the full grid
    double infl_box[6] = {0, 0, 0, 0, 0, 0};
    size_t G = 0, Gc = 0;
};

template <class R>
struct Atoms {
    AtomR<R>* at = nullptr;
    AtomR<R>* atS = nullptr;  // the same sites in cell order (gathered each evaluation after the sort)
    R4<R>* u4 = nullptr;  // [n][2] dipoles
    R4<R>* p4 = nullptr;  // [n][2] PCG directions
    R4<R>* s4 = nullptr;  // [n][2] alpha r, input of the sparse preconditioner
    R4<R>* c0 = nullptr;  // [n][cap] stored T coefficients (pack_tensor)
    R4<R>* cu0 = nullptr; // [n][cap] sparse preconditioner coefficients (pack_tensor), rows nbru
    int cap = 0;
};

}  // namespace

struct amg_ctx {
    // configuration
    int n = 0, prec = AMG_PREC_MIXED, poltyp = AMG_POL_NONE, politer = 100, guess = 1, device = 0;
    bool ewald = false, bounds = false, has_pol = false;
    double aewald = 0, cut = 0, f = 0, debye = 4.80321, poleps = 1e-6;
    int K[3] = {0, 0, 0}, order = kOrder;
    std::string err;
    double box[6] = {0, 0, 0, 90, 90, 90};
    int cell_shape = AMG_CELL_FROM_ANGLES;  // amg_params cell_shape
    // PME lattice transform (grid units per Cartesian axis) and cell volume
    Frac frac{};
    double vol = 0;
    double latA[3][3] = {}, latR[3][3] = {};  // lattice rows and their inverse (non-orthogonal cells)
    Box bx{};
    bool have_coords = false;
    int nsp = 0;
    // device, persistent
    double *pole13 = nullptr, *pol = nullptr, *thole = nullptr, *pdamp = nullptr, *xyz = nullptr, *rp10 = nullptr;
    int *zax = nullptr, *xax = nullptr, *yax = nullptr, *axe = nullptr, *mol = nullptr;
    ScaledPair* sp = nullptr;
    int *xoff = nullptr, *xidx = nullptr;  // scaled partners of each atom (CSR)
    int2* xrange = nullptr;                // smallest and largest scaled-partner index of each atom
    Atoms<float> af;
    Atoms<double> ad;
    // cell list / neighbour list
    unsigned *keys = nullptr, *skeys = nullptr;
    int *ids = nullptr, *sids = nullptr, *cstart = nullptr, *cend = nullptr;
    size_t ncell_alloc = 0;
    char* cubtmp = nullptr;
    size_t cubtmp_bytes = 0;
    int* nbr = nullptr;
    int* nnb = nullptr;
    int* rank = nullptr;  // position of each site in cell order (inverse of sids)
    int* cnb = nullptr;   // [n][cap] cell-order positions of the PCG coefficient rows' neighbours
    double2* sdt = nullptr;  // (pdamp, thole) in cell order, for the FP64 sweep
    int cap = 0, lpa = 16, num_sms = 148;
    int* overflow = nullptr;
    // sparse PCG preconditioner (pcgprec): rows of the pairs within usolvcut,
    // a subset of the neighbour rows, so they share the capacity cap
    bool sparse_prec = false;
    double usolvcut = 0;
    int *nbru = nullptr, *nnbu = nullptr;
    int capu = 0;
    double4* spos = nullptr;  // coordinates in cell order
    // vectors
    double *Ed = nullptr, *Ep = nullptr, *ud = nullptr, *up = nullptr, *rd = nullptr, *rp = nullptr, *zd = nullptr,
           *zp = nullptr, *pd = nullptr, *pp = nullptr, *Apd = nullptr, *App = nullptr, *Fd = nullptr, *Fp = nullptr,
           *resd = nullptr;
    double *scal = nullptr, *eacc = nullptr;  // eacc: [kEacc]
    bool want_vir = false;                    // this evaluation adds the virial (eacc + kVir, + kVirP)
    bool have_vir = false;
    double vir_parts[2][9] = {};              // last evaluation's virial: em part, ep part
    unsigned long long* cnt = nullptr;
    double *grad_m = nullptr, *grad_p = nullptr, *trq_m = nullptr, *trq_p = nullptr, *aem = nullptr,
           *aep = nullptr;
    double *phiM = nullptr, *phiU = nullptr, *phiU4 = nullptr;
    Pme<float> pmf;
    Pme<double> pmd;
    cudaStream_t st = nullptr, st2 = nullptr;
    // side streams: real-space pair kernels run there while the PME chain
    // runs on the main stream; side[0] pairs with st, side[1] with st2 (the
    // PCG loop body is captured on st2 into its own graph); side[kMpoleSide]
    // carries the permanent-multipole forces from the end of the front to
    // the end of the back, beside the dipole solve
    cudaStream_t side[3] = {nullptr, nullptr, nullptr};
    cudaEvent_t efork[3] = {}, ejoin[3] = {};
    cudaEvent_t erot = nullptr;  // rotated multipoles ready (the list build starts before them)
    cudaEvent_t ev[6] = {};
    CellGrid cg{};
    double cell_volume = 1.0;
    int npolar = 0;
    int *iter = nullptr, *cont = nullptr;
    int* blk_done = nullptr;  // last-block counter of k_precond and k_pcg_update (back to 0 after every launch)
    // OPT: order, copm_k = sum_{j>=k} copt_j, and the perturbation orders
    // u^(k) [K+1][2][3n] followed by one [3n] scratch vector
    int optorder = 0;
    OptCoef copm{};
    double* uopt = nullptr;
    // captured evaluation (periodic systems)
    bool use_graphs = true, graph_dirty = true, graphed_last = false;
    cudaGraphExec_t gexec = nullptr;
    // the adjoint solve captured the same way (set-up, conditional WHILE
    // node, sweep); recaptured after every capture of the forward (fwd_gen)
    cudaGraphExec_t adj_gexec = nullptr;
    long long fwd_gen = 0, adj_gen = -1;
    int gflags = -1;
    // kernel launches of this library: counter, and per captured graph the
    // launches outside the PCG loop and per loop iteration
    long long kcount = 0, kmain = 0, kbody = 0, klast = 0;
    char* flushbuf = nullptr;
    // pinned host staging of one evaluation's read-back (status, scalars,
    // gradients), filled by asynchronous copies behind one synchronisation
    struct Readback {
        int over, iters, over_m;
        double e[kEacc];
        unsigned long long c[4];
        double hs[NSCAL];
    };
    Readback* rb = nullptr;
    double* rb_grad = nullptr;  // [2][3n]
    cudaEvent_t rbev[1 + kRbChunks] = {};  // scalars read back, then each gradient piece
    // the permanent-multipole gradient, read back on its own stream while the
    // solve still runs: gm_ready is recorded when the force stream is done
    // (an external event node in the captured graph), rbevm per piece
    cudaStream_t rbst = nullptr;
    cudaEvent_t gm_ready = nullptr;
    cudaEvent_t rbevm[kRbChunks] = {};
    size_t flush_bytes = 0;
    // adjoint buffers (allocated on the first amg_backward)
    double *adj = nullptr;       // [3n] x 11 vectors: gd gp wd wp bd bp vbar mwp grad trq zero
    double *adj_pot = nullptr;   // [n][10]
    double *adj_n = nullptr;     // [n] x 4: dpd dth dpol zero-pad
    double4* adj_vec = nullptr;  // [n][5]
    double* adj_phi = nullptr;   // [3][2][n][20]
    double* adj_dpole = nullptr; // [n][13]
    double* adj_opt = nullptr;   // OPT: cotangent orders [K+1][2][3n], then P1, P2 [3n] each
    double* adj_host = nullptr;  // pinned staging [n][25]: cotangents in (6), gradients out (19)
    double qtot = 0;             // net charge of the last forward (Ewald)
    // induced-dipole predictor (amg_set_predictor): history [kPredSteps][2][3n]
    // and its device state (next slot, filled slots)
    int pred = AMG_PRED_NONE;
    PredCoef pred_coef{};
    double* pred_hist = nullptr;
    int* pred_state = nullptr;
    std::string graph_note;
    double timing[5] = {0, 0, 0, 0, 0};
    // last forward state for the adjoint
    bool have_forward = false;
    // charge penetration / charge flux of the multipoles (non-Ewald, no
    // polarization): damping tables, per-site core charges and exponents,
    // the bond and angle terms of the flux, the increments dq and the sites'
    // potentials cfpot of the current evaluation
    bool cp_mode = false, cflux = false;
    CpTables cpt{};
    double *pcore = nullptr, *palpha = nullptr, *dq = nullptr, *cfpot = nullptr;
    int nbond = 0, nangle = 0;
    int2* bonds = nullptr;
    double2* bflux = nullptr;
    int* angles = nullptr;
    double* aflux = nullptr;
};

namespace {

struct Fail {
    int code;
};

#define CK(call)                                                                                   \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess) {                                                                   \
            ctx->err = std::string(#call) + ": " + cudaGetErrorString(e_);                         \
            throw Fail{AMG_ERR_CUDA};                                                              \
        }                                                                                          \
    } while (0)
#define CKFFT(call)                                                                                \
    do {                                                                                           \
        cufftResult r_ = (call);                                                                   \
        if (r_ != CUFFT_SUCCESS) {                                                                 \
            ctx->err = std::string(#call) + ": cufft error " + std::to_string((int)r_);            \
            throw Fail{AMG_ERR_CUDA};                                                              \
        }                                                                                          \
    } while (0)
#define KCHECK()                 \
    do {                         \
        CK(cudaGetLastError());  \
        ctx->kcount++;           \
    } while (0)

template <class T>
void dalloc(amg_ctx* ctx, T*& p, size_t count) {
    if (p) cudaFree(p);
    p = nullptr;
    if (count == 0) count = 1;
    CK(cudaMalloc((void**)&p, sizeof(T) * count));
}
template <class T>
void dfree(T*& p) {
    if (p) cudaFree(p);
    p = nullptr;
}
template <class T>
void upload(amg_ctx* ctx, T*& d, const T* h, size_t count) {
    dalloc(ctx, d, count);
    if (h && count) CK(cudaMemcpy(d, h, sizeof(T) * count, cudaMemcpyHostToDevice));
}

// ------------------------------------------------------------ scaled pairs
// The scaled-pair table: m-scales by 1-2..1-5 (applied in order, a later
// list overwrites, as the reference's exclusion set-up at
// src/md/empole.cpp:224-235); p-scales by 1-n with the intra-group value for
// partners in the same polarization group; d- and u-scales by group
// connectivity ip11..ip14 (polpot.h:18-45 meanings).
std::vector<ScaledPair> build_scaled(const amg_params* P) {
    struct S {
        double m = 1, p = 1, d = 1, u = 1;
    };
    std::vector<ScaledPair> out;
    const amg_list* bonded[4] = {&P->i12, &P->i13, &P->i14, &P->i15};
    const amg_list* groups[4] = {&P->ip11, &P->ip12, &P->ip13, &P->ip14};
    std::vector<int> touched;
    std::vector<S> sc(P->n);
    std::vector<char> mark(P->n, 0), ingrp(P->n, 0);
    for (int i = 0; i < P->n; i++) {
        touched.clear();
        if (P->ip11.offsets)
            for (int j = P->ip11.offsets[i]; j < P->ip11.offsets[i + 1]; j++) ingrp[P->ip11.indices[j]] = 1;
        auto touch = [&](int k) {
            if (!mark[k]) {
                mark[k] = 1;
                touched.push_back(k);
                sc[k] = S{};
            }
        };
        for (int b = 0; b < 4; b++) {
            const amg_list& L = *bonded[b];
            if (!L.offsets) continue;
            for (int j = L.offsets[i]; j < L.offsets[i + 1]; j++) {
                int k = L.indices[j];
                if (k == i) continue;
                touch(k);
                sc[k].m = P->m_scale[b];
                sc[k].p = ingrp[k] ? P->p_iscale[b] : P->p_scale[b];
            }
        }
        if (P->polarity)
            for (int g = 0; g < 4; g++) {
                const amg_list& L = *groups[g];
                if (!L.offsets) continue;
                for (int j = L.offsets[i]; j < L.offsets[i + 1]; j++) {
                    int k = L.indices[j];
                    if (k == i) continue;
                    touch(k);
                    sc[k].d = P->d_scale[g];
                    sc[k].u = P->u_scale[g];
                }
            }
        for (int k : touched) {
            mark[k] = 0;
            if (k <= i) continue;
            const S& s = sc[k];
            if (s.m != 1 || s.p != 1 || s.d != 1 || s.u != 1) out.push_back(ScaledPair{i, k, 0, 0, s.m, s.p, s.d, s.u});
        }
        if (P->ip11.offsets)
            for (int j = P->ip11.offsets[i]; j < P->ip11.offsets[i + 1]; j++) ingrp[P->ip11.indices[j]] = 0;
    }
    return out;
}

// ------------------------------------------------------------ PME set-up
void bsmod_axis(int K, int p, std::vector<double>& out) {
    // |sum_{k=0}^{p-2} M_p(k+1) e^{2 pi i m k / K}|^2, zeros (odd p at the
    // Nyquist frequency) replaced by the mean of the neighbours
    std::vector<double> Mp(p + 1, 0.0);
    {
        // cardinal B-spline values at integers 1..p-1 by the order recursion
        std::vector<double> b(p + 1, 0.0), nb(p + 1, 0.0);
        b[1] = 1.0;  // M_2(1) = 1 (values at x = 0..n)
        int order = 2;
        // M_n(x) at integer x: M_n(x) = (x M_{n-1}(x) + (n - x) M_{n-1}(x-1)) / (n-1)
        while (order < p) {
            order++;
            std::fill(nb.begin(), nb.end(), 0.0);
            for (int x = 1; x < order; x++) nb[x] = (x * b[x] + (order - x) * b[x - 1]) / (order - 1);
            b = nb;
        }
        for (int x = 0; x <= p; x++) Mp[x] = b[x];
    }
    out.assign(K, 0.0);
    for (int m = 0; m < K; m++) {
        double re = 0, im = 0;
        for (int k = 0; k <= p - 2; k++) {
            double ang = 2 * kPi * m * k / K;
            re += Mp[k + 1] * cos(ang);
            im += Mp[k + 1] * sin(ang);
        }
        out[m] = re * re + im * im;
    }
    for (int m = 0; m < K; m++)
        if (out[m] < 1e-7) out[m] = 0.5 * (out[(m - 1 + K) % K] + out[(m + 1) % K]);
}

template <class R>
void pme_prepare(amg_ctx* ctx, Pme<R>& pm) {
    const int K1 = ctx->K[0], K2 = ctx->K[1], K3 = ctx->K[2];
    if (!pm.ready) {
        pm.G = (size_t)K1 * K2 * K3;
        pm.Gc = (size_t)K1 * K2 * (K3 / 2 + 1);
        dalloc(ctx, pm.grid, 2 * pm.G);
        dalloc(ctx, pm.phig, 2 * pm.G);
        CK(cudaMemset(pm.grid, 0, sizeof(R) * 2 * pm.G));
        dalloc(ctx, pm.cgrid, 2 * pm.Gc);
        dalloc(ctx, pm.infl, pm.Gc);
        dalloc(ctx, pm.theta, (size_t)ctx->n * 3 * 4 * kOrder);
        dalloc(ctx, pm.k0, (size_t)ctx->n * 3);
        int dims[3] = {K1, K2, K3};
        CKFFT(cufftPlanMany(&pm.f1, 3, dims, nullptr, 1, 0, nullptr, 1, 0, CufftTypes<R>::r2c, 1));
        CKFFT(cufftPlanMany(&pm.i1, 3, dims, nullptr, 1, 0, nullptr, 1, 0, CufftTypes<R>::c2r, 1));
        cufftHandle hs[2] = {pm.f1, pm.i1};
        for (int k = 0; k < 2; k++) CKFFT(cufftSetStream(hs[k], ctx->st));
        dalloc(ctx, pm.zg, pm.G);
        dalloc(ctx, pm.zq, pm.G);
        CK(cudaMemset(pm.zg, 0, sizeof(typename Cplx<R>::type) * pm.G));
        dalloc(ctx, pm.Gfull, pm.G);
        // in-place complex transform of the dipole grid (d + i p)
        CKFFT(cufftPlan3d(&pm.zplan, K1, K2, K3, CufftTypes<R>::c2c));
        CKFFT(cufftSetStream(pm.zplan, ctx->st));
        pm.ready = true;
    }
    if (!std::equal(ctx->box, ctx->box + 6, pm.infl_box)) {
        std::vector<double> b1, b2, b3;
        bsmod_axis(K1, kOrder, b1);
        bsmod_axis(K2, kOrder, b2);
        bsmod_axis(K3, kOrder, b3);
        const double V = ctx->vol;
        const double pref = 1.0 / (kPi * V), a2 = ctx->aewald * ctx->aewald;
        const Frac& F = ctx->frac;  // reciprocal vector b_j = (column j of F.m) / K_j
        std::vector<R> h(pm.Gc);
        const int K3h = K3 / 2 + 1;
        for (int a = 0; a < K1; a++)
            for (int b = 0; b < K2; b++)
                for (int c = 0; c < K3h; c++) {
                    size_t id = ((size_t)a * K2 + b) * K3h + c;
                    if (a == 0 && b == 0 && c == 0) { h[id] = 0; continue; }
                    int ma = a <= K1 / 2 ? a : a - K1, mb = b <= K2 / 2 ? b : b - K2, mc = c;
                    const double fa = (double)ma / K1, fb = (double)mb / K2, fc = (double)mc / K3;
                    double hx = F.m[0][0] * fa + F.m[0][1] * fb + F.m[0][2] * fc;
                    double hy = F.m[1][0] * fa + F.m[1][1] * fb + F.m[1][2] * fc;
                    double hz = F.m[2][0] * fa + F.m[2][1] * fb + F.m[2][2] * fc;
                    if (!F.general) { hx = ma / ctx->box[0]; hy = mb / ctx->box[1]; hz = mc / ctx->box[2]; }
                    double h2 = hx * hx + hy * hy + hz * hz;
                    h[id] = (R)(pref * exp(-kPi * kPi * h2 / a2) / h2 / (b1[a] * b2[b] * b3[c]));
                    // octahedron and dodecahedron: the cell's lattice is the
                    // prism's plus its body-centring translation (half of every
                    // edge), so its reciprocal vectors are the prism's with an
                    // even index sum; the others cancel between the two halves
                    if (ctx->bx.shape >= 3 && ((ma + mb + mc) & 1)) h[id] = 0;
                }
        CK(cudaMemcpy(pm.infl, h.data(), sizeof(R) * pm.Gc, cudaMemcpyHostToDevice));
        // the same function on the full grid (even: G(m) = G(-m))
        std::vector<R> hf(pm.G);
        for (int a = 0; a < K1; a++)
            for (int b = 0; b < K2; b++)
                for (int c = 0; c < K3; c++) {
                    const int a2 = a == 0 ? 0 : K1 - a, b2 = b == 0 ? 0 : K2 - b;
                    // c > K3/2: G(a,b,c) = G(-a,-b,K3-c), held in the half-complex layout
                    hf[((size_t)a * K2 + b) * K3 + c] =
                        c < K3h ? h[((size_t)a * K2 + b) * K3h + c] : h[((size_t)a2 * K2 + b2) * K3h + (K3 - c)];
                }
        CK(cudaMemcpy(pm.Gfull, hf.data(), sizeof(R) * pm.G, cudaMemcpyHostToDevice));
        std::copy(ctx->box, ctx->box + 6, pm.infl_box);
    }
}

template <class R>
void pme_destroy(Pme<R>& pm) {
    cufftHandle* hs[3] = {&pm.f1, &pm.i1, &pm.zplan};
    for (int k = 0; k < 3; k++)
        if (*hs[k]) { cufftDestroy(*hs[k]); *hs[k] = 0; }
    dfree(pm.zg); dfree(pm.zq); dfree(pm.Gfull);
    dfree(pm.grid); dfree(pm.phig); dfree(pm.cgrid); dfree(pm.infl); dfree(pm.theta); dfree(pm.k0);
    pm.ready = false;
}

template <class R>
Atoms<R>& atoms_of(amg_ctx* ctx);
template <>
Atoms<float>& atoms_of<float>(amg_ctx* ctx) { return ctx->af; }
template <>
Atoms<double>& atoms_of<double>(amg_ctx* ctx) { return ctx->ad; }
template <class R>
Pme<R>& pme_of(amg_ctx* ctx);
template <>
Pme<float>& pme_of<float>(amg_ctx* ctx) { return ctx->pmf; }
template <>
Pme<double>& pme_of<double>(amg_ctx* ctx) { return ctx->pmd; }

// ------------------------------------------------------------ pipeline
template <class R>
void rotate_and_pack(amg_ctx* ctx, cudaStream_t s) {
    Atoms<R>& A = atoms_of<R>(ctx);
    k_rotate<R><<<nblk(ctx->n), kThreads, 0, s>>>(ctx->n, ctx->xyz, ctx->pole13, ctx->zax, ctx->xax, ctx->yax,
                                                  ctx->axe, ctx->has_pol ? ctx->pdamp : nullptr,
                                                  ctx->has_pol ? ctx->thole : nullptr,
                                                  ctx->has_pol ? ctx->pol : nullptr, ctx->cflux ? ctx->dq : nullptr,
                                                  ctx->rp10, A.at);
    KCHECK();
}

// Cell grid for the current box (periodic) or coordinate bounding box
// (non-periodic), computed on the host when coordinates are set.
// Cell shape and lattice terms of a periodic box (src/md/lattice.cpp:36-110
// restated): truncated octahedron and rhombic dodecahedron by the context's
// cell_shape (right angles required), else orthogonal / monoclinic (only beta
// off 90) / triclinic by the angles.
bool set_lattice(amg_ctx* ctx, const double box[6], Box& b) {
    const bool right = box[3] == 90.0 && box[4] == 90.0 && box[5] == 90.0;
    b.shape = 0;
    b.bsin = 1; b.bcos = 0; b.gsin = 1; b.gcos = 0; b.bterm = 0; b.gterm = 1;
    if (ctx->cell_shape != AMG_CELL_FROM_ANGLES) {
        if (!right) {
            ctx->err = "octahedron and dodecahedron cells take right angles";
            return false;
        }
        b.shape = ctx->cell_shape == AMG_CELL_OCTAHEDRON ? 3 : 4;
        return true;
    }
    if (right) return true;
    const double rad = 180.0 / kPi;
    b.bsin = std::sin(box[4] / rad);
    b.bcos = std::cos(box[4] / rad);
    if (box[3] == 90.0 && box[5] == 90.0) {
        b.shape = 1;
        b.gterm = b.bsin;
        return true;
    }
    b.shape = 2;
    b.gsin = std::sin(box[5] / rad);
    b.gcos = std::cos(box[5] / rad);
    b.bterm = (std::cos(box[3] / rad) - b.bcos * b.gcos) / b.gsin;
    const double g2 = b.bsin * b.bsin - b.bterm * b.bterm;
    if (!(g2 > 0)) {
        ctx->err = "box angles do not form a cell";
        return false;
    }
    b.gterm = std::sqrt(g2);
    return true;
}

// Lattice rows (a along x, b in the xy plane; src/md/lattice.cpp:122-140),
// their inverse and the PME transform m[i][j] = inverse[i][j] K_j; for an
// orthogonal box m = diag(K/L) exactly as the orthogonal kernels scale.
void set_frac(amg_ctx* ctx) {
    const Box& b = ctx->bx;
    Frac& F = ctx->frac;
    F = Frac{};
    if (b.shape == 0) {
        for (int a = 0; a < 3; a++) F.m[a][a] = ctx->K[a] / ctx->box[a];
        ctx->vol = ctx->box[0] * ctx->box[1] * ctx->box[2];
        return;
    }
    double A[3][3] = {}, R[3][3] = {};
    A[0][0] = ctx->box[0];
    A[1][0] = ctx->box[1] * b.gcos;
    A[1][1] = ctx->box[1] * b.gsin;
    A[2][0] = ctx->box[2] * b.bcos;
    A[2][1] = ctx->box[2] * b.bterm;
    A[2][2] = ctx->box[2] * b.gterm;
    // truncated octahedron and rhombic dodecahedron: the PME grid spans the
    // enclosing prism (a cube; L x L x sqrt(2) L for the dodecahedron, whose
    // image wraps z by sqrt(2) L, src/md/image.cpp:109-121) and the cell is
    // half of it
    if (b.shape == 4) A[2][2] *= kSqrt2;
    R[0][0] = 1 / A[0][0];
    R[1][1] = 1 / A[1][1];
    R[2][2] = 1 / A[2][2];
    R[1][0] = -A[1][0] * R[0][0] / A[1][1];
    R[2][1] = -A[2][1] * R[1][1] / A[2][2];
    R[2][0] = -(A[2][0] * R[0][0] + A[2][1] * R[1][0]) / A[2][2];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            F.m[i][j] = R[i][j] * ctx->K[j];
            ctx->latA[i][j] = A[i][j];
            ctx->latR[i][j] = R[i][j];
        }
    F.general = 1;
    ctx->vol = A[0][0] * A[1][1] * A[2][2] * (b.shape >= 3 ? 0.5 : 1.0);
}

// Cell grid of the neighbour-list build.  A non-orthogonal cell is one cell
// with every atom a candidate of every other (the minimum image decides);
// the orthogonal box and open systems get cells of at least the cutoff.
void cell_grid(amg_ctx* ctx, const double* hxyz) {
    CellGrid& cg = ctx->cg;
    cg = CellGrid{};
    cg.periodic = ctx->bounds;
    if (ctx->bounds && ctx->bx.shape != 0) {
        const Box& b = ctx->bx;
        double vol = ctx->box[0] * ctx->box[1] * ctx->box[2];
        vol *= b.shape == 1 ? b.bsin : b.shape == 2 ? b.gsin * b.gterm : b.shape == 3 ? 0.5 : 0.5 * kSqrt2;
        ctx->cell_volume = vol;
        for (int a = 0; a < 3; a++) {
            cg.nc[a] = 1;
            cg.size[a] = ctx->box[a];
        }
        if (b.shape <= 2) {
            // monoclinic / triclinic: the lattice's parallelepipeds, as many
            // per axis as fit with a width (the distance between the cell's
            // faces, V / |A_b x A_c| per lattice step) of at least the cutoff;
            // with 3 or more on every axis the 27 cells around a cell hold
            // every atom within the cutoff of it
            const double(&A)[3][3] = ctx->latA;
            auto width = [&](int a) {
                const int b1 = (a + 1) % 3, b2 = (a + 2) % 3;
                const double cx = A[b1][1] * A[b2][2] - A[b1][2] * A[b2][1];
                const double cy = A[b1][2] * A[b2][0] - A[b1][0] * A[b2][2];
                const double cz = A[b1][0] * A[b2][1] - A[b1][1] * A[b2][0];
                return vol / std::sqrt(cx * cx + cy * cy + cz * cz);
            };
            int nc[3];
            for (int a = 0; a < 3; a++) nc[a] = std::max(1, std::min(256, (int)std::floor(width(a) / ctx->cut)));
            if (nc[0] >= 3 && nc[1] >= 3 && nc[2] >= 3) {
                cg.general = 1;
                for (int a = 0; a < 3; a++) {
                    cg.nc[a] = nc[a];
                    cg.off_lo[a] = -1;
                    cg.off_hi[a] = 1;
                    for (int c = 0; c < 3; c++) {
                        cg.A[a][c] = A[a][c];
                        cg.R[a][c] = ctx->latR[a][c];
                    }
                }
            }
        }
        if (b.shape >= 3) {
            // truncated octahedron / rhombic dodecahedron (equal box lengths):
            // the lattice is the enclosing prism's (L, L, L; or L, L, sqrt(2) L)
            // plus half of every edge, so the cells of the prism with an even
            // count of at least 6 per axis, and the stencil around the home
            // cell plus the one half a prism away, hold every atom within the
            // cutoff (k_neighbors_cells<false, true>)
            const double L = ctx->box[0];
            const bool equal = std::fabs(ctx->box[1] - L) <= 1e-12 * L && std::fabs(ctx->box[2] - L) <= 1e-12 * L;
            const double P[3] = {L, L, b.shape == 4 ? kSqrt2 * L : L};
            int nc[3];
            for (int a = 0; a < 3; a++) nc[a] = std::min(256, (int)std::floor(P[a] / ctx->cut)) & ~1;
            if (equal && nc[0] >= 6 && nc[1] >= 6 && nc[2] >= 6) {
                cg.centred = 1;
                for (int a = 0; a < 3; a++) {
                    cg.nc[a] = nc[a];
                    cg.size[a] = P[a] / nc[a];
                    cg.off_lo[a] = -1;
                    cg.off_hi[a] = 1;
                }
            }
        }
        return;
    }
    double lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
    if (!ctx->bounds) {
        for (int a = 0; a < 3; a++) { lo[a] = 1e300; hi[a] = -1e300; }
        for (int i = 0; i < ctx->n; i++)
            for (int a = 0; a < 3; a++) {
                lo[a] = std::min(lo[a], hxyz[3 * i + a]);
                hi[a] = std::max(hi[a], hxyz[3 * i + a]);
            }
    }
    double vol = 1.0;
    for (int a = 0; a < 3; a++) {
        if (ctx->bounds) {
            double L = ctx->box[a];
            cg.nc[a] = std::max(1, (int)std::floor(L / ctx->cut));
            cg.size[a] = L / cg.nc[a];
            vol *= L;
            if (cg.nc[a] >= 3) { cg.off_lo[a] = -1; cg.off_hi[a] = 1; }
            else if (cg.nc[a] == 2) { cg.off_lo[a] = 0; cg.off_hi[a] = 1; }
            else { cg.off_lo[a] = 0; cg.off_hi[a] = 0; }
        } else {
            double ext = hi[a] - lo[a] + 1e-6;
            cg.nc[a] = std::max(1, std::min(128, (int)std::floor(ext / ctx->cut)));
            cg.size[a] = ext / cg.nc[a];
            cg.origin[a] = lo[a];
            vol *= std::max(ext, 1.0);
            cg.off_lo[a] = -1;
            cg.off_hi[a] = 1;
        }
    }
    ctx->cell_volume = vol;
}

template <class R>
void ensure_coeff_buffers(amg_ctx* ctx, Atoms<R>& A) {
    if (ctx->sparse_prec && ctx->capu != ctx->cap) {
        dalloc(ctx, ctx->nbru, (size_t)ctx->cap * ctx->n);
        if (!ctx->nnbu) dalloc(ctx, ctx->nnbu, ctx->n);
        ctx->capu = ctx->cap;
        ctx->graph_dirty = true;
    }
    if (A.cap == ctx->cap && A.c0) return;
    dalloc(ctx, A.c0, (size_t)ctx->cap * ctx->n);
    if (ctx->sparse_prec) {
        dalloc(ctx, A.cu0, (size_t)ctx->cap * ctx->n);
        if (!A.s4) {
            dalloc(ctx, A.s4, 2 * (size_t)ctx->n);
            CK(cudaMemset(A.s4, 0, sizeof(R4<R>) * 2 * (size_t)ctx->n));  // the w words stay zero
        }
    }
    A.cap = ctx->cap;
    ctx->graph_dirty = true;
}

void ensure_list_buffers(amg_ctx* ctx) {
    const int n = ctx->n;
    size_t ncell = (size_t)ctx->cg.nc[0] * ctx->cg.nc[1] * ctx->cg.nc[2];
    if (ncell > ctx->ncell_alloc) {
        dalloc(ctx, ctx->cstart, ncell);
        dalloc(ctx, ctx->cend, ncell);
        ctx->ncell_alloc = ncell;
        ctx->graph_dirty = true;
    }
    if (!ctx->keys) {
        dalloc(ctx, ctx->keys, n);
        dalloc(ctx, ctx->skeys, n);
        dalloc(ctx, ctx->ids, n);
        dalloc(ctx, ctx->sids, n);
        dalloc(ctx, ctx->nnb, n);
        dalloc(ctx, ctx->overflow, 1);
        dalloc(ctx, ctx->spos, n);
        dalloc(ctx, ctx->rank, n);
        dalloc(ctx, ctx->sdt, n);
        size_t bytes = 0;
        cub::DeviceRadixSort::SortPairs(nullptr, bytes, ctx->keys, ctx->skeys, ctx->ids, ctx->sids, n);
        dalloc(ctx, ctx->cubtmp, bytes);
        ctx->cubtmp_bytes = bytes;
    }
    if (ctx->cap == 0) {
        double rho = n / ctx->cell_volume;
        int nx = 0;
        {
            std::vector<int> off(n + 1);
            CK(cudaMemcpy(off.data(), ctx->xoff, sizeof(int) * (n + 1), cudaMemcpyDeviceToHost));
            for (int i = 0; i < n; i++) nx = std::max(nx, off[i + 1] - off[i]);
        }
        double est = 4.0 / 3.0 * kPi * ctx->cut * ctx->cut * ctx->cut * rho;
        int cap = (int)std::min<double>(n - 1 + nx, std::ceil(1.4 * est) + 64 + nx);
        ctx->cap = std::max(cap, 1);
        dalloc(ctx, ctx->nbr, (size_t)ctx->cap * n);
        dalloc(ctx, ctx->cnb, (size_t)ctx->cap * n);
        ctx->graph_dirty = true;
    }
}

// cell binning (CUB radix sort on the cell key) and the exact lists; an
// overflow of the per-atom capacity is flagged on the device and handled by
// the caller after the evaluation (grow and evaluate again)
void enqueue_lists(amg_ctx* ctx, cudaStream_t s) {
    const int n = ctx->n;
    const CellGrid& cg = ctx->cg;
    size_t ncell = (size_t)cg.nc[0] * cg.nc[1] * cg.nc[2];
    int nbits = 1;
    while ((1ull << nbits) < ncell) nbits++;
    k_zero<int><<<nblk(ncell, 256), 256, 0, s>>>(ctx->cstart, ncell);
    KCHECK();
    k_zero<int><<<nblk(ncell, 256), 256, 0, s>>>(ctx->cend, ncell);
    KCHECK();
    k_cell_index<<<nblk(n), kThreads, 0, s>>>(n, ctx->xyz, cg, ctx->bx, ctx->keys, ctx->ids);
    KCHECK();
    size_t bytes = ctx->cubtmp_bytes;
    CK(cub::DeviceRadixSort::SortPairs(ctx->cubtmp, bytes, ctx->keys, ctx->skeys, ctx->ids, ctx->sids, n, 0, nbits, s));
    k_cell_bounds<<<nblk(n), kThreads, 0, s>>>(n, ctx->skeys, ctx->sids, ctx->xyz, ctx->cstart, ctx->cend, ctx->spos,
                                               ctx->rank, ctx->pdamp, ctx->thole,
                                               ctx->has_pol ? ctx->sdt : nullptr);
    KCHECK();
    const double cut2 = ctx->cut * ctx->cut;
    if (!cg.periodic || (cg.nc[0] >= 3 && cg.nc[1] >= 3 && cg.nc[2] >= 3)) {
        // block per cell, stencil staged in shared memory; FP32 test with an
        // FP64 decision within 1e-3 cut^2 of the cutoff
        // (monoclinic and triclinic cells: parallelepiped cells, every pair
        // decided by the FP64 image of the cell)
        auto kern = cg.general ? k_neighbors_cells<true> : cg.centred ? k_neighbors_cells<false, true>
                                                                      : k_neighbors_cells<false>;
        kern<<<(unsigned)ncell, kNbrThreads, 0, s>>>(ctx->spos, ctx->sids, ctx->cstart, ctx->cend, cg, ctx->bx, cut2,
                                                     1e-3 * cut2, ctx->cap, ctx->xoff, ctx->xidx, ctx->xrange, ctx->nbr,
                                                     ctx->cnb, ctx->nnb, ctx->overflow);
    } else {
        k_neighbors<<<nblk((size_t)n * 32), kThreads, 0, s>>>(n, ctx->spos, ctx->skeys, ctx->sids, ctx->cstart,
                                                              ctx->cend, cg, ctx->bx, cut2, ctx->cap, ctx->xoff,
                                                              ctx->xidx, ctx->xrange, ctx->nbr, ctx->cnb, ctx->nnb, ctx->overflow);
    }
    KCHECK();
}

// Fork: the side stream of s starts after everything enqueued on s so far.
// Join: s continues only after everything enqueued on the side stream.
// Under stream capture these become graph edges.
int side_index(const amg_ctx* ctx, cudaStream_t s) { return s == ctx->st2 ? 1 : 0; }

cudaStream_t fork_side(amg_ctx* ctx, cudaStream_t s) {
    const int k = side_index(ctx, s);
    CK(cudaEventRecord(ctx->efork[k], s));
    CK(cudaStreamWaitEvent(ctx->side[k], ctx->efork[k], 0));
    return ctx->side[k];
}

void join_side(amg_ctx* ctx, cudaStream_t s) {
    const int k = side_index(ctx, s);
    CK(cudaEventRecord(ctx->ejoin[k], ctx->side[k]));
    CK(cudaStreamWaitEvent(s, ctx->ejoin[k], 0));
}

// the permanent-multipole force stream, forked from and joined to st
constexpr int kMpoleSide = 2;
cudaStream_t fork_mpole(amg_ctx* ctx, cudaStream_t s) {
    CK(cudaEventRecord(ctx->efork[kMpoleSide], s));
    CK(cudaStreamWaitEvent(ctx->side[kMpoleSide], ctx->efork[kMpoleSide], 0));
    return ctx->side[kMpoleSide];
}
void join_mpole(amg_ctx* ctx, cudaStream_t s) {
    CK(cudaEventRecord(ctx->ejoin[kMpoleSide], ctx->side[kMpoleSide]));
    CK(cudaStreamWaitEvent(s, ctx->ejoin[kMpoleSide], 0));
}

// B-spline stencils of every site
template <class R>
void pme_stencils(amg_ctx* ctx, cudaStream_t s, bool with_fp64 = false) {
    // the FP64 stencils, the FP32 ones, or (a mixed-precision solve with its
    // FP64 correction sweep) both from one pass
    constexpr int BS = 64;
    const unsigned blocks = (unsigned)((ctx->n + BS - 1) / BS);
    const int3 K = make_int3(ctx->K[0], ctx->K[1], ctx->K[2]);
    if constexpr (sizeof(R) == 8) {
        Pme<double>& pd = pme_of<double>(ctx);
        k_bspline_rows<kOrder, BS, true, false><<<blocks, BS, 0, s>>>(ctx->n, ctx->xyz, ctx->bx, ctx->frac, K, pd.theta,
                                                                      pd.k0, nullptr, nullptr);
    } else if (with_fp64) {
        Pme<double>& pd = pme_of<double>(ctx);
        Pme<float>& pf = pme_of<float>(ctx);
        k_bspline_rows<kOrder, BS, true, true><<<blocks, BS, 0, s>>>(ctx->n, ctx->xyz, ctx->bx, ctx->frac, K, pd.theta,
                                                                     pd.k0, pf.theta, pf.k0);
    } else {
        Pme<float>& pf = pme_of<float>(ctx);
        k_bspline_rows<kOrder, BS, false, true><<<blocks, BS, 0, s>>>(ctx->n, ctx->xyz, ctx->bx, ctx->frac, K, nullptr,
                                                                      nullptr, pf.theta, pf.k0);
    }
    KCHECK();
}

// k-space constant of the reciprocal virial, pi^2/alpha^2
inline double kvir_c2(const amg_ctx* ctx) { return kPi * kPi / (ctx->aewald * ctx->aewald); }

// reciprocal potential derivatives of the permanent multipoles -> phiM [n][20];
// with `vir`, also the k-space part of the permanent virial (six sums) and a
// copy of the grid's transform (second half of cgrid) for the polarization's
template <class R>
void pme_mpole(amg_ctx* ctx, cudaStream_t s, double* vir = nullptr) {
    Pme<R>& pm = pme_of<R>(ctx);
    int3 K = make_int3(ctx->K[0], ctx->K[1], ctx->K[2]);
    k_spread_mpole<R, kOrder><<<nblk(ctx->n), kThreads, 0, s>>>(ctx->n, ctx->rp10, pm.theta, pm.k0, K, ctx->frac,
                                                                pm.grid);
    KCHECK();
    CKFFT(cufftSetStream(pm.f1, s));
    CKFFT(cufftSetStream(pm.i1, s));
    CKFFT(CufftTypes<R>::fwd(pm.f1, pm.grid, pm.cgrid));
    if (vir) {
        using C = typename Cplx<R>::type;
        k_kvir_mpole<R><<<(unsigned)ctx->num_sms * 2, 256, 0, s>>>(pm.Gc, K, ctx->frac, kvir_c2(ctx), ctx->f,
                                                                   pm.infl, (const C*)pm.cgrid,
                                                                   (C*)pm.cgrid + pm.Gc, vir);
        KCHECK();
    }
    k_convolve<R><<<nblk(pm.Gc, 256), 256, 0, s>>>(pm.Gc, 1, pm.infl, (typename Cplx<R>::type*)pm.cgrid, pm.grid, pm.G);
    KCHECK();
    CKFFT(CufftTypes<R>::inv(pm.i1, pm.cgrid, pm.phig));
    k_gather<R, kOrder, 20, kGatherLanes, 1><<<nblk((size_t)ctx->n * kGatherLanes), kThreads, 0, s>>>(
        ctx->n, pm.phig, pm.theta, pm.k0, K, ctx->frac, ctx->phiM);
    KCHECK();
}

// spread two dipole sets into the complex grid pm.zg (d + i p), transform,
// convolve into pm.zq (clearing pm.zg for the next spreading) and transform
// pm.zq back in place.  `spread` false: the grid already holds the spread
// dipoles (the PCG's fused direction update put them there).  The PCG's
// last direction update leaves a spread grid behind, so every other caller
// clears it first.
template <class R>
void spread_dipoles(amg_ctx* ctx, cudaStream_t s, const double* vd, const double* vp) {
    Pme<R>& pm = pme_of<R>(ctx);
    int3 K = make_int3(ctx->K[0], ctx->K[1], ctx->K[2]);
    k_spread_dipoles<R, kOrder><<<spread_blocks<R>(ctx->n), 128, 0, s>>>(ctx->n, ctx->sids, vd, vp, pm.theta, pm.k0,
                                                                          K, ctx->frac,
                                                        pm.zg);
    KCHECK();
}

// `vir`: the k-space part of the polarization virial (six sums), from this
// transform and the permanent one saved by pme_mpole
template <class R>
void pme_dipole_grids(amg_ctx* ctx, cudaStream_t s, const double* vd, const double* vp, bool spread = true,
                      double* vir = nullptr, bool mterms = true, bool clear = true) {
    Pme<R>& pm = pme_of<R>(ctx);
    if (spread) {
        if (clear) CK(cudaMemsetAsync(pm.zg, 0, sizeof(typename Cplx<R>::type) * pm.G, s));
        spread_dipoles<R>(ctx, s, vd, vp);
    }
    CKFFT(cufftSetStream(pm.zplan, s));
    CKFFT(CufftTypes<R>::cc(pm.zplan, pm.zg, CUFFT_FORWARD));
    if (vir) {
        using C = typename Cplx<R>::type;
        k_kvir_polar<R><<<(unsigned)ctx->num_sms * 2, 256, 0, s>>>(
            pm.G, make_int3(ctx->K[0], ctx->K[1], ctx->K[2]), ctx->frac, kvir_c2(ctx), ctx->f,
            mterms ? ctx->poltyp == AMG_POL_MUTUAL : 1, mterms, pm.Gfull, pm.zg, (const C*)pm.cgrid + pm.Gc, vir);
        KCHECK();
    }
    k_scale_grid<R><<<nblk(pm.G, 256), 256, 0, s>>>(pm.G, pm.Gfull, pm.zg, pm.zq);  // also clears zg
    KCHECK();
    CKFFT(CufftTypes<R>::cc(pm.zplan, pm.zq, CUFFT_INVERSE));
}

// reciprocal potentials of two dipole sets -> phi [2][n][NC]
template <class R, int NC>
void pme_dipoles(amg_ctx* ctx, cudaStream_t s, const double* vd, const double* vp, double* phi,
                 double* vir = nullptr, bool mterms = true) {
    Pme<R>& pm = pme_of<R>(ctx);
    int3 K = make_int3(ctx->K[0], ctx->K[1], ctx->K[2]);
    pme_dipole_grids<R>(ctx, s, vd, vp, true, vir, mterms);
    k_gather<R, kOrder, NC, kGatherLanes, 2><<<nblk((size_t)ctx->n * kGatherLanes), kThreads, 0, s>>>(
        ctx->n, pm.zq, pm.theta, pm.k0, K, ctx->frac, phi);
    KCHECK();
}

double ewald_alpha(const amg_ctx* ctx) { return ctx->ewald ? ctx->aewald : 0.0; }

double self_coef(const amg_ctx* ctx) {
    double a = ctx->aewald;
    return ctx->ewald ? 4.0 * a * a * a / (3.0 * kSqrtPi) : 0.0;
}

// Ewald in a monoclinic or triclinic cell: the pair kernels' CELLS instances
bool ewald_cells(const amg_ctx* ctx) { return ctx->ewald && ctx->bx.shape != 0; }

// A v for both dipole sets (v/alpha - field of v), pair tensors computed on
// the fly (FP64 correction sweep, OPT orders).  `cells` (the sweep, which
// follows a solve and so has the cell-order partner rows cnb): the FP64
// real-space part gathers from cell-order copies (k_Tu_cells).
template <class R>
void matvec(amg_ctx* ctx, cudaStream_t s, const double* vd, const double* vp, double* Ad, double* Ap,
            bool cells = false) {
    const int n = ctx->n;
    Atoms<R>& A = atoms_of<R>(ctx);
    k_pack_u<R><<<nblk(n), kThreads, 0, s>>>(n, vd, vp, A.u4, cells ? ctx->rank : nullptr);
    KCHECK();
    // real space on the side stream, PME on s
    cudaStream_t r = ctx->ewald ? fork_side(ctx, s) : s;
    if constexpr (sizeof(R) == 8) {
        if (cells) {
            LPA_DISPATCH(ctx->lpa, {
                if (ewald_cells(ctx))
                    k_Tu_cells<true, 8, true><<<nblk((size_t)n * 8), kThreads, 0, r>>>(
                        n, ctx->sids, ctx->spos, ctx->sdt, A.u4, ctx->bx, ctx->aewald, ctx->cnb, ctx->cap, ctx->nnb,
                        ctx->Fd, ctx->Fp);
                else if (ctx->ewald)
                    k_Tu_cells<true, L><<<nblk((size_t)n * L), kThreads, 0, r>>>(
                        n, ctx->sids, ctx->spos, ctx->sdt, A.u4, ctx->bx, ctx->aewald, ctx->cnb, ctx->cap, ctx->nnb,
                        ctx->Fd, ctx->Fp);
                else
                    k_Tu_cells<false, L><<<nblk((size_t)n * L), kThreads, 0, r>>>(
                        n, ctx->sids, ctx->spos, ctx->sdt, A.u4, ctx->bx, 0.0, ctx->cnb, ctx->cap, ctx->nnb, ctx->Fd,
                        ctx->Fp);
            });
        }
    }
    if (!(cells && sizeof(R) == 8)) LPA_DISPATCH(ctx->lpa, {
        if (ewald_cells(ctx))
            k_Tu<R, true, 8, true><<<nblk((size_t)n * 8), kThreads, 0, r>>>(n, ctx->sids, A.at, A.u4, ctx->bx, (R)ctx->aewald,
                                                                            ctx->nbr, ctx->cap, ctx->nnb, ctx->Fd, ctx->Fp);
        else if (ctx->ewald)
            k_Tu<R, true, L><<<nblk((size_t)n * L), kThreads, 0, r>>>(n, ctx->sids, A.at, A.u4, ctx->bx, (R)ctx->aewald, ctx->nbr,
                                                                      ctx->cap, ctx->nnb, ctx->Fd, ctx->Fp);
        else
            k_Tu<R, false, L><<<nblk((size_t)n * L), kThreads, 0, r>>>(n, ctx->sids, A.at, A.u4, ctx->bx, (R)0, ctx->nbr, ctx->cap,
                                                                       ctx->nnb, ctx->Fd, ctx->Fp);
    });
    KCHECK();
    if (ctx->nsp) {
        k_scaled_Tu<<<nblk(ctx->nsp), kThreads, 0, r>>>(ctx->nsp, ctx->sp, ctx->xyz, ctx->pdamp, ctx->thole, ctx->bx,
                                                       ctx->cut * ctx->cut, ewald_alpha(ctx), vd, vp, ctx->Fd, ctx->Fp);
        KCHECK();
    }
    if (ctx->ewald) {
        pme_dipoles<R, 4>(ctx, s, vd, vp, ctx->phiU4);
        join_side(ctx, s);
    }
    k_matvec_finish<<<nblk(n), kThreads, 0, s>>>(n, vd, vp, ctx->Fd, ctx->Fp, ctx->phiU4, ctx->ewald, self_coef(ctx),
                                                 ctx->pol, Ad, Ap);
    KCHECK();
}

// the scaled partners' coefficients in the rows' tails (after the bulk
// pairs, whose counts must be final)
template <class R>
void build_scaled_coeffs(amg_ctx* ctx, cudaStream_t s) {
    if (!ctx->nsp) return;
    Atoms<R>& A = atoms_of<R>(ctx);
    const bool sp = ctx->sparse_prec;
    k_scaled_coeffs<R><<<nblk(ctx->nsp), kThreads, 0, s>>>(
        ctx->nsp, ctx->sp, ctx->xyz, ctx->pdamp, ctx->thole, ctx->bx, ctx->cut * ctx->cut, ewald_alpha(ctx), ctx->nnb,
        ctx->cap, ctx->rank, ctx->cnb, A.c0, ctx->usolvcut * ctx->usolvcut, sp ? ctx->nnbu : nullptr,
        sp ? ctx->nbru : nullptr, sp ? A.cu0 : nullptr);
    KCHECK();
}

// pair coefficients of the real-space T for the whole solve (the adjoint's
// FP64 solve; the forward builds them with the permanent field)
template <class R>
void build_tu_coeffs(amg_ctx* ctx, cudaStream_t s) {
    const int n = ctx->n;
    Atoms<R>& A = atoms_of<R>(ctx);
    const bool sp = ctx->sparse_prec;
    const double u2 = ctx->usolvcut * ctx->usolvcut;
    int* nbru = sp ? ctx->nbru : nullptr;
    int* nnbu = sp ? ctx->nnbu : nullptr;
    R4<R>* cu0 = sp ? A.cu0 : nullptr;
    LPA_DISPATCH(ctx->lpa, {
        if (ewald_cells(ctx))
            k_tu_coeffs<R, true, 8, true><<<nblk((size_t)n * 8), kThreads, 0, s>>>(n, ctx->sids, A.atS, ctx->bx, (R)ctx->aewald,
                                                                                   ctx->cnb, ctx->cap, ctx->nnb, A.c0,
                                                                                   (R)u2, nbru, cu0, nnbu);
        else if (ctx->ewald)
            k_tu_coeffs<R, true, L><<<nblk((size_t)n * L), kThreads, 0, s>>>(n, ctx->sids, A.atS, ctx->bx, (R)ctx->aewald, ctx->cnb,
                                                                             ctx->cap, ctx->nnb, A.c0, (R)u2, nbru,
                                                                             cu0, nnbu);
        else
            k_tu_coeffs<R, false, L><<<nblk((size_t)n * L), kThreads, 0, s>>>(n, ctx->sids, A.atS, ctx->bx, (R)0, ctx->cnb, ctx->cap,
                                                                              ctx->nnb, A.c0, (R)u2, nbru, cu0,
                                                                              nnbu);
    });
    KCHECK();
    build_scaled_coeffs<R>(ctx, s);
}

// A v with the stored coefficients; v4 is the R4 copy of (vd, vp).  With
// vAv (Ewald only) the dot products v.Av are added to vAv[0..1].  `apart`
// (Ewald, with vAv) keeps the real-space field out of Ad, Ap: the gather then
// runs beside the real-space kernel instead of after it, each adds its share
// of v.Av, and the caller takes A v = Ad - Fd (k_pcg_update).
template <class R>
void matvec_stored(amg_ctx* ctx, cudaStream_t s, const R4<R>* v4, const double* vd, const double* vp, double* Ad,
                   double* Ap, double* vAv = nullptr, bool spread = true, bool apart = false, bool clear = true) {
    const int n = ctx->n;
    Atoms<R>& A = atoms_of<R>(ctx);
    apart = apart && ctx->ewald && vAv;
    // real space on the side stream, PME on s
    cudaStream_t r = ctx->ewald ? fork_side(ctx, s) : s;
    LPA_DISPATCH(ctx->lpa, {
        k_tu_stored<R, L><<<nblk((size_t)n * L), kThreads, 0, r>>>(n, ctx->sids, ctx->cnb, A.c0, ctx->cap, ctx->nnb, ctx->xoff,
                                                                    v4, ctx->Fd, ctx->Fp, apart ? vd : nullptr,
                                                                    apart ? vp : nullptr, apart ? vAv : nullptr);
    });
    KCHECK();
    if (ctx->ewald) {
        Pme<R>& pm = pme_of<R>(ctx);
        pme_dipole_grids<R>(ctx, s, vd, vp, spread, nullptr, true, clear);
        if (!apart) join_side(ctx, s);
        int3 K = make_int3(ctx->K[0], ctx->K[1], ctx->K[2]);
        constexpr int G = 8;  // lanes per site
        const unsigned blocks = (unsigned)std::min<size_t>(nblk((size_t)n * G), (size_t)ctx->num_sms * 8);
        k_gather_field<R, kOrder, G><<<blocks, kThreads, 0, s>>>(n, pm.zq, pm.theta, pm.k0, K, ctx->frac, vd,
                                                                 vp, apart ? nullptr : ctx->Fd,
                                                                 apart ? nullptr : ctx->Fp, self_coef(ctx), ctx->pol,
                                                                 Ad, Ap, vAv);
        KCHECK();
        if (apart) join_side(ctx, s);
    } else {
        k_matvec_finish<<<nblk(n), kThreads, 0, s>>>(n, vd, vp, ctx->Fd, ctx->Fp, ctx->phiU4, 0, 0.0, ctx->pol, Ad, Ap);
        KCHECK();
    }
}

bool iterative(const amg_ctx* ctx) { return ctx->has_pol && ctx->poltyp == AMG_POL_MUTUAL && ctx->npolar > 0; }

double pcg_threshold(const amg_ctx* ctx) {
    double t = ctx->poleps / ctx->debye;
    return t * t * ctx->npolar;
}

// diagonal weight of the sparse preconditioner M = w alpha + alpha T_u alpha
// (2: fewest iterations on water boxes, with M safely positive definite)
constexpr double kPrecDiag = 2.0;

// z = M r for both residual sets from the packed s = alpha r (A.s4); adds
// r.z to the scalars and (its last block) rolls them for the direction update
template <class R>
void precondition(amg_ctx* ctx, cudaStream_t s) {
    const int n = ctx->n;
    Atoms<R>& A = atoms_of<R>(ctx);
    constexpr int L = 4;  // lanes per site: the rows are short
    const unsigned blocks = (unsigned)std::min<size_t>(nblk((size_t)n * L), (size_t)ctx->num_sms * 8);
    k_precond<R, L><<<blocks, kThreads, 0, s>>>(n, ctx->sids, ctx->nbru, A.cu0, ctx->cap, ctx->nnbu, ctx->xoff, A.s4,
                                                ctx->pol, kPrecDiag, ctx->rd, ctx->rp, ctx->zd, ctx->zp, ctx->scal,
                                                ctx->blk_done);
    KCHECK();
}

// Up to this many sites the PCG direction update and the spreading of p are
// separate kernels, and the spreading runs beside k_tu_stored (4,096 waters:
// 3.5% faster per evaluation); above it the fused k_pcg_dir_spread is as fast
// (32,768 waters) with fewer launches.
constexpr int kSplitSpreadSites = 65536;
bool split_spread(const amg_ctx* ctx) { return ctx->ewald && ctx->n <= kSplitSpreadSites; }

// p = z + beta p after the rz scalars were rolled; with Ewald (and above
// kSplitSpreadSites) fused with the spreading of p for the next matvec
template <class R>
void direction(amg_ctx* ctx, cudaStream_t s) {
    const int n = ctx->n;
    Atoms<R>& A = atoms_of<R>(ctx);
    if (ctx->ewald && !split_spread(ctx)) {
        Pme<R>& pm = pme_of<R>(ctx);
        const int3 K = make_int3(ctx->K[0], ctx->K[1], ctx->K[2]);
        k_pcg_dir_spread<R, kOrder><<<spread_blocks<R>(n), 128, 0, s>>>(n, ctx->zd, ctx->zp, ctx->pd, ctx->pp, ctx->scal, A.p4, pm.theta,
                                                       pm.k0, K, ctx->frac, pm.zg, ctx->rank);
    } else {
        k_pcg_dir<R><<<nblk(n), kThreads, 0, s>>>(n, ctx->zd, ctx->zp, ctx->pd, ctx->pp, ctx->scal, A.p4, ctx->rank);
    }
    KCHECK();
}

// set-up of the solve: r = E - A u0 (with the diagonal preconditioner also
// z = alpha r and r.z) and the first control decision (continue while
// rr > threshold and iterations < politer)
template <class R>
void enqueue_pcg_init(amg_ctx* ctx, cudaStream_t s, cudaGraphConditionalHandle h, int use_handle,
                      bool coeffs_built) {
    const int n = ctx->n;
    Atoms<R>& A = atoms_of<R>(ctx);
    if (!ctx->guess) {
        k_zero<double><<<nblk(3 * n, 256), 256, 0, s>>>(ctx->ud, 3 * (size_t)n);
        KCHECK();
        k_zero<double><<<nblk(3 * n, 256), 256, 0, s>>>(ctx->up, 3 * (size_t)n);
        KCHECK();
    }
    k_zero<double><<<1, 32, 0, s>>>(ctx->scal, NSCAL);
    KCHECK();
    if (!coeffs_built) build_tu_coeffs<R>(ctx, s);
    k_pack_u<R><<<nblk(n), kThreads, 0, s>>>(n, ctx->ud, ctx->up, A.u4, ctx->rank);  // cell order
    KCHECK();
    // leaves the dipole grid clear for the direction updates' spreading
    matvec_stored<R>(ctx, s, A.u4, ctx->ud, ctx->up, ctx->Apd, ctx->App);
    k_pcg_init<R><<<nblk(n), kThreads, 0, s>>>(n, ctx->Ed, ctx->Ep, ctx->Apd, ctx->App, ctx->pol, ctx->rd, ctx->rp,
                                               ctx->zd, ctx->zp, ctx->scal, ctx->sparse_prec ? A.s4 : nullptr,
                                               ctx->rank);
    KCHECK();
    k_pcg_control<<<1, 1, 0, s>>>(ctx->scal, ctx->iter, pcg_threshold(ctx), ctx->politer, 1, 0, h, use_handle,
                                  ctx->cont);
    KCHECK();
}

// one PCG iteration (both right-hand sides): preconditioner (sparse), the
// direction update (spreading p with Ewald), matvec, and the residual update
// whose last block takes the control decision.  Ending with the decision, the iteration that meets the
// threshold leaves no preconditioner or direction work behind it.
template <class R>
void enqueue_pcg_iter(amg_ctx* ctx, cudaStream_t s, cudaGraphConditionalHandle h, int use_handle) {
    const int n = ctx->n, n3 = 3 * n;
    Atoms<R>& A = atoms_of<R>(ctx);
    if (ctx->sparse_prec) precondition<R>(ctx, s);
    direction<R>(ctx, s);
    // p.Ap: fused into the PME gather with Ewald, a separate pass without
    const bool apart = ctx->ewald;  // real-space field kept apart: the gather overlaps k_tu_stored
    // split: the direction kernel only updates p; p is spread here, beside
    // k_tu_stored, into the grid the previous transform left cleared
    matvec_stored<R>(ctx, s, A.p4, ctx->pd, ctx->pp, ctx->Apd, ctx->App, ctx->ewald ? ctx->scal + PAP_D : nullptr,
                     split_spread(ctx), apart, false);
    if (!ctx->ewald) {
        k_dot2<<<nblk(n3, 256), 256, 0, s>>>(n3, ctx->pd, ctx->Apd, ctx->pp, ctx->App, ctx->scal + PAP_D,
                                              ctx->scal + PAP_P);
        KCHECK();
    }
    const unsigned ublocks = (unsigned)std::min<size_t>(nblk(3 * (size_t)n, 256), (size_t)ctx->num_sms * 4);
    k_pcg_update<R><<<ublocks, 256, 0, s>>>(n, ctx->pol, ctx->pd, ctx->pp, ctx->Apd, ctx->App, ctx->ud, ctx->up,
                                                 ctx->rd, ctx->rp, ctx->zd, ctx->zp, ctx->scal,
                                                 ctx->sparse_prec ? A.s4 : nullptr, ctx->rank,
                                                 apart ? ctx->Fd : nullptr, apart ? ctx->Fp : nullptr,
                                                 ctx->blk_done, ctx->iter, pcg_threshold(ctx), ctx->politer,
                                                 ctx->sparse_prec ? 0 : 1, h, use_handle, ctx->cont);
    KCHECK();
}

// FP64 correction sweep: the true residual with every term in FP64, one
// diagonal-preconditioned step u += alpha r, and the residual norms
void enqueue_sweep(amg_ctx* ctx, cudaStream_t s) {
    matvec<double>(ctx, s, ctx->ud, ctx->up, ctx->Apd, ctx->App, true);
    k_zero<double><<<1, 32, 0, s>>>(ctx->scal + PAP_D, 6);
    KCHECK();
    k_correct<<<nblk(ctx->n), kThreads, 0, s>>>(ctx->n, ctx->Ed, ctx->Ep, ctx->Apd, ctx->App, ctx->pol, ctx->ud, ctx->up,
                                                ctx->resd, ctx->scal);
    KCHECK();
}

// everything before the PCG loop: frames, lists, stencils, permanent field,
// direct dipoles
template <class R>
void enqueue_front(amg_ctx* ctx, cudaStream_t s) {
    const int n = ctx->n;
    const bool mixed = ctx->prec == AMG_PREC_MIXED;
    CK(cudaEventRecord(ctx->ev[0], s));
    if (ctx->cflux) {  // monopole increments of this geometry, before the rotation uses them
        k_zero<double><<<nblk(n, 256), 256, 0, s>>>(ctx->dq, (size_t)n);
        KCHECK();
        k_cflux_charges<<<nblk((size_t)ctx->nbond + ctx->nangle), kThreads, 0, s>>>(
            ctx->nbond, ctx->bonds, ctx->bflux, ctx->nangle, ctx->angles, ctx->aflux, ctx->xyz, ctx->dq);
        KCHECK();
    }
    // neighbour list and real-space permanent field on the side stream (the
    // list build needs only the positions, so it starts beside the frame
    // rotations); PME stencils and the reciprocal permanent potential on s
    cudaStream_t r = fork_side(ctx, s);
    enqueue_lists(ctx, r);
    rotate_and_pack<R>(ctx, s);
    if (mixed && iterative(ctx)) rotate_and_pack<double>(ctx, s);
    k_zero<double><<<1, 32, 0, s>>>(ctx->eacc, kEacc);
    KCHECK();
    k_zero<unsigned long long><<<1, 32, 0, s>>>(ctx->cnt, 4);
    KCHECK();
    CK(cudaEventRecord(ctx->erot, s));  // the packed sites for the cell-order copy
    CK(cudaStreamWaitEvent(r, ctx->erot, 0));
    k_gather_atoms<R><<<nblk(n), kThreads, 0, r>>>(n, ctx->sids, atoms_of<R>(ctx).at, atoms_of<R>(ctx).atS);
    KCHECK();
    if (ctx->ewald) {
        pme_stencils<R>(ctx, s, mixed && iterative(ctx));  // FP64 ones too for the sweep
        Pme<R>& pm = pme_of<R>(ctx);
        k_zero<R><<<nblk(2 * pm.G, 256), 256, 0, s>>>(pm.grid, 2 * pm.G);
        KCHECK();
        if (mixed && iterative(ctx)) {
            Pme<double>& pd = pme_of<double>(ctx);
            k_zero<double><<<nblk(2 * pd.G, 256), 256, 0, s>>>(pd.grid, 2 * pd.G);
            KCHECK();
        }
    }
    CK(cudaEventRecord(ctx->ev[1], s));
    Atoms<R>& A = atoms_of<R>(ctx);
    const R aew = (R)ctx->aewald;
    if (ctx->has_pol) {
        // with a solve to follow, the same pass fills the PCG's coefficient rows
        const bool coef = iterative(ctx);
        const bool sp = coef && ctx->sparse_prec;
        const R u2 = (R)(ctx->usolvcut * ctx->usolvcut);
        auto launch = [&](auto kern, unsigned nb) {
            kern<<<nb, kThreads, 0, r>>>(n, ctx->sids, A.atS, ctx->bx, aew, ctx->cnb, ctx->cap, ctx->nnb, ctx->Ed, ctx->Ep,
                                         coef ? A.c0 : nullptr, u2, sp ? ctx->nbru : nullptr,
                                         sp ? A.cu0 : nullptr, sp ? ctx->nnbu : nullptr);
        };
        LPA_DISPATCH(ctx->lpa, {
            const unsigned nb = nblk((size_t)n * L);
            if (ewald_cells(ctx)) {  // Ewald in a monoclinic or triclinic cell: 8 lanes
                if (coef) launch(k_perm_field<R, true, 8, true, true>, nblk((size_t)n * 8));
                else launch(k_perm_field<R, true, 8, false, true>, nblk((size_t)n * 8));
            } else if (ctx->ewald) {
                if (coef) launch(k_perm_field<R, true, L, true>, nb);
                else launch(k_perm_field<R, true, L, false>, nb);
            } else {
                if (coef) launch(k_perm_field<R, false, L, true>, nb);
                else launch(k_perm_field<R, false, L, false>, nb);
            }
        });
        KCHECK();
        if (coef) build_scaled_coeffs<R>(ctx, r);
        if (ctx->nsp) {
            k_scaled_field<<<nblk(ctx->nsp), kThreads, 0, r>>>(ctx->nsp, ctx->sp, ctx->xyz, ctx->rp10, ctx->pdamp,
                                                              ctx->thole, ctx->bx, ctx->cut * ctx->cut, ewald_alpha(ctx),
                                                              ctx->Ed, ctx->Ep);
            KCHECK();
        }
    }
    if (ctx->ewald) pme_mpole<R>(ctx, s, ctx->want_vir ? ctx->eacc + kVir : nullptr);
    join_side(ctx, s);
    if (ctx->has_pol) {
        k_field_finish<<<nblk(n), kThreads, 0, s>>>(n, ctx->phiM, ctx->ewald, ctx->rp10, self_coef(ctx), ctx->pol, ctx->Ed,
                                                    ctx->Ep, ctx->ud, ctx->up);
        KCHECK();
    }
    CK(cudaEventRecord(ctx->ev[2], s));
}

// OPT dipoles (extrapolated perturbation theory): from the direct dipoles
// u^(0) = alpha E left in (ud, up) by the permanent field, optorder
// applications of the dipole field, u^(k) = alpha T u^(k-1) = v - alpha A v,
// mixed into u = sum_k copm_k u^(k); every u^(k) is kept for the forces
template <class R>
void enqueue_opt(amg_ctx* ctx, cudaStream_t s) {
    const int n3 = 3 * ctx->n;
    const size_t blk = 6 * (size_t)ctx->n;  // one order: d set then p set
    double* uo = ctx->uopt;
    k_opt_init<<<nblk(n3), kThreads, 0, s>>>(n3, ctx->copm.c[0], ctx->ud, ctx->up, uo, uo + n3);
    KCHECK();
    for (int k = 1; k <= ctx->optorder; k++) {
        const double* vd = uo + (k - 1) * blk;
        matvec<R>(ctx, s, vd, vd + n3, ctx->Apd, ctx->App);
        k_opt_step<<<nblk(n3), kThreads, 0, s>>>(n3, ctx->pol, vd, vd + n3, ctx->Apd, ctx->App, ctx->copm.c[k],
                                                 uo + k * blk, uo + k * blk + n3, ctx->ud, ctx->up);
        KCHECK();
    }
}

// OPT force terms between perturbation orders: for b = 0..K-1 the
// dipole-dipole interaction of ud^(b) with V_b = sum_a copm_{a+b+1} up^(a)
// (from d(alpha T)^k = sum_{a+b=k-1} (alpha T)^a alpha dT (alpha T)^b), in
// real space (bulk and scaled pairs) and reciprocal space, on stream s
template <class R>
void enqueue_opt_cross(amg_ctx* ctx, cudaStream_t s, double* virp) {
    const int n = ctx->n, n3 = 3 * n;
    const size_t blk = 6 * (size_t)n;
    double* uo = ctx->uopt;
    double* V = uo + (ctx->optorder + 1) * blk;
    Atoms<R>& A = atoms_of<R>(ctx);
    const R aew = (R)ctx->aewald;
    for (int b = 0; b < ctx->optorder; b++) {
        const double* Y = uo + b * blk;  // ud^(b)
        k_opt_cross<<<nblk(n3), kThreads, 0, s>>>(n3, ctx->optorder, b, ctx->copm, uo, V);
        KCHECK();
        k_pack_u<R><<<nblk(n), kThreads, 0, s>>>(n, Y, V, A.u4, ctx->rank);  // cell order
        KCHECK();
        auto launch = [&](auto kern) {
            kern<<<nblk((size_t)n * 8), kThreads, 0, s>>>(n, ctx->sids, A.atS, A.u4, ctx->bx, aew, ctx->cnb, ctx->cap,
                                                          ctx->nnb, 1, ctx->f, ctx->grad_p, ctx->trq_p, virp);
        };
        if (ewald_cells(ctx)) {
            if (virp) launch(k_polar_pair<R, true, 8, true, true, true>);
            else launch(k_polar_pair<R, true, 8, false, true, true>);
        } else if (ctx->ewald) {
            if (virp) launch(k_polar_pair<R, true, 8, true, true>);
            else launch(k_polar_pair<R, true, 8, false, true>);
        } else {
            if (virp) launch(k_polar_pair<R, false, 8, true, true>);
            else launch(k_polar_pair<R, false, 8, false, true>);
        }
        KCHECK();
        if (ctx->nsp) {
            k_scaled_polar<<<nblk(ctx->nsp), kThreads, 0, s>>>(ctx->nsp, ctx->sp, ctx->xyz, ctx->rp10, ctx->pdamp,
                                                              ctx->thole, ctx->bx, ctx->cut * ctx->cut, ewald_alpha(ctx),
                                                              Y, V, 1, 1, ctx->f, ctx->grad_p, ctx->trq_p, virp);
            KCHECK();
        }
        if (ctx->ewald) {
            pme_dipoles<R, 20>(ctx, s, Y, V, ctx->phiU, virp, false);
            k_recip_polar<<<nblk(n), kThreads, 0, s>>>(n, ctx->rp10, ctx->phiM, ctx->phiU, ctx->phiU + 20 * (size_t)n,
                                                       Y, V, 1, 1, self_coef(ctx), ctx->f, ctx->grad_p, ctx->trq_p,
                                                       virp);
            KCHECK();
        }
    }
}

// everything after the solve: energies, gradients, torques
// predictor: the starting dipoles from the history (before the PCG set-up)
// and the converged dipoles into it (after the correction sweep)
void enqueue_predict(amg_ctx* ctx, cudaStream_t s) {
    if (!ctx->pred) return;
    const int n3 = 3 * ctx->n;
    k_predict<<<nblk(n3), kThreads, 0, s>>>(n3, ctx->pred_hist, ctx->pred_state, ctx->pred_coef, ctx->ud, ctx->up);
    KCHECK();
}
void enqueue_pred_store(amg_ctx* ctx, cudaStream_t s) {
    if (!ctx->pred) return;
    const int n3 = 3 * ctx->n;
    k_pred_store<<<nblk(n3), kThreads, 0, s>>>(n3, ctx->pred_hist, ctx->pred_state, ctx->ud, ctx->up);
    KCHECK();
    k_pred_advance<<<1, 1, 0, s>>>(ctx->pred_state);
    KCHECK();
}

// Permanent-multipole energy and forces: the real-space pair kernels (atomic
// accumulation), then the reciprocal part and the frame torques, which add to
// the same arrays without atomics.  They need only what the front computed
// (lists, rotated multipoles, the permanent PME potentials) and touch none of
// the solve's arrays, so they run on their own stream m beside the dipole
// solve; enqueue_back joins m at its end.
template <class R>
void enqueue_mpole_forces(amg_ctx* ctx, cudaStream_t m, int flags) {
    const int n = ctx->n;
    const bool grad = flags & AMG_DO_GRADIENT;
    const bool analysis = flags & AMG_DO_ANALYSIS;
    const double cut2 = ctx->cut * ctx->cut;
    Atoms<R>& A = atoms_of<R>(ctx);
    const R aew = (R)ctx->aewald;
    k_zero<double><<<nblk(3 * n, 256), 256, 0, m>>>(ctx->grad_m, 3 * (size_t)n);
    KCHECK();
    k_zero<double><<<nblk(3 * n, 256), 256, 0, m>>>(ctx->trq_m, 3 * (size_t)n);
    KCHECK();
    k_zero<double><<<nblk(n, 256), 256, 0, m>>>(ctx->aem, (size_t)n);
    KCHECK();
    const cudaStream_t r = m;
    const int* mol = ctx->mol;
    double* vir = ctx->want_vir ? ctx->eacc + kVir : nullptr;  // em terms
    // Analysis and Virial outputs come from the EXTRA pair kernels
    const bool extra = analysis || vir;
    if (ctx->cp_mode) {
        // charge penetration / charge flux: the core/valence pairs in FP64
        if (ctx->cflux) {
            k_zero<double><<<nblk(n, 256), 256, 0, r>>>(ctx->cfpot, (size_t)n);
            KCHECK();
        }
        auto launch = [&](auto kern) {
            kern<<<nblk((size_t)n * 8), kThreads, 0, r>>>(
                n, ctx->sids, ctx->xyz, ctx->rp10, ctx->pcore, ctx->palpha, ctx->cpt, ctx->bx, ctx->nbr, ctx->cap,
                ctx->nnb, ctx->f, ctx->grad_m, ctx->trq_m, ctx->cflux ? ctx->cfpot : nullptr, ctx->eacc,
                analysis ? ctx->aem : nullptr, analysis ? mol : nullptr, analysis ? ctx->cnt : nullptr, vir);
        };
        if (extra) launch(k_cp_pair<8, true>);
        else launch(k_cp_pair<8, false>);
        KCHECK();
        if (ctx->nsp) {
            k_cp_scaled<<<nblk(ctx->nsp), kThreads, 0, r>>>(
                ctx->nsp, ctx->sp, ctx->xyz, ctx->rp10, ctx->pcore, ctx->palpha, ctx->cpt, ctx->bx, cut2, ctx->f,
                ctx->grad_m, ctx->trq_m, ctx->cflux ? ctx->cfpot : nullptr, ctx->eacc, analysis ? ctx->aem : nullptr,
                analysis ? mol : nullptr, analysis ? ctx->cnt : nullptr, vir);
            KCHECK();
        }
    } else {
    LPA_DISPATCH(ctx->lpa, {
        const size_t nb = nblk((size_t)n * L);
        auto launch_n = [&](auto kern, size_t blocks) {
            kern<<<blocks, kThreads, 0, r>>>(n, ctx->sids, A.atS, ctx->bx, aew, ctx->cnb, ctx->cap, ctx->nnb, ctx->f,
                                             ctx->grad_m, ctx->trq_m, ctx->eacc, analysis ? ctx->aem : nullptr,
                                             analysis ? mol : nullptr, analysis ? ctx->cnt : nullptr, vir);
        };
        auto launch = [&](auto kern) { launch_n(kern, nb); };
        auto launch_cells = [&](auto kern) { launch_n(kern, nblk((size_t)n * 8)); };
        if (ewald_cells(ctx)) {
            if (extra) launch_cells(k_mpole_pair<R, true, true, 8, true>);
            else launch_cells(k_mpole_pair<R, true, false, 8, true>);
        } else if (ctx->ewald) {
            if (extra) launch(k_mpole_pair<R, true, true, L>);
            else launch(k_mpole_pair<R, true, false, L>);
        } else {
            if (extra) launch(k_mpole_pair<R, false, true, L>);
            else launch(k_mpole_pair<R, false, false, L>);
        }
    });
    KCHECK();
    if (ctx->nsp) {
        k_scaled_mpole<<<nblk(ctx->nsp), kThreads, 0, r>>>(ctx->nsp, ctx->sp, ctx->xyz, ctx->rp10, ctx->bx, cut2,
                                                          ewald_alpha(ctx), ctx->f, ctx->grad_m, ctx->trq_m, ctx->eacc,
                                                          analysis ? ctx->aem : nullptr, analysis ? mol : nullptr,
                                                          analysis ? ctx->cnt : nullptr, vir);
        KCHECK();
    }
    }
    if (ctx->ewald) {
        k_recip_mpole<<<nblk(n), kThreads, 0, m>>>(n, ctx->rp10, ctx->phiM, ctx->f, ctx->aewald, ctx->grad_m, ctx->trq_m,
                                                   ctx->eacc + 2, analysis ? ctx->aem : nullptr, ctx->eacc + 3, vir);
        KCHECK();
    }
    if (grad) {
        k_torque<<<nblk(n), kThreads, 0, m>>>(n, ctx->xyz, ctx->zax, ctx->xax, ctx->yax, ctx->axe, ctx->trq_m,
                                              ctx->grad_m, vir);
        KCHECK();
        if (ctx->cflux) {  // the gradient through the geometry-dependent monopoles
            k_cflux_grad<<<nblk((size_t)ctx->nbond + ctx->nangle), kThreads, 0, m>>>(
                ctx->nbond, ctx->bonds, ctx->bflux, ctx->nangle, ctx->angles, ctx->aflux, ctx->xyz, ctx->cfpot,
                ctx->grad_m, vir);
            KCHECK();
        }
    }
    // grad_m is final: the read-back stream may copy it while the solve runs
    // (inside a capture, an event node that work outside the graph can wait on)
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    CK(cudaStreamIsCapturing(m, &cs));
    if (cs == cudaStreamCaptureStatusActive) CK(cudaEventRecordWithFlags(ctx->gm_ready, m, cudaEventRecordExternal));
    else CK(cudaEventRecord(ctx->gm_ready, m));
}

// Polarization energy and forces after the solve; the permanent-multipole
// forces, forked onto their own stream after the front, join here.
template <class R>
void enqueue_back(amg_ctx* ctx, cudaStream_t s, int flags) {
    const int n = ctx->n;
    const bool grad = flags & AMG_DO_GRADIENT;
    const bool analysis = flags & AMG_DO_ANALYSIS;
    const bool polgrad = grad && ctx->has_pol;
    const double cut2 = ctx->cut * ctx->cut;
    Atoms<R>& A = atoms_of<R>(ctx);
    const R aew = (R)ctx->aewald;
    const int mutual = ctx->poltyp == AMG_POL_MUTUAL;
    CK(cudaEventRecord(ctx->ev[3], s));
    if (polgrad) {
        k_zero<double><<<nblk(3 * n, 256), 256, 0, s>>>(ctx->grad_p, 3 * (size_t)n);
        KCHECK();
        k_zero<double><<<nblk(3 * n, 256), 256, 0, s>>>(ctx->trq_p, 3 * (size_t)n);
        KCHECK();
        k_pack_u<R><<<nblk(n), kThreads, 0, s>>>(n, ctx->ud, ctx->up, A.u4, ctx->rank);  // cell order
        KCHECK();
    }
    // Real-space polarization pair kernels (atomic accumulation) on the side
    // stream; the PME dipole potentials and the polarization energy on s.
    // The reciprocal-space force kernels add to the same arrays without
    // atomics, so they run after the join.
    cudaStream_t r = fork_side(ctx, s);
    double* virp = ctx->want_vir ? ctx->eacc + kVirP : nullptr;  // ep terms
    if (polgrad) {
        auto launch = [&](auto kern, int lanes) {
            kern<<<nblk((size_t)n * lanes), kThreads, 0, r>>>(n, ctx->sids, A.atS, A.u4, ctx->bx, aew, ctx->cnb, ctx->cap,
                                                              ctx->nnb, mutual, ctx->f, ctx->grad_p, ctx->trq_p, virp);
        };
        if (ewald_cells(ctx)) {  // one lane count for the cell variants
            if (virp) launch(k_polar_pair<R, true, 8, true, false, true>, 8);
            else launch(k_polar_pair<R, true, 8, false, false, true>, 8);
        } else if (virp) {  // one lane count for the virial variants
            if (ctx->ewald) launch(k_polar_pair<R, true, 8, true>, 8);
            else launch(k_polar_pair<R, false, 8, true>, 8);
        } else {
            LPA_DISPATCH(ctx->lpa, {
                if (ctx->ewald) launch(k_polar_pair<R, true, L, false>, L);
                else launch(k_polar_pair<R, false, L, false>, L);
            });
        }
        KCHECK();
        if (ctx->nsp) {
            k_scaled_polar<<<nblk(ctx->nsp), kThreads, 0, r>>>(ctx->nsp, ctx->sp, ctx->xyz, ctx->rp10, ctx->pdamp,
                                                              ctx->thole, ctx->bx, cut2, ewald_alpha(ctx), ctx->ud,
                                                              ctx->up, mutual, 0, ctx->f, ctx->grad_p, ctx->trq_p, virp);
            KCHECK();
        }
    }
    if (ctx->has_pol) {
        k_polar_energy<<<nblk(n), kThreads, 0, s>>>(n, ctx->ud, ctx->Ep, ctx->f, ctx->eacc + 4,
                                                    analysis ? ctx->aep : nullptr, ctx->cnt + 1);
        KCHECK();
    }
    if (polgrad && ctx->ewald) pme_dipoles<R, 20>(ctx, s, ctx->ud, ctx->up, ctx->phiU, virp);
    join_side(ctx, s);
    if (polgrad) {
        if (ctx->ewald) {
            k_recip_polar<<<nblk(n), kThreads, 0, s>>>(n, ctx->rp10, ctx->phiM, ctx->phiU, ctx->phiU + 20 * (size_t)n,
                                                       ctx->ud, ctx->up, mutual, 0, self_coef(ctx), ctx->f, ctx->grad_p,
                                                       ctx->trq_p, virp);
            KCHECK();
        }
        if (ctx->poltyp == AMG_POL_OPT && ctx->npolar > 0) enqueue_opt_cross<R>(ctx, s, virp);
        k_torque<<<nblk(n), kThreads, 0, s>>>(n, ctx->xyz, ctx->zax, ctx->xax, ctx->yax, ctx->axe, ctx->trq_p,
                                              ctx->grad_p, virp);
        KCHECK();
    }
    join_mpole(ctx, s);
    CK(cudaEventRecord(ctx->ev[4], s));
}

// Captures the whole evaluation as one CUDA graph: the PCG loop is a
// conditional WHILE node whose body is one iteration; its last kernel sets
// the condition from the FP64 residual norms on the device.
template <class R>
bool capture_graph(amg_ctx* ctx, int flags) {
    cudaStream_t s = ctx->st;
    cudaGraph_t graph = nullptr;
    auto fail = [&](const char* what, cudaError_t e) {
        ctx->graph_note = std::string(what) + ": " + cudaGetErrorString(e);
        cudaStreamCaptureStatus st;
        if (cudaStreamIsCapturing(s, &st) == cudaSuccess && st != cudaStreamCaptureStatusNone) {
            cudaGraph_t g2;
            cudaStreamEndCapture(s, &g2);
            if (g2) cudaGraphDestroy(g2);
        }
        cudaGetLastError();
        return false;
    };
    cudaError_t e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return fail("begin capture", e);
    const long long k0 = ctx->kcount;
    long long kb = 0;
    try {
        enqueue_front<R>(ctx, s);
        enqueue_mpole_forces<R>(ctx, fork_mpole(ctx, s), flags);
        if (ctx->poltyp == AMG_POL_OPT && ctx->npolar > 0) enqueue_opt<R>(ctx, s);
        if (iterative(ctx)) {
            const cudaGraphNode_t* deps = nullptr;
            size_t ndeps = 0;
            cudaStreamCaptureStatus cs;
            e = cudaStreamGetCaptureInfo(s, &cs, nullptr, &graph, &deps, &ndeps);
            if (e != cudaSuccess) return fail("capture info", e);
            cudaGraphConditionalHandle h;
            e = cudaGraphConditionalHandleCreate(&h, graph, 0, 0);
            if (e != cudaSuccess) return fail("conditional handle", e);
            enqueue_predict(ctx, s);
            enqueue_pcg_init<R>(ctx, s, h, 1, true);
            e = cudaStreamGetCaptureInfo(s, &cs, nullptr, &graph, &deps, &ndeps);
            if (e != cudaSuccess) return fail("capture info", e);
            cudaGraphNodeParams cp = {};
            cp.type = cudaGraphNodeTypeConditional;
            cp.conditional.handle = h;
            cp.conditional.type = cudaGraphCondTypeWhile;
            cp.conditional.size = 1;
            cudaGraphNode_t cnode;
            e = cudaGraphAddNode(&cnode, graph, deps, ndeps, &cp);
            if (e != cudaSuccess) return fail("add conditional node", e);
            cudaGraph_t body = cp.conditional.phGraph_out[0];
            e = cudaStreamUpdateCaptureDependencies(s, &cnode, 1, cudaStreamSetCaptureDependencies);
            if (e != cudaSuccess) return fail("update dependencies", e);
            e = cudaStreamBeginCaptureToGraph(ctx->st2, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
            if (e != cudaSuccess) return fail("body capture", e);
            const long long kb0 = ctx->kcount;
            enqueue_pcg_iter<R>(ctx, ctx->st2, h, 1);
            kb = ctx->kcount - kb0;
            e = cudaStreamEndCapture(ctx->st2, &body);
            if (e != cudaSuccess) return fail("end body capture", e);
            enqueue_sweep(ctx, s);
            enqueue_pred_store(ctx, s);
        }
        enqueue_back<R>(ctx, s, flags);
    } catch (Fail&) {
        return fail("enqueue", cudaGetLastError());
    }
    e = cudaStreamEndCapture(s, &graph);
    if (e != cudaSuccess) return fail("end capture", e);
    if (ctx->gexec) cudaGraphExecDestroy(ctx->gexec);
    ctx->gexec = nullptr;
    e = cudaGraphInstantiate(&ctx->gexec, graph, cudaGraphInstantiateFlagUseNodePriority);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) {
        ctx->gexec = nullptr;
        return fail("instantiate", e);
    }
    ctx->gflags = flags;
    ctx->graph_dirty = false;
    ctx->fwd_gen++;
    ctx->kbody = kb;
    ctx->kmain = ctx->kcount - k0 - kb;
    ctx->kcount = k0;
    return true;
}

template <class R>
void enqueue_eager(amg_ctx* ctx, int flags) {
    cudaStream_t s = ctx->st;
    enqueue_front<R>(ctx, s);
    enqueue_mpole_forces<R>(ctx, fork_mpole(ctx, s), flags);
    if (ctx->poltyp == AMG_POL_OPT && ctx->npolar > 0) enqueue_opt<R>(ctx, s);
    if (iterative(ctx)) {
        enqueue_predict(ctx, s);
        enqueue_pcg_init<R>(ctx, s, 0, 0, true);
        int cont = 1;
        while (true) {
            CK(cudaMemcpyAsync(&cont, ctx->cont, sizeof(int), cudaMemcpyDeviceToHost, s));
            CK(cudaStreamSynchronize(s));
            if (!cont) break;
            enqueue_pcg_iter<R>(ctx, s, 0, 0);
        }
        enqueue_sweep(ctx, s);
        enqueue_pred_store(ctx, s);
    }
    enqueue_back<R>(ctx, s, flags);
}

template <class R>
int forward_impl(amg_ctx* ctx, int flags, amg_results* res) {
    const int n = ctx->n;
    const bool grad = flags & AMG_DO_GRADIENT;
    const bool analysis = flags & AMG_DO_ANALYSIS;
    ctx->want_vir = (flags & AMG_DO_VIRIAL) != 0;
    cudaStream_t st = ctx->st;
    if (!ctx->rb) {
        CK(cudaMallocHost((void**)&ctx->rb, sizeof(amg_ctx::Readback)));
        CK(cudaMallocHost((void**)&ctx->rb_grad, sizeof(double) * 6 * (size_t)n));
        for (auto& e : ctx->rbev) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        for (auto& e : ctx->rbevm) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    }
    bool dem_added = false;  // the permanent-multipole gradient is in res->dem
    for (int attempt = 0; attempt < 2; attempt++) {
        ensure_list_buffers(ctx);
        if (iterative(ctx)) ensure_coeff_buffers<R>(ctx, atoms_of<R>(ctx));
        if (ctx->ewald) {
            pme_prepare<R>(ctx, pme_of<R>(ctx));
            if (ctx->prec == AMG_PREC_MIXED && iterative(ctx)) pme_prepare<double>(ctx, pme_of<double>(ctx));
        }
        bool graphed = false;
        const long long kstart = ctx->kcount;
        if (ctx->use_graphs && ctx->bounds) {
            if (ctx->graph_dirty || !ctx->gexec || ctx->gflags != flags) capture_graph<R>(ctx, flags);
            if (ctx->gexec) {
                CK(cudaGraphLaunch(ctx->gexec, st));
                graphed = true;
            }
        }
        if (!graphed) enqueue_eager<R>(ctx, flags);
        ctx->klast = graphed ? -1 : ctx->kcount - kstart;  // graph: completed below from the iteration count
        // status, scalars and gradients behind one synchronisation
        amg_ctx::Readback* rb = ctx->rb;
        CK(cudaMemcpyAsync(&rb->over, ctx->overflow, sizeof(int), cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(rb->e, ctx->eacc, sizeof(rb->e), cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(rb->c, ctx->cnt, sizeof(rb->c), cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(rb->hs, ctx->scal, sizeof(double) * NSCAL, cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(&rb->iters, ctx->iter, sizeof(int), cudaMemcpyDeviceToHost, st));
        CK(cudaEventRecord(ctx->rbev[0], st));
        // the gradients in kRbChunks pieces, each with its event: the host adds
        // a piece to the caller's arrays while the next one is in flight.  The
        // permanent-multipole gradient is final once its force stream is done
        // (gm_ready), so its pieces are copied, and added, beside the solve;
        // the list-overflow flag, final by then too, is read with them.
        const size_t n3 = 3 * (size_t)n, piece = (n3 + kRbChunks - 1) / kRbChunks;
        const bool early_m = grad && res->dem;
        if (early_m) {
            CK(cudaStreamWaitEvent(ctx->rbst, ctx->gm_ready, 0));
            CK(cudaMemcpyAsync(&rb->over_m, ctx->overflow, sizeof(int), cudaMemcpyDeviceToHost, ctx->rbst));
            for (int k = 0; k < kRbChunks; k++) {
                const size_t a = std::min(n3, k * piece), b = std::min(n3, a + piece);
                if (b > a)
                    CK(cudaMemcpyAsync(ctx->rb_grad + a, ctx->grad_m + a, sizeof(double) * (b - a),
                                       cudaMemcpyDeviceToHost, ctx->rbst));
                CK(cudaEventRecord(ctx->rbevm[k], ctx->rbst));
            }
        }
        for (int k = 0; k < kRbChunks; k++) {
            const size_t a = std::min(n3, k * piece), b = std::min(n3, a + piece);
            if (b > a && grad && res->dep && ctx->has_pol)
                CK(cudaMemcpyAsync(ctx->rb_grad + n3 + a, ctx->grad_p + a, sizeof(double) * (b - a),
                                   cudaMemcpyDeviceToHost, st));
            CK(cudaEventRecord(ctx->rbev[1 + k], st));
        }
        if (early_m) {
            CK(cudaEventSynchronize(ctx->rbevm[0]));  // over_m landed before the first piece
            if (rb->over_m <= ctx->cap) {
                dem_added = true;
                for (int k = 0; k < kRbChunks; k++) {
                    const size_t a = std::min(n3, k * piece), b = std::min(n3, a + piece);
                    CK(cudaEventSynchronize(ctx->rbevm[k]));
                    for (size_t q = a; q < b; q++) res->dem[q] += ctx->rb_grad[q];
                }
            }
        }
        CK(cudaEventSynchronize(ctx->rbev[0]));
        const int over = rb->over;
        if (over <= ctx->cap) break;
        CK(cudaStreamSynchronize(st));
        if (attempt == 1) {
            ctx->err = "neighbour list overflow";
            return AMG_ERR_CUDA;
        }
        ctx->cap = ((over * 5 / 4) + 31) / 32 * 32;
        dalloc(ctx, ctx->nbr, (size_t)ctx->cap * n);
        dalloc(ctx, ctx->cnb, (size_t)ctx->cap * n);
        ctx->graph_dirty = true;
        // the overflowed evaluation's dipoles went into the predictor's
        // history: start the history again
        if (ctx->pred_state) CK(cudaMemsetAsync(ctx->pred_state, 0, 2 * sizeof(int), st));
    }
    ctx->graphed_last = ctx->use_graphs && ctx->bounds && ctx->gexec != nullptr;
    // ---- results
    const double* e = ctx->rb->e;
    const double* hs = ctx->rb->hs;
    const unsigned long long* c = ctx->rb->c;
    int iters = ctx->rb->iters;
    double eps = 0;
    int status = AMG_OK;
    if (ctx->klast < 0) ctx->klast = ctx->kmain + (long long)iters * ctx->kbody;
    if (iterative(ctx)) {
        eps = ctx->debye * std::sqrt(std::max(hs[RR_D], hs[RR_P]) / ctx->npolar);
        if (eps > ctx->poleps) status = AMG_ERR_NO_CONVERGE;
    } else {
        iters = ctx->poltyp == AMG_POL_OPT ? ctx->optorder : 0;
    }
    auto fetch = [&](double* dst, const double* src, size_t cnt) {
        if (!dst) return;
        CK(cudaMemcpyAsync(dst, src, sizeof(double) * cnt, cudaMemcpyDeviceToHost, st));
    };
    double em = e[0] + e[2], echg = 0;
    if (ctx->ewald) {
        double V = ctx->vol;
        double qt = e[3];
        ctx->qtot = qt;
        echg = -ctx->f * kPi * qt * qt / (2 * V * ctx->aewald * ctx->aewald);
        em += echg;
    }
    ctx->have_vir = ctx->want_vir;
    if (ctx->want_vir) {  // six sums -> symmetric 3x3, added; the net-charge term goes as 1/V
        for (int part = 0; part < 2; part++) {
            const double* v = e + (part ? kVirP : kVir);
            const double c = part ? 0.0 : echg;
            const double w[9] = {v[0] - c, v[3], v[4], v[3], v[1] - c, v[5], v[4], v[5], v[2] - c};
            for (int k = 0; k < 9; k++) {
                ctx->vir_parts[part][k] = w[k];
                res->vir[k] += w[k];
            }
        }
    }
    res->em = em;
    res->ep = ctx->has_pol ? e[4] : 0.0;
    res->einter = e[1];
    res->nem = (int64_t)(c[0] / 2);
    res->nep = (int64_t)c[1];
    res->pcg_iters = iters;
    res->pcg_eps = eps;
    if (grad) {  // added to the caller's arrays piece by piece as the copies land
        double* dem = dem_added ? nullptr : res->dem;
        double* dep = ctx->has_pol ? res->dep : nullptr;
        const size_t n3 = 3 * (size_t)n, piece = (n3 + kRbChunks - 1) / kRbChunks;
        const double* gm = ctx->rb_grad;
        const double* gp = ctx->rb_grad + n3;
        for (int k = 0; k < kRbChunks; k++) {
            const size_t a = std::min(n3, k * piece), b = std::min(n3, a + piece);
            CK(cudaEventSynchronize(ctx->rbev[1 + k]));
            if (dem)
                for (size_t q = a; q < b; q++) dem[q] += gm[q];
            if (dep)
                for (size_t q = a; q < b; q++) dep[q] += gp[q];
        }
    }
    if (analysis) {
        fetch(res->aem, ctx->aem, n);
        if (ctx->has_pol) fetch(res->aep, ctx->aep, n);
    }
    if ((flags & AMG_DO_DIPOLES) && ctx->has_pol) {
        fetch(res->uind, ctx->ud, 3 * (size_t)n);
        fetch(res->uinp, ctx->up, 3 * (size_t)n);
    }
    if (res->rpole) {
        std::vector<double> r10(10 * (size_t)n);
        CK(cudaMemcpyAsync(r10.data(), ctx->rp10, sizeof(double) * 10 * n, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        for (int i = 0; i < n; i++) {
            const double* m = &r10[10 * (size_t)i];
            double* o = res->rpole + 13 * (size_t)i;
            double v[13] = {m[0], m[1], m[2], m[3], m[4], m[5], m[6], m[5], m[7], m[8], m[6], m[8], m[9]};
            std::memcpy(o, v, sizeof(v));
        }
    }
    CK(cudaStreamSynchronize(st));
    float ms[4] = {0, 0, 0, 0};
    for (int k = 0; k < 4; k++)
        if (cudaEventElapsedTime(&ms[k], ctx->ev[k], ctx->ev[k + 1]) != cudaSuccess) ms[k] = 0;
    cudaGetLastError();
    ctx->timing[0] = ms[0] + ms[1] + ms[2] + ms[3];
    for (int k = 0; k < 4; k++) ctx->timing[k + 1] = ms[k];
    ctx->have_forward = true;
    if (!std::isfinite(res->em) || !std::isfinite(res->ep)) {
        ctx->err = "non-finite energy";
        return AMG_ERR_NAN;
    }
    if (status != AMG_OK) ctx->err = "PCG did not reach poleps within politer iterations";
    return status;
}

void release(amg_ctx* ctx) {
    if (ctx->rb) { cudaFreeHost(ctx->rb); ctx->rb = nullptr; }
    if (ctx->rb_grad) { cudaFreeHost(ctx->rb_grad); ctx->rb_grad = nullptr; }
    for (auto& e : ctx->rbev)
        if (e) { cudaEventDestroy(e); e = nullptr; }
    for (auto& e : ctx->rbevm)
        if (e) { cudaEventDestroy(e); e = nullptr; }
    if (ctx->gm_ready) { cudaEventDestroy(ctx->gm_ready); ctx->gm_ready = nullptr; }
    if (ctx->rbst) { cudaStreamDestroy(ctx->rbst); ctx->rbst = nullptr; }
    if (ctx->adj_host) { cudaFreeHost(ctx->adj_host); ctx->adj_host = nullptr; }
    double** dbl[] = {&ctx->pole13, &ctx->pol, &ctx->thole, &ctx->pdamp, &ctx->xyz, &ctx->rp10, &ctx->Ed, &ctx->Ep,
                      &ctx->ud, &ctx->up, &ctx->rd, &ctx->rp, &ctx->zd, &ctx->zp, &ctx->pd, &ctx->pp, &ctx->Apd,
                      &ctx->App, &ctx->Fd, &ctx->Fp, &ctx->resd, &ctx->scal, &ctx->eacc, &ctx->grad_m, &ctx->grad_p,
                      &ctx->trq_m, &ctx->trq_p, &ctx->aem, &ctx->aep, &ctx->phiM, &ctx->phiU, &ctx->phiU4,
                      &ctx->uopt};
    for (double** p : dbl) dfree(*p);
    int** ints[] = {&ctx->zax, &ctx->xax, &ctx->yax, &ctx->axe, &ctx->mol, &ctx->ids, &ctx->sids, &ctx->cstart,
                    &ctx->cend, &ctx->nbr, &ctx->nnb, &ctx->overflow, &ctx->xoff, &ctx->xidx};
    dfree(ctx->xrange);
    for (int** p : ints) dfree(*p);
    dfree(ctx->keys);
    dfree(ctx->skeys);
    dfree(ctx->rank);
    dfree(ctx->cnb);
    dfree(ctx->sdt);
    dfree(ctx->spos);
    dfree(ctx->cnt);
    dfree(ctx->sp);
    if (ctx->cubtmp) cudaFree(ctx->cubtmp);
    ctx->cubtmp = nullptr;
    dfree(ctx->af.at); dfree(ctx->af.u4); dfree(ctx->ad.at); dfree(ctx->ad.u4);
    dfree(ctx->af.atS); dfree(ctx->ad.atS);
    dfree(ctx->af.p4); dfree(ctx->ad.p4); dfree(ctx->af.c0); dfree(ctx->ad.c0);
    dfree(ctx->af.s4); dfree(ctx->ad.s4); dfree(ctx->af.cu0); dfree(ctx->ad.cu0);
    dfree(ctx->nbru); dfree(ctx->nnbu);
    pme_destroy(ctx->pmf);
    pme_destroy(ctx->pmd);
    for (auto& e : ctx->ev)
        if (e) { cudaEventDestroy(e); e = nullptr; }
    for (int k = 0; k < 3; k++) {
        if (ctx->efork[k]) { cudaEventDestroy(ctx->efork[k]); ctx->efork[k] = nullptr; }
        if (ctx->ejoin[k]) { cudaEventDestroy(ctx->ejoin[k]); ctx->ejoin[k] = nullptr; }
        if (ctx->side[k]) { cudaStreamDestroy(ctx->side[k]); ctx->side[k] = nullptr; }
    }
    if (ctx->gexec) { cudaGraphExecDestroy(ctx->gexec); ctx->gexec = nullptr; }
    if (ctx->adj_gexec) { cudaGraphExecDestroy(ctx->adj_gexec); ctx->adj_gexec = nullptr; }
    dfree(ctx->iter);
    dfree(ctx->cont);
    dfree(ctx->blk_done);
    dfree(ctx->flushbuf);
    dfree(ctx->adj); dfree(ctx->adj_pot); dfree(ctx->adj_n); dfree(ctx->adj_vec); dfree(ctx->adj_phi);
    dfree(ctx->adj_dpole);
    dfree(ctx->adj_opt);
    dfree(ctx->pred_hist); dfree(ctx->pred_state);
    dfree(ctx->pcore); dfree(ctx->palpha); dfree(ctx->dq); dfree(ctx->cfpot);
    dfree(ctx->bonds); dfree(ctx->bflux); dfree(ctx->angles); dfree(ctx->aflux);
    if (ctx->erot) { cudaEventDestroy(ctx->erot); ctx->erot = nullptr; }
    if (ctx->st) { cudaStreamDestroy(ctx->st); ctx->st = nullptr; }
    if (ctx->st2) { cudaStreamDestroy(ctx->st2); ctx->st2 = nullptr; }
}

// Damping polynomials of the charge-penetration densities: Q_0 the base of
// each family, Q_{n+1} = Q_n + x (Q_n - Q_n') / (2n + 1), the relation that
// makes B_n = bare_n (1 - Q_n(x) e^{-x}) the radial hierarchy of the base
// potential (see kernels_cp.cuh)
CpTables cp_tables(int pentype) {
    CpTables T{};
    T.pentype = pentype;
    auto family = [](std::initializer_list<double> base, double (&out)[6][kCpTerms]) {
        for (auto& row : out)
            for (double& c : row) c = 0.0;
        int j = 0;
        for (double c : base) out[0][j++] = c;
        for (int n = 0; n < 5; n++) {
            for (int q = 0; q < kCpTerms; q++) out[n + 1][q] = out[n][q];
            for (int q = 0; q + 1 < kCpTerms; q++) {
                const double qmd = out[n][q] - (q + 1) * out[n][q + 1];  // (Q - Q') at x^q
                out[n + 1][q + 1] += qmd / (2 * n + 1);
            }
        }
    };
    family({1.0, 0.5}, T.f1);
    family({1.0}, T.f2);
    family({1.0, 11.0 / 16, 3.0 / 16, 1.0 / 48}, T.e1);
    return T;
}

int create_impl(amg_ctx* ctx, const amg_params* P) {
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        ctx->err = "no CUDA device";
        return AMG_ERR_NO_DEVICE;
    }
    if (P->device < 0 || P->device >= ndev) {
        ctx->err = "device ordinal out of range";
        return AMG_ERR_BAD_ARG;
    }
    CK(cudaSetDevice(P->device));
    cudaDeviceProp prop;
    CK(cudaGetDeviceProperties(&prop, P->device));
    ctx->num_sms = prop.multiProcessorCount;
    if (prop.major < 10) {
        ctx->err = "libamoeba_gpu is built for sm_100a (B200)";
        return AMG_ERR_NO_DEVICE;
    }
    const int n = P->n;
    ctx->n = n;
    ctx->device = P->device;
    ctx->prec = P->precision;
    ctx->ewald = P->use_ewald;
    ctx->bounds = P->use_bounds;
    ctx->aewald = P->aewald;
    ctx->cut = P->cutoff;
    ctx->f = P->electric / P->dielec;
    ctx->debye = P->debye;
    ctx->poleps = P->poleps;
    ctx->politer = P->politer;
    ctx->guess = P->pcg_guess;
    ctx->has_pol = P->polarity != nullptr && P->poltyp != AMG_POL_NONE;
    ctx->poltyp = ctx->has_pol ? P->poltyp : AMG_POL_NONE;
    ctx->sparse_prec = ctx->has_pol && ctx->poltyp == AMG_POL_MUTUAL && P->pcg_prec != 0;
    ctx->usolvcut = std::min(P->usolvcut, P->cutoff);
    ctx->cell_shape = P->cell_shape;
    for (int a = 0; a < 3; a++) ctx->K[a] = P->nfft[a];
    // the solve's streams at the highest priority, the permanent-multipole
    // force stream at the lowest: its blocks fill what the solve leaves idle
    int plo = 0, phi = 0;
    CK(cudaDeviceGetStreamPriorityRange(&plo, &phi));
    const int pmain = phi;
    CK(cudaStreamCreateWithPriority(&ctx->st, cudaStreamNonBlocking, pmain));
    CK(cudaStreamCreateWithPriority(&ctx->st2, cudaStreamNonBlocking, pmain));
    for (int k = 0; k < 3; k++) {
        CK(cudaStreamCreateWithPriority(&ctx->side[k], cudaStreamNonBlocking, k == kMpoleSide ? plo : pmain));
        CK(cudaEventCreateWithFlags(&ctx->efork[k], cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&ctx->ejoin[k], cudaEventDisableTiming));
    }
    if (const char* g = getenv("AMG_NO_GRAPH")) ctx->use_graphs = !(g[0] == '1');
    ctx->lpa = 8;  // lanes per site (8 measured fastest at 12k and 98k sites)
    if (const char* l = getenv("AMG_LPA")) ctx->lpa = atoi(l);
    if (ctx->lpa != 8 && ctx->lpa != 16 && ctx->lpa != 32) ctx->lpa = 16;
    dalloc(ctx, ctx->iter, 1);
    dalloc(ctx, ctx->cont, 1);
    dalloc(ctx, ctx->blk_done, 1);
    CK(cudaMemset(ctx->blk_done, 0, sizeof(int)));
    CK(cudaMemset(ctx->iter, 0, sizeof(int)));
    if (ctx->has_pol)
        for (int i = 0; i < n; i++) ctx->npolar += P->polarity[i] > 0;
    if (ctx->poltyp == AMG_POL_OPT) {  // src/md/kpolar.cpp:226-236 restated
        for (int k = 1; k <= AMG_MAX_OPT; k++)
            if (P->opt_coef[k] != 0.0) ctx->optorder = k;
        for (int k = 0; k <= ctx->optorder; k++)
            for (int j = k; j <= ctx->optorder; j++) ctx->copm.c[k] += P->opt_coef[j];
        dalloc(ctx, ctx->uopt, (size_t)(ctx->optorder + 1) * 6 * n + 3 * (size_t)n);
    }
    for (auto& e : ctx->ev) CK(cudaEventCreate(&e));
    CK(cudaEventCreateWithFlags(&ctx->erot, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&ctx->gm_ready, cudaEventDisableTiming));
    CK(cudaStreamCreateWithFlags(&ctx->rbst, cudaStreamNonBlocking));
    upload(ctx, ctx->pole13, P->pole, 13 * (size_t)n);
    upload(ctx, ctx->zax, P->zaxis, n);
    upload(ctx, ctx->xax, P->xaxis, n);
    upload(ctx, ctx->yax, P->yaxis, n);
    upload(ctx, ctx->axe, P->polaxe, n);
    if (P->molcule) upload(ctx, ctx->mol, P->molcule, n);
    std::vector<double> zeros(n, 0.0);
    upload(ctx, ctx->pol, ctx->has_pol ? P->polarity : zeros.data(), n);
    upload(ctx, ctx->thole, ctx->has_pol ? P->thole : zeros.data(), n);
    upload(ctx, ctx->pdamp, ctx->has_pol ? P->pdamp : zeros.data(), n);
    std::vector<ScaledPair> sp = build_scaled(P);
    ctx->nsp = (int)sp.size();
    {
        // scaled partners of each site (CSR); si/sk locate each pair in the
        // two rows so the stored-coefficient rows can append them
        std::vector<int> off(n + 1, 0), idx(2 * sp.size() + 1);
        for (const ScaledPair& q : sp) { off[q.i + 1]++; off[q.k + 1]++; }
        for (int i = 0; i < n; i++) off[i + 1] += off[i];
        std::vector<int> fill(off.begin(), off.end() - 1);
        for (ScaledPair& q : sp) {
            q.si = fill[q.i] - off[q.i];
            idx[fill[q.i]++] = q.k;
            q.sk = fill[q.k] - off[q.k];
            idx[fill[q.k]++] = q.i;
        }
        upload(ctx, ctx->xoff, off.data(), off.size());
        upload(ctx, ctx->xidx, idx.data(), idx.size());
        std::vector<int2> xr(n, make_int2(INT_MAX, -1));  // empty range when no partners
        for (int i = 0; i < n; i++)
            for (int q = off[i]; q < off[i + 1]; q++) {
                xr[i].x = std::min(xr[i].x, idx[q]);
                xr[i].y = std::max(xr[i].y, idx[q]);
            }
        upload(ctx, ctx->xrange, xr.data(), xr.size());
    }
    upload(ctx, ctx->sp, sp.data(), sp.size());
    dalloc(ctx, ctx->xyz, 3 * (size_t)n);
    dalloc(ctx, ctx->rp10, 10 * (size_t)n);
    dalloc(ctx, ctx->ad.at, n);
    dalloc(ctx, ctx->ad.atS, n);
    dalloc(ctx, ctx->ad.u4, 2 * (size_t)n);
    dalloc(ctx, ctx->ad.p4, 2 * (size_t)n);
    if (ctx->prec == AMG_PREC_MIXED) {
        dalloc(ctx, ctx->af.at, n);
        dalloc(ctx, ctx->af.atS, n);
        dalloc(ctx, ctx->af.u4, 2 * (size_t)n);
        dalloc(ctx, ctx->af.p4, 2 * (size_t)n);
    }
    double** vecs[] = {&ctx->Ed, &ctx->Ep, &ctx->ud, &ctx->up, &ctx->rd, &ctx->rp, &ctx->zd, &ctx->zp, &ctx->pd,
                       &ctx->pp, &ctx->Apd, &ctx->App, &ctx->Fd, &ctx->Fp, &ctx->resd, &ctx->grad_m, &ctx->grad_p,
                       &ctx->trq_m, &ctx->trq_p};
    for (double** p : vecs) {
        dalloc(ctx, *p, 3 * (size_t)n);
        CK(cudaMemset(*p, 0, sizeof(double) * 3 * n));
    }
    if (P->pentype != AMG_PEN_NONE || P->cflux) {
        ctx->cp_mode = true;
        ctx->cpt = cp_tables(P->pentype);
        if (P->pentype != AMG_PEN_NONE) {
            upload(ctx, ctx->pcore, P->pcore, n);
            upload(ctx, ctx->palpha, P->palpha, n);
        }
        if (P->cflux) {
            ctx->cflux = true;
            ctx->nbond = P->nbond;
            ctx->nangle = P->nangle;
            std::vector<int2> b(std::max(1, P->nbond));
            std::vector<double2> bf(std::max(1, P->nbond));
            for (int q = 0; q < P->nbond; q++) {
                b[q] = make_int2(P->bond_atoms[2 * q], P->bond_atoms[2 * q + 1]);
                bf[q] = make_double2(P->bond_flux[2 * q], P->bond_flux[2 * q + 1]);
            }
            upload(ctx, ctx->bonds, b.data(), b.size());
            upload(ctx, ctx->bflux, bf.data(), bf.size());
            upload(ctx, ctx->angles, P->nangle ? P->angle_atoms : nullptr, 3 * (size_t)std::max(1, P->nangle));
            upload(ctx, ctx->aflux, P->nangle ? P->angle_flux : nullptr, 7 * (size_t)std::max(1, P->nangle));
            dalloc(ctx, ctx->dq, n);
            dalloc(ctx, ctx->cfpot, n);
        }
    }
    dalloc(ctx, ctx->aem, n);
    dalloc(ctx, ctx->aep, n);
    dalloc(ctx, ctx->scal, 16);
    dalloc(ctx, ctx->eacc, kEacc);
    dalloc(ctx, ctx->cnt, 4);
    dalloc(ctx, ctx->phiM, 20 * (size_t)n);
    CK(cudaMemset(ctx->phiM, 0, sizeof(double) * 20 * n));
    if (ctx->has_pol) {
        dalloc(ctx, ctx->phiU, 40 * (size_t)n);
        dalloc(ctx, ctx->phiU4, 8 * (size_t)n);
    }
    return AMG_OK;
}

int validate(const amg_params* P, std::string& why) {
    if (!P || P->n <= 0 || !P->pole || !P->zaxis || !P->xaxis || !P->yaxis || !P->polaxe) {
        why = "missing required arrays";
        return AMG_ERR_BAD_ARG;
    }
    if (P->precision != AMG_PREC_FP64 && P->precision != AMG_PREC_MIXED) {
        why = "precision must be AMG_PREC_FP64 or AMG_PREC_MIXED";
        return AMG_ERR_BAD_ARG;
    }
    if (P->cutoff <= 0 || P->electric <= 0 || P->dielec <= 0) {
        why = "cutoff, electric and dielec must be positive";
        return AMG_ERR_BAD_ARG;
    }
    if (P->use_ewald) {
        if (!P->use_bounds) { why = "Ewald needs a periodic box"; return AMG_ERR_BAD_ARG; }
        if (P->bsorder != kOrder) { why = "only B-spline order 5 is compiled"; return AMG_ERR_UNSUPPORTED; }
        if (P->aewald <= 0 || P->nfft[0] < 8 || P->nfft[1] < 8 || P->nfft[2] < 8) {
            why = "Ewald alpha and PME grid (>= 8) required";
            return AMG_ERR_BAD_ARG;
        }
    }
    if (P->polarity && P->poltyp != AMG_POL_NONE && (!P->thole || !P->pdamp)) {
        why = "polarization needs thole and pdamp";
        return AMG_ERR_BAD_ARG;
    }
    if (P->poltyp == AMG_POL_OPT) {
        int order = 0;
        for (int k = 1; k <= AMG_MAX_OPT; k++)
            if (P->opt_coef[k] != 0.0) order = k;
        if (order < 1) {
            why = "OPT needs a nonzero coefficient of order 1 or more";
            return AMG_ERR_BAD_ARG;
        }
    } else if (P->poltyp != AMG_POL_NONE && P->poltyp != AMG_POL_MUTUAL && P->poltyp != AMG_POL_DIRECT) {
        why = "unknown polarization model";
        return AMG_ERR_UNSUPPORTED;
    }
    if (P->pcg_prec && !(P->usolvcut > 0)) {
        why = "the sparse preconditioner needs usolvcut > 0";
        return AMG_ERR_BAD_ARG;
    }
    if (P->cell_shape < AMG_CELL_FROM_ANGLES || P->cell_shape > AMG_CELL_DODECAHEDRON) {
        why = "unknown cell shape";
        return AMG_ERR_BAD_ARG;
    }
    if (P->pentype != AMG_PEN_NONE || P->cflux) {
        // the reference has both only in its non-Ewald multipole mode
        if (P->use_ewald || (P->polarity && P->poltyp != AMG_POL_NONE)) {
            why = "charge penetration and charge flux need the non-Ewald multipole mode without polarization";
            return AMG_ERR_UNSUPPORTED;
        }
        if (P->pentype < AMG_PEN_NONE || P->pentype > AMG_PEN_GORDON2) {
            why = "unknown charge penetration type";
            return AMG_ERR_BAD_ARG;
        }
        if (P->pentype != AMG_PEN_NONE && (!P->pcore || !P->palpha)) {
            why = "charge penetration needs pcore and palpha";
            return AMG_ERR_BAD_ARG;
        }
        if (P->cflux) {
            if (P->nbond < 0 || P->nangle < 0 || (P->nbond && (!P->bond_atoms || !P->bond_flux)) ||
                (P->nangle && (!P->angle_atoms || !P->angle_flux))) {
                why = "charge flux needs its bond and angle arrays";
                return AMG_ERR_BAD_ARG;
            }
            for (int q = 0; q < 2 * P->nbond; q++)
                if (P->bond_atoms[q] < 0 || P->bond_atoms[q] >= P->n) { why = "bond atom out of range"; return AMG_ERR_BAD_ARG; }
            for (int q = 0; q < 3 * P->nangle; q++)
                if (P->angle_atoms[q] < 0 || P->angle_atoms[q] >= P->n) { why = "angle atom out of range"; return AMG_ERR_BAD_ARG; }
        }
    }
    for (int i = 0; i < P->n; i++) {
        int ft = P->polaxe[i];
        if (ft < AMG_FRAME_NONE || ft > AMG_FRAME_THREEFOLD) { why = "bad frame type"; return AMG_ERR_BAD_ARG; }
        if (ft != AMG_FRAME_NONE) {
            int need[3] = {P->zaxis[i], ft == AMG_FRAME_ZONLY ? 1 : P->xaxis[i],
                           (ft == AMG_FRAME_ZBISECT || ft == AMG_FRAME_THREEFOLD) ? std::abs(P->yaxis[i]) : 1};
            for (int v : need)
                if (v < 1 || v > P->n) { why = "frame atom out of range"; return AMG_ERR_BAD_ARG; }
        }
    }
    return AMG_OK;
}

// the adjoint pair kernel's five vectors of site i, in precision R, at the
// site's cell-order position rank[i]
template <class R>
__global__ void k_adj_pack(int n, const int* __restrict__ rank, const double* __restrict__ vbar,
                           const double* __restrict__ p1, const double* __restrict__ q1, const double* __restrict__ p2,
                           const double* __restrict__ q2, R4<R>* __restrict__ vec) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double* src[5] = {vbar, p1, q1, p2, q2};
    const size_t o = 5 * (size_t)rank[i];
    for (int k = 0; k < 5; k++)
        vec[o + k] = make_r4<R>((R)src[k][3 * i], (R)src[k][3 * i + 1], (R)src[k][3 * i + 2], R(0));
}

// bulk real-space adjoint pairs in precision R (the forward's pair
// precision): the vectors packed in cell order, then the pair kernel
template <class R>
void adjoint_pairs(amg_ctx* ctx, cudaStream_t s, const double* vbar, const double* p1, const double* q1,
                   const double* p2, const double* q2, int mutual, double cm, double* grad, double* trq,
                   double* dpd, double* dth) {
    const int n = ctx->n;
    Atoms<R>& A = atoms_of<R>(ctx);
    R4<R>* vec = reinterpret_cast<R4<R>*>(ctx->adj_vec);  // [n][5] double4 of room
    k_adj_pack<R><<<nblk(n), kThreads, 0, s>>>(n, ctx->rank, vbar, p1, q1, p2, q2, vec);
    KCHECK();
    LPA_DISPATCH(ctx->lpa, {
        if (ctx->ewald)
            k_adjoint_pair<R, true, L><<<nblk((size_t)n * L), kThreads, 0, s>>>(
                n, ctx->sids, A.atS, vec, ctx->bx, (R)ctx->aewald, ctx->cnb, ctx->cap, ctx->nnb, mutual, cm, grad, trq,
                ctx->adj_pot, dpd, dth);
        else
            k_adjoint_pair<R, false, L><<<nblk((size_t)n * L), kThreads, 0, s>>>(
                n, ctx->sids, A.atS, vec, ctx->bx, R(0), ctx->cnb, ctx->cap, ctx->nnb, mutual, cm, grad, trq,
                ctx->adj_pot, dpd, dth);
    });
    KCHECK();
}

__global__ void k_scale3(int n, const double* __restrict__ pol, const double* __restrict__ g, double* __restrict__ w) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (int c = 0; c < 3; c++) w[3 * i + c] = pol[i] * g[3 * i + c];
}

// dst[0, cnt) = src[0, cnt); nothing for a null dst
void host_copy(double* dst, const double* src, size_t cnt) {
    if (dst) std::memcpy(dst, src, sizeof(double) * cnt);
}

// the adjoint solve A w = g for both right-hand sides, as the forward solves
// A u = E: PCG in the context's precision on the forward's stored coefficient
// rows and grids (same coordinates), then the FP64 correction sweep.  The
// caller has pointed the context's field and dipole vectors at g and w, with
// w = alpha g as the starting guess.
template <class R>
bool capture_adjoint(amg_ctx* ctx) {
    cudaStream_t s = ctx->st;
    cudaGraph_t graph = nullptr;
    const long long k0 = ctx->kcount;
    auto fail = [&](cudaError_t) {
        cudaStreamCaptureStatus st;
        if (cudaStreamIsCapturing(s, &st) == cudaSuccess && st != cudaStreamCaptureStatusNone) {
            cudaGraph_t g2 = nullptr;
            cudaStreamEndCapture(s, &g2);
            if (g2) cudaGraphDestroy(g2);
        }
        cudaGetLastError();
        ctx->kcount = k0;
        return false;
    };
    cudaError_t e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return fail(e);
    try {
        const cudaGraphNode_t* deps = nullptr;
        size_t ndeps = 0;
        cudaStreamCaptureStatus cs;
        e = cudaStreamGetCaptureInfo(s, &cs, nullptr, &graph, &deps, &ndeps);
        if (e != cudaSuccess) return fail(e);
        cudaGraphConditionalHandle h;
        e = cudaGraphConditionalHandleCreate(&h, graph, 0, 0);
        if (e != cudaSuccess) return fail(e);
        enqueue_pcg_init<R>(ctx, s, h, 1, true);
        e = cudaStreamGetCaptureInfo(s, &cs, nullptr, &graph, &deps, &ndeps);
        if (e != cudaSuccess) return fail(e);
        cudaGraphNodeParams cp = {};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = h;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        cudaGraphNode_t cnode;
        e = cudaGraphAddNode(&cnode, graph, deps, ndeps, &cp);
        if (e != cudaSuccess) return fail(e);
        cudaGraph_t body = cp.conditional.phGraph_out[0];
        e = cudaStreamUpdateCaptureDependencies(s, &cnode, 1, cudaStreamSetCaptureDependencies);
        if (e != cudaSuccess) return fail(e);
        e = cudaStreamBeginCaptureToGraph(ctx->st2, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) return fail(e);
        enqueue_pcg_iter<R>(ctx, ctx->st2, h, 1);
        e = cudaStreamEndCapture(ctx->st2, &body);
        if (e != cudaSuccess) return fail(e);
        enqueue_sweep(ctx, s);
    } catch (Fail&) {
        return fail(cudaGetLastError());
    }
    e = cudaStreamEndCapture(s, &graph);
    if (e != cudaSuccess) return fail(e);
    if (ctx->adj_gexec) cudaGraphExecDestroy(ctx->adj_gexec);
    ctx->adj_gexec = nullptr;
    e = cudaGraphInstantiate(&ctx->adj_gexec, graph, cudaGraphInstantiateFlagUseNodePriority);
    cudaGraphDestroy(graph);
    ctx->kcount = k0;
    if (e != cudaSuccess) {
        ctx->adj_gexec = nullptr;
        cudaGetLastError();
        return false;
    }
    ctx->adj_gen = ctx->fwd_gen;
    return true;
}

template <class R>
void adjoint_solve(amg_ctx* ctx, cudaStream_t s) {
    // periodic systems: one graph launch, the loop's control on the device
    // (captured with the vectors the caller set; they are the same buffers on
    // every call)
    if (ctx->use_graphs && ctx->bounds && ctx->gexec) {
        if (!ctx->adj_gexec || ctx->adj_gen != ctx->fwd_gen) capture_adjoint<R>(ctx);
        if (ctx->adj_gexec) {
            CK(cudaGraphLaunch(ctx->adj_gexec, s));
            return;
        }
    }
    enqueue_pcg_init<R>(ctx, s, 0, 0, true);
    int cont = 1;
    while (true) {
        CK(cudaMemcpyAsync(&cont, ctx->cont, sizeof(int), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        if (!cont) break;
        enqueue_pcg_iter<R>(ctx, s, 0, 0);
    }
    enqueue_sweep(ctx, s);
}

// amg_backward: the adjoint solve in the context's precision (above), every
// other term in FP64 (see kernels_adjoint.cuh for the algebra)
int backward_impl(amg_ctx* ctx, const amg_cotangents* cot, amg_param_grads* gr) {
    const int n = ctx->n;
    cudaStream_t s = ctx->st;
    const size_t n3 = 3 * (size_t)n;
    if (!ctx->adj) {
        dalloc(ctx, ctx->adj, 11 * n3);
        dalloc(ctx, ctx->adj_pot, 10 * (size_t)n);
        dalloc(ctx, ctx->adj_n, 4 * (size_t)n);
        dalloc(ctx, ctx->adj_vec, 5 * (size_t)n);
        dalloc(ctx, ctx->adj_phi, 3 * 2 * 20 * (size_t)n);
        dalloc(ctx, ctx->adj_dpole, 13 * (size_t)n);
        CK(cudaMallocHost((void**)&ctx->adj_host, sizeof(double) * 25 * (size_t)n));
    }
    double *gd = ctx->adj, *gp = gd + n3, *wd = gp + n3, *wp = wd + n3, *bd = wp + n3, *bp = bd + n3,
           *vbar = bp + n3, *mwp = vbar + n3, *grad = mwp + n3, *trq = grad + n3, *zeros = trq + n3;
    double *dpd = ctx->adj_n, *dth = dpd + n, *dpol = dth + n;
    const bool have_g = cot->d_uind || cot->d_uinp;
    const bool iter = iterative(ctx);
    const bool opt = ctx->poltyp == AMG_POL_OPT && ctx->npolar > 0;
    const int K = ctx->optorder;
    if (opt && !ctx->adj_opt) dalloc(ctx, ctx->adj_opt, (size_t)(2 * K + 4) * n3);
    // FP64 copies of the sites (also in cell order), stencils and T coefficients
    rotate_and_pack<double>(ctx, s);
    k_gather_atoms<double><<<nblk(n), kThreads, 0, s>>>(n, ctx->sids, ctx->ad.at, ctx->ad.atS);
    KCHECK();
    if (ctx->ewald) {
        pme_prepare<double>(ctx, pme_of<double>(ctx));
        pme_stencils<double>(ctx, s);
    }
    k_zero<double><<<nblk(2 * n3, 256), 256, 0, s>>>(wd, 2 * n3);
    KCHECK();
    k_zero<double><<<nblk(n3, 256), 256, 0, s>>>(zeros, n3);
    KCHECK();
    if (have_g && ctx->has_pol) {
        // adjoint solve A w = g for both right-hand sides (the forward's PCG)
        double* hg = ctx->adj_host;  // both cotangents through the pinned staging buffer
        if (cot->d_uind) std::memcpy(hg, cot->d_uind, sizeof(double) * n3);
        else std::fill(hg, hg + n3, 0.0);
        if (cot->d_uinp) std::memcpy(hg + n3, cot->d_uinp, sizeof(double) * n3);
        else std::fill(hg + n3, hg + 2 * n3, 0.0);
        CK(cudaMemcpyAsync(gd, hg, sizeof(double) * 2 * n3, cudaMemcpyHostToDevice, s));  // gp follows gd
        if (ctx->poltyp == AMG_POL_DIRECT) {
            k_scale3<<<nblk(n), kThreads, 0, s>>>(n, ctx->pol, gd, wd);
            KCHECK();
            k_scale3<<<nblk(n), kThreads, 0, s>>>(n, ctx->pol, gp, wp);
            KCHECK();
        } else if (opt) {
            // orders w^(k) = (alpha T)^k alpha g of both cotangents, and
            // w = S g = sum_k c_k w^(k) (no solve: S is the OPT polynomial)
            double* wo = ctx->adj_opt;
            k_scale3<<<nblk(n), kThreads, 0, s>>>(n, ctx->pol, gd, wo);
            KCHECK();
            k_scale3<<<nblk(n), kThreads, 0, s>>>(n, ctx->pol, gp, wo + n3);
            KCHECK();
            for (int k = 1; k <= K; k++) {
                const double* vd = wo + (size_t)(2 * k - 2) * n3;
                matvec<double>(ctx, s, vd, vd + n3, ctx->Apd, ctx->App);
                k_opt_step<<<nblk(n3), kThreads, 0, s>>>((int)n3, ctx->pol, vd, vd + n3, ctx->Apd, ctx->App, 0.0,
                                                         wo + (size_t)(2 * k) * n3, wo + (size_t)(2 * k + 1) * n3,
                                                         zeros, zeros);
                KCHECK();
            }
            k_opt_combine<<<nblk(n3), kThreads, 0, s>>>((int)n3, K, ctx->copm, wo, wd, wp);
            KCHECK();
        } else if (iter) {
            double *Ed = ctx->Ed, *Ep = ctx->Ep, *ud = ctx->ud, *up = ctx->up;
            ctx->Ed = gd; ctx->Ep = gp; ctx->ud = wd; ctx->up = wp;
            int guess = ctx->guess;
            ctx->guess = 1;
            k_scale3<<<nblk(n), kThreads, 0, s>>>(n, ctx->pol, gd, wd);
            KCHECK();
            k_scale3<<<nblk(n), kThreads, 0, s>>>(n, ctx->pol, gp, wp);
            KCHECK();
            bool ok = true;
            try {
                if (ctx->prec == AMG_PREC_MIXED)
                    adjoint_solve<float>(ctx, s);
                else
                    adjoint_solve<double>(ctx, s);
            } catch (Fail&) {
                ok = false;
            }
            ctx->Ed = Ed; ctx->Ep = Ep; ctx->ud = ud; ctx->up = up;
            ctx->guess = guess;
            if (!ok) throw Fail{AMG_ERR_CUDA};
        }
    }
    const double c = cot->d_energy, f = ctx->f, cf = c * f;
    k_adj_vectors<<<nblk(n), kThreads, 0, s>>>(n, cf, ctx->has_pol ? ctx->ud : zeros, ctx->has_pol ? ctx->up : zeros,
                                               wd, wp, bd, bp, vbar, mwp, ctx->pol, dpol);
    KCHECK();
    if (opt) {
        if (!(have_g && ctx->has_pol)) {  // no dipole cotangents: all orders w^(k) vanish
            k_zero<double><<<nblk((size_t)2 * (K + 1) * n3, 256), 256, 0, s>>>(ctx->adj_opt, (size_t)2 * (K + 1) * n3);
            KCHECK();
        }
        k_opt_adj_diag<<<nblk(n), kThreads, 0, s>>>(n, K, ctx->copm, cf, ctx->pol, ctx->adj_opt, ctx->uopt, dpol);
        KCHECK();
    }
    k_zero<double><<<nblk(2 * n3, 256), 256, 0, s>>>(grad, 2 * n3);
    KCHECK();
    k_zero<double><<<nblk(10 * (size_t)n, 256), 256, 0, s>>>(ctx->adj_pot, 10 * (size_t)n);
    KCHECK();
    k_zero<double><<<nblk(2 * (size_t)n, 256), 256, 0, s>>>(dpd, 2 * (size_t)n);
    KCHECK();
    const int mutual = ctx->poltyp == AMG_POL_MUTUAL;
    const bool mixed = ctx->prec == AMG_PREC_MIXED;
    // potentials (and derivatives, 20) of two dipole sets from the PME grid
    auto adj_pme = [&](const double* a, const double* b, double* ph) {
        if (mixed) pme_dipoles<float, 20>(ctx, s, a, b, ph);
        else pme_dipoles<double, 20>(ctx, s, a, b, ph);
    };
    if (mixed)
        adjoint_pairs<float>(ctx, s, vbar, bd, ctx->ud, mwp, ctx->up, mutual, cf, grad, trq, dpd, dth);
    else
        adjoint_pairs<double>(ctx, s, vbar, bd, ctx->ud, mwp, ctx->up, mutual, cf, grad, trq, dpd, dth);
    if (ctx->nsp) {
        k_adjoint_scaled<<<nblk(ctx->nsp), kThreads, 0, s>>>(ctx->nsp, ctx->sp, ctx->xyz, ctx->rp10, ctx->pdamp,
                                                            ctx->thole, ctx->bx, ctx->cut * ctx->cut, ewald_alpha(ctx),
                                                            bd, bp, bd, ctx->ud, mwp, ctx->up, mutual, cf, grad, trq,
                                                            ctx->adj_pot, dpd, dth);
        KCHECK();
    }
    double qtot = 0;
    if (ctx->ewald) {
        // permanent potentials (overwrite the forward's phiM), in the forward's
        // grid precision like the dipole potentials below
        if (mixed) pme_mpole<float>(ctx, s);
        else pme_mpole<double>(ctx, s);
        double* ph = ctx->adj_phi;
        const size_t blk = 2 * 20 * (size_t)n;
        adj_pme(vbar, bd, ph);              // phi of vbar, P1
        adj_pme(ctx->ud, ctx->up, ph + blk);  // phi of Q1, Q2
        adj_pme(mwp, zeros, ph + 2 * blk);    // phi of P2
        const size_t one = 20 * (size_t)n;
        k_adjoint_recip<<<nblk(n), kThreads, 0, s>>>(n, ctx->rp10, ctx->phiM, ph, ph + one, ph + blk, ph + 2 * blk,
                                                     ph + blk + one, vbar, bd, ctx->ud, mwp, ctx->up, mutual,
                                                     self_coef(ctx), ctx->aewald, cf, grad, trq, ctx->adj_pot);
        KCHECK();
        qtot = ctx->qtot;  // the forward's net charge (monopoles do not rotate)
    }
    if (opt) {
        // OPT dipole-dipole terms: the pairs (-V1_b, u_d^(b)) and (-V2_b,
        // u_p^(b)) of U_u for b = 0..K-1, through the same adjoint kernels
        // with the multipole channels off (cm = 0, vbar = 0)
        double* P1 = ctx->adj_opt + (size_t)(2 * K + 2) * n3;
        double* P2 = P1 + n3;
        for (int b = 0; b < K; b++) {
            const double* Q1 = ctx->uopt + (size_t)(2 * b) * n3;
            const double* Q2 = Q1 + n3;
            k_opt_adj_cross<<<nblk(n3), kThreads, 0, s>>>((int)n3, K, b, ctx->copm, cf, ctx->adj_opt, ctx->uopt, P1, P2);
            KCHECK();
            if (mixed)
                adjoint_pairs<float>(ctx, s, zeros, P1, Q1, P2, Q2, 1, 0.0, grad, trq, dpd, dth);
            else
                adjoint_pairs<double>(ctx, s, zeros, P1, Q1, P2, Q2, 1, 0.0, grad, trq, dpd, dth);
            if (ctx->nsp) {
                k_adjoint_scaled<<<nblk(ctx->nsp), kThreads, 0, s>>>(
                    ctx->nsp, ctx->sp, ctx->xyz, ctx->rp10, ctx->pdamp, ctx->thole, ctx->bx, ctx->cut * ctx->cut,
                    ewald_alpha(ctx), zeros, zeros, P1, Q1, P2, Q2, 1, 0.0, grad, trq, ctx->adj_pot, dpd, dth);
                KCHECK();
            }
            if (ctx->ewald) {
                double* ph = ctx->adj_phi;
                const size_t blk = 2 * 20 * (size_t)n, one = 20 * (size_t)n;
                adj_pme(zeros, P1, ph);
                adj_pme(Q1, Q2, ph + blk);
                adj_pme(P2, zeros, ph + 2 * blk);
                k_adjoint_recip<<<nblk(n), kThreads, 0, s>>>(n, ctx->rp10, ctx->phiM, ph, ph + one, ph + blk,
                                                             ph + 2 * blk, ph + blk + one, zeros, P1, Q1, P2, Q2, 1,
                                                             self_coef(ctx), ctx->aewald, 0.0, grad, trq, ctx->adj_pot);
                KCHECK();
            }
        }
    }
    k_torque<<<nblk(n), kThreads, 0, s>>>(n, ctx->xyz, ctx->zax, ctx->xax, ctx->yax, ctx->axe, trq, grad, nullptr);
    KCHECK();
    k_pole_grad_local<<<nblk(n), kThreads, 0, s>>>(n, ctx->xyz, ctx->pole13, ctx->zax, ctx->xax, ctx->yax, ctx->axe,
                                                   ctx->adj_pot, ctx->adj_dpole);
    KCHECK();
    // net-charge term of the Ewald energy, -f pi Q^2 / (2 V alpha^2): dq_i
    double dq = 0;
    if (ctx->ewald) {
        double V = ctx->vol;
        dq = -cf * kPi * qtot / (V * ctx->aewald * ctx->aewald);
    }
    k_adj_finish<<<nblk(n), kThreads, 0, s>>>(n, dq, ctx->has_pol ? 1 : 0, ctx->pol, ctx->pdamp, dpd, dth, dpol,
                                              ctx->adj_dpole);
    KCHECK();
    // outputs through the pinned staging buffer: d_xyz [3n], d_pole [13n],
    // d_thole [n], d_polarity [n]
    double* h = ctx->adj_host;
    double *hx = h, *hpole = h + n3, *hth = hpole + 13 * (size_t)n, *hpol = hth + n;
    if (gr->d_xyz) CK(cudaMemcpyAsync(hx, grad, sizeof(double) * n3, cudaMemcpyDeviceToHost, s));
    if (gr->d_pole) CK(cudaMemcpyAsync(hpole, ctx->adj_dpole, sizeof(double) * 13 * n, cudaMemcpyDeviceToHost, s));
    if (gr->d_thole) CK(cudaMemcpyAsync(hth, dth, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
    if (gr->d_polarity) CK(cudaMemcpyAsync(hpol, dpol, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    host_copy(gr->d_xyz, hx, n3);
    host_copy(gr->d_pole, hpole, 13 * (size_t)n);
    host_copy(gr->d_thole, hth, n);
    host_copy(gr->d_polarity, hpol, n);
    return AMG_OK;
}

}  // namespace

extern "C" {

int amg_abi_version(void) { return AMG_ABI_VERSION; }

int amg_create(const amg_params* params, amg_ctx** out) {
    if (!out) return AMG_ERR_BAD_ARG;
    *out = nullptr;
    std::string why;
    int rc = validate(params, why);
    if (rc != AMG_OK) return rc;
    amg_ctx* ctx = new amg_ctx();
    try {
        rc = create_impl(ctx, params);
    } catch (Fail& f) {
        rc = f.code;
    }
    if (rc != AMG_OK) {
        release(ctx);
        delete ctx;
        return rc;
    }
    *out = ctx;
    return AMG_OK;
}

// true when no value is an infinity or a NaN (exponent bits not all set);
// branch-free, so the compiler vectorises it
static bool all_finite(const double* x, size_t count) {
    uint64_t bad = 0;
    for (size_t i = 0; i < count; i++) {
        uint64_t b;
        std::memcpy(&b, x + i, sizeof b);
        bad |= (uint64_t)((b & 0x7ff0000000000000ull) == 0x7ff0000000000000ull);
    }
    return bad == 0;
}

int amg_set_coords(amg_ctx* ctx, const double* xyz, const double box[6]) {
    if (!ctx || !xyz) return AMG_ERR_BAD_ARG;
    try {
        CK(cudaSetDevice(ctx->device));
        if (ctx->bounds) {
            if (!box || box[0] <= 0 || box[1] <= 0 || box[2] <= 0) {
                ctx->err = "periodic box lengths must be positive";
                return AMG_ERR_BAD_ARG;
            }
            Box nb = ctx->bx;
            if (!set_lattice(ctx, box, nb)) return AMG_ERR_BAD_ARG;
            // The dodecahedron's image (src/md/image.cpp:111-121) wraps z by
            // sqrt(2) c and moves corners by (a/2, a/2, c/sqrt(2)): a lattice
            // (the face-centred one whose cell is the rhombic dodecahedron)
            // only when c = a.  The reference's unitcell() sets c = sqrt(2) a
            // (src/md/unitcell.cpp:148), for which these translations form no
            // lattice and no Ewald sum exists; without Ewald the image is used
            // as it stands.
            if (ctx->ewald && nb.shape == 4 && std::fabs(box[2] - box[0]) > 1e-9 * box[0]) {
                ctx->err = "Ewald in a rhombic dodecahedron needs c = a (its minimum image is a lattice only then)";
                return AMG_ERR_UNSUPPORTED;
            }
            if (nb.shape != ctx->bx.shape) ctx->graph_dirty = true;
            for (int a = 3; a < 6; a++)
                if (ctx->box[a] != box[a]) ctx->graph_dirty = true;
            ctx->bx = nb;
            for (int a = 0; a < 3; a++)
                if (ctx->cut > 0.5 * box[a] + 1e-12) {
                    ctx->err = "cutoff exceeds half the box (minimum image)";
                    return AMG_ERR_BAD_ARG;
                }
            for (int a = 0; a < 3; a++)
                if (ctx->box[a] != box[a]) ctx->graph_dirty = true;
            for (int a = 0; a < 6; a++) ctx->box[a] = box[a];
            for (int a = 0; a < 3; a++) { ctx->bx.L[a] = box[a]; ctx->bx.iL[a] = 1.0 / box[a]; }
            set_frac(ctx);
        } else {
            for (int a = 0; a < 3; a++) { ctx->bx.L[a] = 0; ctx->bx.iL[a] = 0; }
        }
        // the copy is under way while the host checks the values (a non-finite
        // coordinate leaves the context without coordinates, and without the
        // forward evaluation a backward needs)
        ctx->have_coords = false;
        ctx->have_forward = false;
        CK(cudaMemcpyAsync(ctx->xyz, xyz, sizeof(double) * 3 * ctx->n, cudaMemcpyHostToDevice, ctx->st));
        if (!all_finite(xyz, 3 * (size_t)ctx->n)) {
            ctx->err = "non-finite coordinate";
            return AMG_ERR_NAN;
        }
        cell_grid(ctx, xyz);
        ctx->have_coords = true;
    } catch (Fail& f) {
        return f.code;
    }
    return AMG_OK;
}

int amg_forward(amg_ctx* ctx, int32_t flags, amg_results* res) {
    if (!ctx || !res) return AMG_ERR_BAD_ARG;
    if (!ctx->have_coords) {
        ctx->err = "amg_set_coords not called";
        return AMG_ERR_BAD_ARG;
    }
    if (flags & AMG_DO_VIRIAL) flags |= AMG_DO_GRADIENT;  // the virial needs the torques' frame forces
    try {
        CK(cudaSetDevice(ctx->device));
        if (ctx->prec == AMG_PREC_MIXED) return forward_impl<float>(ctx, flags, res);
        return forward_impl<double>(ctx, flags, res);
    } catch (Fail& f) {
        return f.code;
    }
}

int amg_backward(amg_ctx* ctx, const amg_cotangents* cot, amg_param_grads* grads) {
    if (!ctx || !cot || !grads) return AMG_ERR_BAD_ARG;
    if (!ctx->have_forward) {
        ctx->err = "amg_backward needs an amg_forward at the current coordinates";
        return AMG_ERR_BAD_ARG;
    }
    try {
        CK(cudaSetDevice(ctx->device));
        return backward_impl(ctx, cot, grads);
    } catch (Fail& f) {
        return f.code;
    }
}

int amg_bench(amg_ctx* ctx, int32_t flags, int32_t steps, int64_t flush_bytes, double* ms_steps,
              int64_t* launches) {
    if (!ctx || steps <= 0 || !ms_steps) return AMG_ERR_BAD_ARG;
    if (!ctx->have_coords) {
        ctx->err = "amg_set_coords not called";
        return AMG_ERR_BAD_ARG;
    }
    if (flags & AMG_DO_VIRIAL) flags |= AMG_DO_GRADIENT;  // as amg_forward
    amg_results res{};
    int rc = amg_forward(ctx, flags, &res);  // captures the graph and sizes the lists
    if (rc != AMG_OK) return rc;
    try {
        CK(cudaSetDevice(ctx->device));
        if (flush_bytes > 0 && (size_t)flush_bytes > ctx->flush_bytes) {
            dalloc(ctx, ctx->flushbuf, (size_t)flush_bytes);
            ctx->flush_bytes = (size_t)flush_bytes;
        }
        cudaEvent_t a, b;
        CK(cudaEventCreate(&a));
        CK(cudaEventCreate(&b));
        long long total = 0;
        for (int k = 0; k < steps; k++) {
            if (flush_bytes > 0) CK(cudaMemsetAsync(ctx->flushbuf, k & 0xff, (size_t)flush_bytes, ctx->st));
            const long long kstart = ctx->kcount;
            CK(cudaEventRecord(a, ctx->st));
            bool graphed = false;
            if (ctx->use_graphs && ctx->bounds && ctx->gexec && !ctx->graph_dirty && ctx->gflags == flags) {
                CK(cudaGraphLaunch(ctx->gexec, ctx->st));
                graphed = true;
            } else if (ctx->prec == AMG_PREC_MIXED) {
                enqueue_eager<float>(ctx, flags);
            } else {
                enqueue_eager<double>(ctx, flags);
            }
            CK(cudaEventRecord(b, ctx->st));
            CK(cudaEventSynchronize(b));
            float ms = 0;
            CK(cudaEventElapsedTime(&ms, a, b));
            ms_steps[k] = ms;
            if (graphed) {
                int iters = 0;
                CK(cudaMemcpy(&iters, ctx->iter, sizeof(int), cudaMemcpyDeviceToHost));
                total += ctx->kmain + (long long)(iterative(ctx) ? iters : 0) * ctx->kbody;
            } else {
                total += ctx->kcount - kstart;
            }
        }
        cudaEventDestroy(a);
        cudaEventDestroy(b);
        if (launches) *launches = total;
        int over = 0;
        CK(cudaMemcpy(&over, ctx->overflow, sizeof(int), cudaMemcpyDeviceToHost));
        if (over > ctx->cap) {
            ctx->err = "neighbour list overflow during the benchmark";
            return AMG_ERR_CUDA;
        }
    } catch (Fail& f) {
        return f.code;
    }
    return AMG_OK;
}

// Times the stored-coefficient T.u kernel (the PCG's real-space matvec) on
// its own: `reps` launches on the context's stream, each after an L2 flush of
// flush_bytes, using the coefficients and dipoles of the last evaluation.
// Reports the average device time and the kernel's algorithmic bytes per
// launch (coefficient rows streamed + the dipoles and fields of each site).
int amg_time_tu_kernel(amg_ctx* ctx, int32_t reps, int64_t flush_bytes, double* ms_avg, double* bytes_per_launch,
                       int64_t* directed_pairs) {
    if (!ctx || reps <= 0 || !ms_avg) return AMG_ERR_BAD_ARG;
    if (!ctx->have_forward || !iterative(ctx)) {
        ctx->err = "needs a previous evaluation with mutual polarization";
        return AMG_ERR_BAD_ARG;
    }
    try {
        CK(cudaSetDevice(ctx->device));
        const int n = ctx->n;
        std::vector<int> nnb(n), off(n + 1);
        CK(cudaMemcpy(nnb.data(), ctx->nnb, sizeof(int) * n, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(off.data(), ctx->xoff, sizeof(int) * (n + 1), cudaMemcpyDeviceToHost));
        long long pairs = 0;
        for (int i = 0; i < n; i++) pairs += nnb[i] + (off[i + 1] - off[i]);
        if (flush_bytes > 0 && (size_t)flush_bytes > ctx->flush_bytes) {
            dalloc(ctx, ctx->flushbuf, (size_t)flush_bytes);
            ctx->flush_bytes = (size_t)flush_bytes;
        }
        cudaEvent_t a, b;
        CK(cudaEventCreate(&a));
        CK(cudaEventCreate(&b));
        double tot = 0;
        const bool mixed = ctx->prec == AMG_PREC_MIXED;
        size_t rs = mixed ? sizeof(float) : sizeof(double);
        for (int k = 0; k < reps; k++) {
            if (flush_bytes > 0) CK(cudaMemsetAsync(ctx->flushbuf, k & 0xff, (size_t)flush_bytes, ctx->st));
            CK(cudaEventRecord(a, ctx->st));
            LPA_DISPATCH(ctx->lpa, {
                if (mixed)
                    k_tu_stored<float, L><<<nblk((size_t)n * L), kThreads, 0, ctx->st>>>(
                        n, ctx->sids, ctx->cnb, ctx->af.c0, ctx->cap, ctx->nnb, ctx->xoff, ctx->af.p4,
                        ctx->Fd, ctx->Fp);
                else
                    k_tu_stored<double, L><<<nblk((size_t)n * L), kThreads, 0, ctx->st>>>(
                        n, ctx->sids, ctx->cnb, ctx->ad.c0, ctx->cap, ctx->nnb, ctx->xoff, ctx->ad.p4,
                        ctx->Fd, ctx->Fp);
            });
            KCHECK();
            CK(cudaEventRecord(b, ctx->st));
            CK(cudaEventSynchronize(b));
            float ms = 0;
            CK(cudaEventElapsedTime(&ms, a, b));
            tot += ms;
        }
        cudaEventDestroy(a);
        cudaEventDestroy(b);
        *ms_avg = tot / reps;
        if (bytes_per_launch)
            *bytes_per_launch = (double)pairs * (4.0 + 4.0 * rs) + (double)n * (2 * 4 * rs + 2 * 3 * 8.0 + 8.0);
        if (directed_pairs) *directed_pairs = pairs;
    } catch (Fail& f) {
        return f.code;
    }
    return AMG_OK;
}

}  // extern "C"

namespace {

// FMA throughput kernel: kFmaChains independent multiply-add chains per
// thread (enough to cover the pipeline latency), kFmaIters rounds each; the
// result is stored only in an impossible case, so nothing is optimized away
constexpr int kFmaChains = 8;
constexpr int kFmaIters = 4096;

template <class T>
__global__ void __launch_bounds__(256) k_fma_peak(T a, T b, int* __restrict__ sink) {
    T x[kFmaChains];
#pragma unroll
    for (int c = 0; c < kFmaChains; c++) x[c] = (T)(threadIdx.x + c);
    for (int it = 0; it < kFmaIters; it++) {
#pragma unroll
        for (int c = 0; c < kFmaChains; c++) x[c] = fma(x[c], a, b);
    }
    T s = 0;
#pragma unroll
    for (int c = 0; c < kFmaChains; c++) s += x[c];
    if (s == (T)-12345.678) sink[0] = 1;
}

}  // namespace

extern "C" {

int amg_fma_peak(int32_t device, int32_t fp64, double* gflops) {
    if (!gflops) return AMG_ERR_BAD_ARG;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
        cudaGetLastError();
        return AMG_ERR_NO_DEVICE;
    }
    if (cudaSetDevice(device) != cudaSuccess) return AMG_ERR_CUDA;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return AMG_ERR_CUDA;
    const int blocks = prop.multiProcessorCount * 8, threads = 256;
    int* sink = nullptr;
    cudaEvent_t a = nullptr, b = nullptr;
    int rc = AMG_OK;
    if (cudaMalloc((void**)&sink, sizeof(int)) != cudaSuccess || cudaEventCreate(&a) != cudaSuccess ||
        cudaEventCreate(&b) != cudaSuccess) {
        rc = AMG_ERR_CUDA;
    } else {
        float best = 1e30f;
        for (int rep = 0; rep < 6; rep++) {  // the first run warms up; the best of the rest counts
            cudaEventRecord(a);
            if (fp64)
                k_fma_peak<double><<<blocks, threads>>>(0.999999, 1e-7, sink);
            else
                k_fma_peak<float><<<blocks, threads>>>(0.9999f, 1e-4f, sink);
            cudaEventRecord(b);
            if (cudaEventSynchronize(b) != cudaSuccess) {
                rc = AMG_ERR_CUDA;
                break;
            }
            float ms = 0;
            cudaEventElapsedTime(&ms, a, b);
            if (rep > 0) best = std::min(best, ms);
        }
        if (rc == AMG_OK) {
            const double flops = 2.0 * kFmaChains * kFmaIters * (double)blocks * threads;
            *gflops = flops / (best * 1e-3) / 1e9;
        }
    }
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
    if (sink) cudaFree(sink);
    cudaGetLastError();
    return rc;
}

int amg_last_stats(amg_ctx* ctx, int64_t* launches, int32_t* graphed, int32_t* lanes_per_site) {
    if (!ctx) return AMG_ERR_BAD_ARG;
    if (launches) *launches = ctx->klast;
    if (graphed) *graphed = ctx->graphed_last;
    if (lanes_per_site) *lanes_per_site = ctx->lpa;
    return AMG_OK;
}

int amg_last_virial(amg_ctx* ctx, double vir_em[9], double vir_ep[9]) {
    if (!ctx) return AMG_ERR_BAD_ARG;
    if (!ctx->have_vir) {
        ctx->err = "the last amg_forward did not compute the virial";
        return AMG_ERR_BAD_ARG;
    }
    for (int k = 0; k < 9; k++) {
        if (vir_em) vir_em[k] = ctx->vir_parts[0][k];
        if (vir_ep) vir_ep[k] = ctx->vir_parts[1][k];
    }
    return AMG_OK;
}

int amg_last_timing(amg_ctx* ctx, double ms[5]) {
    if (!ctx || !ms) return AMG_ERR_BAD_ARG;
    for (int k = 0; k < 5; k++) ms[k] = ctx->timing[k];
    return AMG_OK;
}

int amg_set_predictor(amg_ctx* ctx, int32_t kind) {
    if (!ctx) return AMG_ERR_BAD_ARG;
    if (kind != AMG_PRED_NONE && kind != AMG_PRED_GEAR && kind != AMG_PRED_ASPC) {
        ctx->err = "unknown predictor";
        return AMG_ERR_BAD_ARG;
    }
    static_assert(kPredSteps == AMG_PRED_STEPS, "predictor history length");
    try {
        CK(cudaSetDevice(ctx->device));
        // b_j, j = 1..6: Gear's binomial extrapolation (-1)^(j+1) C(6, j); ASPC
        // (Kolafa 2004) (-1)^(j+1) j C(2k+4, k+2-j) / C(2k+2, k+1), k = 4
        auto binom = [](int a, int b) {
            double r = 1;
            for (int i = 1; i <= b; i++) r = r * (a - b + i) / i;
            return r;
        };
        const int k = kPredSteps - 2;
        for (int j = 1; j <= kPredSteps; j++) {
            const double sgn = (j % 2) ? 1.0 : -1.0;
            ctx->pred_coef.b[j - 1] = kind == AMG_PRED_GEAR ? sgn * binom(kPredSteps, j)
                                                            : sgn * j * binom(2 * k + 4, k + 2 - j) / binom(2 * k + 2, k + 1);
        }
        if (kind != AMG_PRED_NONE && !ctx->pred_hist) {
            dalloc(ctx, ctx->pred_hist, (size_t)kPredSteps * 2 * 3 * ctx->n);
            dalloc(ctx, ctx->pred_state, 2);
        }
        if (ctx->pred_state) CK(cudaMemsetAsync(ctx->pred_state, 0, 2 * sizeof(int), ctx->st));
        ctx->pred = kind;
        ctx->graph_dirty = true;
        CK(cudaStreamSynchronize(ctx->st));
    } catch (Fail& f) {
        return f.code;
    }
    return AMG_OK;
}

const char* amg_last_error(amg_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

void amg_destroy(amg_ctx* ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    release(ctx);
    delete ctx;
}

}  // extern "C"

// ===========================================================================
// Allocation-free entry point.
//
// Some callers cannot let a library allocate device memory: codes that carve
// all device memory out of one arena at start-up and forbid later allocation,
// and codes that must not allocate between steps because cudaMalloc and
// cudaFree synchronize the whole device.  amg_empole_direct_noalloc serves
// them (it has no counterpart in the reference): non-Ewald multipoles, pairs
// within a cutoff, 1-n exclusion scaling, with every buffer supplied by the
// caller and the kernels' scratch (rotated multipoles, site torques,
// per-block energy partials) in one fixed device array declared below.  It
// calls no cudaMalloc/cudaFree and no allocating library routine.
// ===========================================================================

namespace {

constexpr int kNoAllocMaxAtoms = 16384;  // AMG_NOALLOC_MAX_ATOMS
constexpr int kNoAllocLanes = 32;
constexpr int kNoAllocThreads = 128;
constexpr int kNoAllocBlocks = kNoAllocMaxAtoms * kNoAllocLanes / kNoAllocThreads;
// scratch layout (doubles): rotated multipoles [n][10], torques [n][3],
// energy partials [blocks]
constexpr size_t kNoAllocScratch = (size_t)kNoAllocMaxAtoms * 13 + kNoAllocBlocks;

// Every GPU that loads the library holds this array (about 1.7 MB) until exit.
// In host code its name is only a stand-in, not a device address: the kernels
// get the address that cudaGetSymbolAddress returns for the current device.
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocScratch];

// rotate the multipoles (as the main path's frame code) into scratch
__global__ void k_noalloc_rotate(int n, const double* __restrict__ xyz, const double* __restrict__ pole13,
                                 const int* __restrict__ zax, const int* __restrict__ xax,
                                 const int* __restrict__ yax, const int* __restrict__ axe,
                                 double* __restrict__ rp10) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double m[10];
    frame_and_rotate(i, xyz, pole13, zax, xax, yax, axe, m);
    for (int j = 0; j < 10; j++) rp10[10 * i + j] = m[j];
}

// m-scale of pair (i, k) from i's 1-2..1-5 lists (later lists overwrite)
__device__ __forceinline__ double noalloc_mscale(int i, int k, const int* const* off, const int* const* idx,
                                                 const double* ms) {
    double s = 1.0;
    for (int b = 0; b < 4; b++)
        for (int q = off[b][i]; q < off[b][i + 1]; q++)
            if (idx[b][q] == k) s = ms[b];
    return s;
}

struct NoAllocLists {
    const int* off[4];
    const int* idx[4];
    double ms[4];
};

// all pairs within the cutoff (32 lanes per site), bare radial scaled by the
// pair's m-scale; writes site torques, adds site gradients to dem, and one
// energy partial per block
__global__ void __launch_bounds__(kNoAllocThreads) k_noalloc_pairs(int n, const double* __restrict__ xyz,
                                                                   const double* __restrict__ rp10, NoAllocLists L,
                                                                   double L0, double L1, double L2, double cut2,
                                                                   double f, double* __restrict__ trq,
                                                                   double* __restrict__ dem,
                                                                   double* __restrict__ partial) {
    const int g = (blockIdx.x * blockDim.x + threadIdx.x) / kNoAllocLanes, lane = threadIdx.x % kNoAllocLanes;
    const int i = min(g, n - 1);
    const bool live = g < n;
    Mpole<double> Mi = mpole64(rp10 + 10 * i);
    double e = 0;
    V3<double> gsum = v3<double>(0, 0, 0), tsum = v3<double>(0, 0, 0);
    for (int k = lane; live && k < n; k += kNoAllocLanes) {
        if (k == i) continue;
        V3<double> r = v3<double>(xyz[3 * k] - xyz[3 * i], xyz[3 * k + 1] - xyz[3 * i + 1],
                                  xyz[3 * k + 2] - xyz[3 * i + 2]);
        if (L0 > 0) r.x -= L0 * rint(r.x / L0);
        if (L1 > 0) r.y -= L1 * rint(r.y / L1);
        if (L2 > 0) r.z -= L2 * rint(r.z / L2);
        double r2 = dot(r, r);
        if (r2 > cut2) continue;
        double s = noalloc_mscale(i, k, L.off, L.idx, L.ms);
        double B[6];
        double rinv = 1.0 / sqrt(r2);
        bare_terms<double, 6>(rinv, rinv * rinv, B);
        for (int q = 0; q < 6; q++) B[q] *= s;
        double E;
        V3<double> gi, ti;
        mm_pair_i<double>(Mi, mpole64(rp10 + 10 * k), r, B, E, gi, ti);
        e += 0.5 * E;
        gsum = gsum + gi;
        tsum = tsum + ti;
    }
    double v[7] = {e, gsum.x, gsum.y, gsum.z, tsum.x, tsum.y, tsum.z};
    for (int q = 0; q < 7; q++) v[q] = warp_sum(v[q]);
    if (lane == 0 && live) {
        dem[3 * i] += f * v[1]; dem[3 * i + 1] += f * v[2]; dem[3 * i + 2] += f * v[3];
        trq[3 * i] = f * v[4]; trq[3 * i + 1] = f * v[5]; trq[3 * i + 2] = f * v[6];
    }
    __shared__ double blk[kNoAllocThreads / kNoAllocLanes];
    if (lane == 0) blk[threadIdx.x / kNoAllocLanes] = live ? f * v[0] : 0.0;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0;
        for (int w = 0; w < kNoAllocThreads / kNoAllocLanes; w++) s += blk[w];
        partial[blockIdx.x] = s;
    }
}

// fixed-order sum of the block partials into *em
__global__ void k_noalloc_energy(int nb, const double* __restrict__ partial, double* __restrict__ em) {
    __shared__ double s[256];
    double v = 0;
    for (int b = threadIdx.x; b < nb; b += blockDim.x) v += partial[b];
    s[threadIdx.x] = v;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) s[threadIdx.x] += s[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) *em = s[0];
}

}  // namespace

extern "C" int amg_empole_direct_noalloc(int32_t n, const double* xyz, const double* pole, const int32_t* zaxis,
                                         const int32_t* xaxis, const int32_t* yaxis, const int32_t* polaxe,
                                         const amg_list* bonded, const double m_scale[4], const double box[3],
                                         double cutoff, double f, double* em, double* dem, void* stream) {
    if (n <= 0 || !xyz || !pole || !zaxis || !xaxis || !yaxis || !polaxe || !bonded || !m_scale || !em || !dem ||
        cutoff <= 0)
        return AMG_ERR_BAD_ARG;
    if (n > kNoAllocMaxAtoms) return AMG_ERR_OUT_OF_RANGE;  // scratch holds AMG_NOALLOC_MAX_ATOMS sites
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return AMG_ERR_NO_DEVICE;
    }
    // The scratch array's device address on the current device, looked up on
    // every call rather than cached: after a cudaDeviceReset, or under another
    // context on the same device, the module is loaded again and the array
    // can move.  The first call on a device also loads the library's device
    // code there (lazy module loading), which is why that first call belongs
    // before any stream capture.
    double* scratch = nullptr;
    {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) {
            cudaGetLastError();
            return AMG_ERR_CUDA;
        }
        scratch = (double*)p;
    }
    if (box)
        for (int a = 0; a < 3; a++)
            if (box[a] > 0 && cutoff > 0.5 * box[a]) return AMG_ERR_BAD_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    double* rp10 = scratch;
    double* trq = scratch + 10 * (size_t)kNoAllocMaxAtoms;
    double* partial = scratch + 13 * (size_t)kNoAllocMaxAtoms;
    NoAllocLists L;
    for (int b = 0; b < 4; b++) {
        if (!bonded[b].offsets || !bonded[b].indices) return AMG_ERR_BAD_ARG;
        L.off[b] = bonded[b].offsets;
        L.idx[b] = bonded[b].indices;
        L.ms[b] = m_scale[b];
    }
    const unsigned nb = (unsigned)(((size_t)n * kNoAllocLanes + kNoAllocThreads - 1) / kNoAllocThreads);
    k_noalloc_rotate<<<(n + 127) / 128, 128, 0, st>>>(n, xyz, pole, zaxis, xaxis, yaxis, polaxe, rp10);
    k_noalloc_pairs<<<nb, kNoAllocThreads, 0, st>>>(n, xyz, rp10, L, box ? box[0] : 0.0, box ? box[1] : 0.0,
                                                    box ? box[2] : 0.0, cutoff * cutoff, f, trq, dem, partial);
    k_noalloc_energy<<<1, 256, 0, st>>>((int)nb, partial, em);
    k_torque<<<(n + 127) / 128, 128, 0, st>>>(n, xyz, zaxis, xaxis, yaxis, polaxe, trq, dem, nullptr);
    if (cudaGetLastError() != cudaSuccess) return AMG_ERR_CUDA;
    if (cudaStreamSynchronize(st) != cudaSuccess) return AMG_ERR_CUDA;
    return AMG_OK;
}
