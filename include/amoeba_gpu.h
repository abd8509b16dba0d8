/*
 * amoeba_gpu.h -- C ABI of libamoeba_gpu.so, the sm_100a (B200) AMOEBA
 * electrostatics library: permanent multipoles (empole), the mutual
 * induced-dipole solve (induce) and polarization energy/forces (epolar),
 * each as real-space Ewald pairs (with Thole damping for polarization) plus
 * a smooth-PME reciprocal part.
 *
 * The entry points replace, for a caller of the reference (momokchung/polmdqc):
 *   - polmdqc::empole<CalcMode>()   src/md/empole.cpp:49-83 (dispatcher) and
 *     empole_a src/md/empole.cpp:96-357 (the only implemented variant; the
 *     Ewald variants empole_c/d are stubs at src/md/empole.cpp:53-64,359-368)
 *   - polmdqc::epolar<CalcMode>()   whose call is commented out at
 *     src/md/energy.cpp:267 (no induce/epolar code exists in the reference)
 *   - the electrostatic part of polmdqc::energy<CalcMode>()
 *     src/md/energy.cpp:31-338
 * Inputs are exactly the module globals those routines read after mechanic()
 * (atoms.h, mpole.h, polar.h, polgrp.h, couple.h, polpot.h, mplpot.h,
 * ewald.h, pme.h, boxes.h, chgpot.h); outputs are the globals they write
 * (energi.h em/ep, deriv.h dem/dep, analyz.h aem/aep, action.h nem/nep,
 * inter.h einter, virial.h vir, polar.h uind/uinp).
 *
 * Conventions (all follow the reference):
 *   - coordinates in Angstrom; energies in kcal/mol; gradients are dE/dx in
 *     kcal/mol/Angstrom (deriv.h "dem"), ADDED to the caller's arrays;
 *   - multipoles: 13 components per atom [c, dx,dy,dz, qxx,qxy,qxz, qyx,qyy,
 *     qyz, qzx,qzy,qzz] in the local frame, dipoles in e*Angstrom and
 *     quadrupoles already divided by 3 (kmpole.cpp:547-550);
 *   - frame atoms zaxis/xaxis/yaxis are 1-based, 0 = none; yaxis < 0 marks a
 *     chiral site (mpole.h); polaxe uses the LocalFrame enum (kmulti.h:23-31);
 *   - 1-n neighbour and polarization-group lists are 0-based (couple.h,
 *     polgrp.h) and passed as CSR (offsets[n+1], indices);
 *   - induced dipoles in e*Angstrom (polar.h uind/uinp); convergence eps in
 *     Debye RMS per polarizable site (polpot.h poleps).
 *
 * Every function returns an int status (AMG_OK = 0) and never exits the
 * process; amg_last_error() gives a message for the last failing call.
 * One host thread per context; calls are synchronous (stream-ordered and
 * synchronized before returning).
 */
#ifndef AMOEBA_GPU_H
#define AMOEBA_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define AMG_ABI_VERSION 4

/* status codes */
#define AMG_OK               0
#define AMG_ERR_BAD_ARG      1
#define AMG_ERR_UNSUPPORTED  2  /* cell shape / feature not implemented */
#define AMG_ERR_NO_CONVERGE  3  /* PCG reached politer without meeting poleps */
#define AMG_ERR_NAN          4  /* non-finite energy or gradient */
#define AMG_ERR_CUDA         5  /* a CUDA runtime / cuFFT call failed */
#define AMG_ERR_NO_DEVICE    6  /* no usable sm_100 device */
#define AMG_ERR_OUT_OF_RANGE 7  /* size limit of the entry point exceeded */

/* local frame types, same numbering as the reference's LocalFrame enum */
#define AMG_FRAME_NONE       0
#define AMG_FRAME_ZTHENX     1
#define AMG_FRAME_ZONLY      2
#define AMG_FRAME_BISECTOR   3
#define AMG_FRAME_ZBISECT    4
#define AMG_FRAME_THREEFOLD  5

/* arithmetic of a context */
#define AMG_PREC_FP64   0  /* every kernel in double precision */
#define AMG_PREC_MIXED  1  /* FP32 pair/grid work; FP64 PCG dots, norms,
                              accumulators and one FP64 correction sweep */

/* periodic cell shapes (boxes.h): the lattice follows from the box angles
 * (orthogonal, monoclinic with only beta != 90, else triclinic) unless the
 * cell is a truncated octahedron or a rhombic dodecahedron (boxes.h
 * octahedron / dodecadron, whose box angles are all 90) */
#define AMG_CELL_FROM_ANGLES   0
#define AMG_CELL_OCTAHEDRON    1
#define AMG_CELL_DODECAHEDRON  2

/* polarization models (polpot.h poltyp) */
#define AMG_POL_NONE    0
#define AMG_POL_MUTUAL  1
#define AMG_POL_DIRECT  2
#define AMG_POL_OPT     3  /* extrapolated perturbation theory, coefficients opt_coef */
#define AMG_MAX_OPT     6  /* highest OPT order (polopt.h maxopt) */

/* charge penetration of the multipoles (mplpot.h pentype; AMOEBA+ and
 * HIPPO, include/md/damping.h): none, Gordon f1, Gordon f2 */
#define AMG_PEN_NONE     0
#define AMG_PEN_GORDON1  1
#define AMG_PEN_GORDON2  2

/* CalcMode flags for amg_forward (reference calcMode.h:18-45) */
#define AMG_DO_ENERGY    1
#define AMG_DO_ANALYSIS  2  /* per-atom energies, pair counts, einter */
#define AMG_DO_GRADIENT  4
#define AMG_DO_VIRIAL    8
#define AMG_DO_DIPOLES  16  /* copy uind/uinp back */

typedef struct amg_list {
    const int32_t* offsets;   /* [n+1] */
    const int32_t* indices;   /* [offsets[n]] 0-based atom numbers */
} amg_list;

typedef struct amg_params {
    int32_t n;                       /* atoms (atoms.h n) */
    const double* pole;              /* [n*13] local-frame multipoles (mpole.h pole) */
    const int32_t* zaxis;            /* [n] 1-based, 0 = none */
    const int32_t* xaxis;
    const int32_t* yaxis;
    const int32_t* polaxe;           /* [n] AMG_FRAME_* */
    const int32_t* molcule;          /* [n] molecule id (molcul.h), for einter; may be NULL */
    const double* polarity;          /* [n] Angstrom^3 (polar.h); NULL if no polarization */
    const double* thole;             /* [n] */
    const double* pdamp;             /* [n] polarity^(1/6) */
    amg_list i12, i13, i14, i15;     /* couple.h */
    amg_list ip11, ip12, ip13, ip14; /* polgrp.h (ip11 includes the atom itself) */
    double m_scale[4];               /* m2..m5   (mplpot.h) */
    double p_scale[4];               /* p2..p5   (polpot.h) */
    double p_iscale[4];              /* p2i..p5i */
    double d_scale[4];               /* d1..d4 */
    double u_scale[4];               /* u1..u4 */
    int32_t use_ewald;               /* limits.h use_ewald */
    int32_t use_bounds;              /* bound.h use_bounds (periodic box) */
    double aewald;                   /* ewald.h aeewald (1/Angstrom) */
    int32_t nfft[3];                 /* pme.h nefft1..3 */
    int32_t bsorder;                 /* pme.h bseorder (B-spline order) */
    double cutoff;                   /* real-space cutoff: ewaldcut with Ewald, mpolecut without */
    int32_t poltyp;                  /* AMG_POL_* */
    double poleps;                   /* polpot.h poleps (Debye RMS) */
    int32_t politer;                 /* polpot.h politer */
    double electric;                 /* chgpot.h electric (kcal/mol*Angstrom/e^2) */
    double dielec;                   /* chgpot.h dielec */
    double debye;                    /* units.h debye (e*Angstrom -> Debye) */
    int32_t precision;               /* AMG_PREC_* */
    int32_t pcg_guess;               /* polpcg.h pcgguess: start from direct dipoles */
    int32_t device;                  /* CUDA device ordinal */
    /* Appended in ABI version 2 (zero keeps the version-1 behaviour): */
    int32_t pcg_prec;                /* polpcg.h pcgprec: 1 = sparse preconditioner
                                        M = 2 alpha + alpha T_u alpha over pairs within
                                        usolvcut (Thole-damped, u-scaled, no Ewald);
                                        0 = diagonal (alpha) */
    double usolvcut;                 /* limits.h usolvcut (Angstrom), at most cutoff */
    /* Appended in ABI version 3 (zero keeps the version-2 behaviour): */
    int32_t cell_shape;              /* AMG_CELL_*: every cell works without
                                        Ewald; with Ewald the prism cells, the
                                        octahedron and the dodecahedron with c = a
                                        (else UNSUPPORTED); their PME grid (nfft)
                                        spans the enclosing prism: a^3, or
                                        a x a x sqrt(2) a */
    double opt_coef[AMG_MAX_OPT + 1]; /* polopt.h copt: with AMG_POL_OPT the dipoles
                                        are sum_k (sum_{j>=k} copt_j) u^(k), u^(0) =
                                        alpha E, u^(k) = alpha T u^(k-1); the order is
                                        the last nonzero entry (src/md/kpolar.cpp:
                                        108-153, 228-236) */
    /* Appended in ABI version 4 (zero keeps the version-3 behaviour): charge
     * penetration and charge flux of the multipoles (AMOEBA+, HIPPO), in the
     * reference's non-Ewald multipole mode only (src/md/empole.cpp:64-82):
     * with Ewald or polarization they return UNSUPPORTED. */
    int32_t pentype;                 /* AMG_PEN_*: core/valence split of each monopole,
                                        valence damped (include/md/pairMpole.h:186-389) */
    const double* pcore;             /* [n] core charge (chgpen.h pcore); valence = q - core */
    const double* palpha;            /* [n] damping exponent (chgpen.h palpha) */
    int32_t cflux;                   /* potent.h use_chgflx: the monopoles follow the
                                        geometry, q = pole[i][0] + dq (src/md/alterchg.cpp);
                                        pole[i][0] is then the unaltered monopole (mpole.h mono0) */
    int32_t nbond;                   /* bonds of the charge flux (bndstr.h nbond) */
    const int32_t* bond_atoms;       /* [nbond*2] 0-based atoms (bndstr.h ibnd) */
    const double* bond_flux;         /* [nbond*2] ideal length bl, flux bflx (cflux.h) */
    int32_t nangle;                  /* angles of the charge flux (angbnd.h nangle) */
    const int32_t* angle_atoms;      /* [nangle*3] 0-based a, b (vertex), c (angbnd.h iang) */
    const double* angle_flux;        /* [nangle*7] ideal angle anat (degrees), ideal
                                        lengths of bonds a-b and c-b (bl via atmlst.h
                                        balist), aflx[2], abflx[2] (cflux.h) */
} amg_params;

typedef struct amg_results {
    double em;          /* permanent multipole energy */
    double ep;          /* polarization energy */
    double einter;      /* intermolecular part of em+ep (AMG_DO_ANALYSIS) */
    int64_t nem;        /* multipole pairs with nonzero energy (AMG_DO_ANALYSIS) */
    int64_t nep;        /* polarization sites with nonzero energy (AMG_DO_ANALYSIS) */
    double vir[9];      /* added to with AMG_DO_VIRIAL: dE/d(strain), symmetric (virial.h vir) */
    double* dem;        /* [n*3] gradient of em, ADDED to; may be NULL */
    double* dep;        /* [n*3] gradient of ep, ADDED to; may be NULL */
    double* aem;        /* [n] per-atom em (AMG_DO_ANALYSIS), overwritten; may be NULL */
    double* aep;        /* [n] per-atom ep (AMG_DO_ANALYSIS), overwritten; may be NULL */
    double* uind;       /* [n*3] mutual induced dipoles (AMG_DO_DIPOLES); may be NULL */
    double* uinp;       /* [n*3] dipoles in the polarization-energy field; may be NULL */
    double* rpole;      /* [n*13] global-frame multipoles; may be NULL */
    int32_t pcg_iters;  /* PCG iterations taken */
    double pcg_eps;     /* final RMS residual (Debye) */
} amg_results;

/* Cotangents (upstream adjoints) for amg_backward.  The scalar seed dE on the
 * total energy em+ep is the usual case; the dipole cotangents make the
 * backward solve one extra PCG with the same symmetric operator. */
typedef struct amg_cotangents {
    double d_energy;          /* dL/d(em+ep) */
    const double* d_uind;     /* [n*3] dL/duind, or NULL */
    const double* d_uinp;     /* [n*3] dL/duinp, or NULL */
} amg_cotangents;

/* Gradients of L with respect to the parameters (overwritten); any pointer
 * may be NULL.  The quadrupole entries of d_pole are the gradient restricted
 * to traceless quadrupoles (AMOEBA quadrupoles are traceless). */
typedef struct amg_param_grads {
    double* d_pole;       /* [n*13] dL/d(local-frame pole) */
    double* d_polarity;   /* [n] dL/dpolarity (includes the pdamp = alpha^(1/6) path) */
    double* d_thole;      /* [n] dL/dthole (through pair thole = min(thole_i, thole_k)) */
    double* d_xyz;        /* [n*3] dL/dx */
} amg_param_grads;

typedef struct amg_ctx amg_ctx;

/* Creates a context on params->device: uploads parameters, topology-derived
 * scaled-pair tables and PME plans.  Arrays in params are copied. */
int amg_create(const amg_params* params, amg_ctx** out);

/* Sets coordinates [n*3] (Angstrom) and the box: a,b,c (Angstrom) and
 * alpha,beta,gamma (degrees) as boxes.h xbox,ybox,zbox,alphaA,betaA,gammaA.
 * With use_bounds, the minimum image of the cell shape (params cell_shape and
 * the angles) is the reference's image() (src/md/image.cpp:37-124).  With Ewald
 * in a truncated octahedron or rhombic dodecahedron the cell volume is half the
 * enclosing prism's (a^3 / 2 and a^3 / sqrt(2)); the dodecahedron needs c = a,
 * for which its image is a lattice (UNSUPPORTED otherwise).  A non-finite
 * coordinate returns AMG_ERR_NAN and leaves the context without coordinates
 * until the next successful call. */
int amg_set_coords(amg_ctx* ctx, const double* xyz, const double box[6]);

/* Evaluates em and ep (and their gradients, analysis data, dipoles) for the
 * current coordinates.  flags: AMG_DO_* bits. */
int amg_forward(amg_ctx* ctx, int32_t flags, amg_results* res);

/* Adjoint of the last amg_forward: gradients of L = d_energy*(em+ep)
 * + <d_uind,uind> + <d_uinp,uinp> with respect to the parameters and
 * coordinates, recomputing pair intermediates instead of storing them. */
int amg_backward(amg_ctx* ctx, const amg_cotangents* cot, amg_param_grads* grads);

/* Timing of the last amg_forward on the device (ms) by phase: 0 total,
 * 1 setup (rotation, sort, lists), 2 permanent field, 3 PCG, 4 forces
 * (zeros when the evaluation ran as one captured graph). */
int amg_last_timing(amg_ctx* ctx, double ms[5]);

/* Benchmark support (no counterpart in the reference): runs `steps`
 * evaluations with the coordinates already on the device and the results
 * left there, writing `flush_bytes` to a scratch buffer before each one
 * (L2 eviction, not timed), and returns each evaluation's device time in
 * ms_steps[steps] (CUDA events on the context's stream) and the number of
 * this library's kernel launches in *launches.  Runs one untimed
 * evaluation first. */
int amg_bench(amg_ctx* ctx, int32_t flags, int32_t steps, int64_t flush_bytes, double* ms_steps,
              int64_t* launches);

/* Benchmark support (no counterpart in the reference): average device time
 * of the PCG's real-space T.u kernel run on its own (`reps` launches, each
 * after writing flush_bytes to evict L2), with its algorithmic bytes per
 * launch and the number of directed pairs it processes.  Needs a previous
 * amg_forward with mutual polarization. */
int amg_time_tu_kernel(amg_ctx* ctx, int32_t reps, int64_t flush_bytes, double* ms_avg, double* bytes_per_launch,
                       int64_t* directed_pairs);

/* Benchmark support (no counterpart in the reference): the measured FMA
 * throughput of `device` in GFLOP/s (2 flops per fused multiply-add), FP32
 * (fp64 = 0) or FP64 (fp64 = 1), from a kernel of independent FMA chains on
 * every SM -- the roofline denominator of the compute-bound pair kernels. */
int amg_fma_peak(int32_t device, int32_t fp64, double* gflops);

/* The two parts of the last amg_forward's virial (AMG_DO_VIRIAL), as added
 * to amg_results.vir: the em terms and the ep terms (the reference keeps one
 * vir array and adds each term's share from its own routine, empole / epolar,
 * virial.h).  Either pointer may be NULL. */
int amg_last_virial(amg_ctx* ctx, double vir_em[9], double vir_ep[9]);

/* Induced-dipole predictor, the reference's uprior module (include/md/uprior.h:
 * use_pred, polpred, udalt/upalt; the reference declares it and leaves it off,
 * src/md/initprm.cpp:396).  With a predictor set, every mutual-polarization
 * amg_forward keeps its converged dipoles (both sets) in a history of the
 * last AMG_PRED_STEPS evaluations on the device; once the history is full,
 * the PCG starts from the extrapolation sum_j b_j u(n-j), j = 1..6, instead
 * of the direct dipoles:
 *   AMG_PRED_GEAR: b_j = (-1)^(j+1) C(6, j), the binomial (polynomial) predictor;
 *   AMG_PRED_ASPC: b_j = (-1)^(j+1) j C(2k+4, k+2-j) / C(2k+2, k+1), k = 4, the
 *   always stable predictor-corrector coefficients (Kolafa, J. Comput. Chem.
 *   25, 335 (2004)).
 * The converged dipoles do not depend on the start beyond poleps; the
 * predictor saves PCG iterations when consecutive calls are consecutive
 * steps of one trajectory.  Setting a predictor (or AMG_PRED_NONE) clears
 * the history. */
#define AMG_PRED_NONE 0
#define AMG_PRED_GEAR 1
#define AMG_PRED_ASPC 2
#define AMG_PRED_STEPS 6
int amg_set_predictor(amg_ctx* ctx, int32_t kind);

/* Kernel launches of the last amg_forward, whether it ran as one captured
 * CUDA graph, and the lanes per site of the pair kernels. */
int amg_last_stats(amg_ctx* ctx, int64_t* launches, int32_t* graphed, int32_t* lanes_per_site);

/* Allocation-free entry point.  It has no counterpart in the reference: it is
 * an addition of this library for callers that cannot let a library allocate
 * device memory -- codes that take all device memory from one arena at
 * start-up and forbid later allocation, and codes that must not call
 * cudaMalloc/cudaFree between steps because those calls synchronize the
 * whole device.  It computes the non-Ewald multipole energy and gradient over
 * all pairs within `cutoff`, minimum image in an orthogonal box (box NULL, or
 * box[a] <= 0: no wrapping on that axis), 1-2..1-5 scaling by m_scale.
 *
 * It calls no cudaMalloc, cudaFree or allocating library routine.  Every
 * pointer argument except m_scale and box is device memory supplied by the
 * caller: xyz [3n], pole [13n], the frame arrays [n], bonded[4] = the
 * 1-2..1-5 lists as device CSR.  *em [1] is overwritten with the energy;
 * dem [3n] is ADDED to.  The kernels' scratch is one fixed device array of
 * about 1.7 MB that every GPU loading the library holds until exit.
 * n above AMG_NOALLOC_MAX_ATOMS returns AMG_ERR_OUT_OF_RANGE.  The first call
 * on a device loads the library's device code there and looks up the
 * array's device address; make that first call before any stream capture.
 * All calls share the array, which keeps the last call's contents: calls
 * that overlap on the GPU (different streams or threads) race and must be
 * serialized by the caller.  Runs on `stream` (NULL: the legacy default
 * stream) and returns after it completes.  f = electric / dielec. */
#define AMG_NOALLOC_MAX_ATOMS 16384
int amg_empole_direct_noalloc(int32_t n, const double* xyz, const double* pole, const int32_t* zaxis,
                              const int32_t* xaxis, const int32_t* yaxis, const int32_t* polaxe,
                              const amg_list* bonded, const double m_scale[4], const double box[3],
                              double cutoff, double f, double* em, double* dem, void* stream);

const char* amg_last_error(amg_ctx* ctx);
int amg_abi_version(void);
void amg_destroy(amg_ctx* ctx);

#ifdef __cplusplus
}
#endif
#endif /* AMOEBA_GPU_H */
