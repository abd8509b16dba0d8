// kernels_setup.cuh -- per-evaluation set-up: frames (rotpole/chkpole),
// cell binning, exact neighbour lists, B-spline stencils.
#pragma once
#include "kernels.cuh"

namespace amg {

// Local-to-global rotation matrix of site i (rows: local x, y, z axes in
// global coordinates), following the frame definitions of the reference's
// rotmat (src/md/rotpole.cpp:102-345), with the chirality test of chkpole
// (src/md/chkpole.cpp:44-89) reported as `flip` (the y-components of the
// local multipole change sign) instead of mutating the inputs, and the
// Z-Bisect planarity case reported as `planar`.
__device__ inline void frame_matrix(int i, const double* __restrict__ xyz, const int* __restrict__ zax,
                                    const int* __restrict__ xax, const int* __restrict__ yax,
                                    const int* __restrict__ axe, double (&a)[3][3], bool& flip, bool& planar) {
    using D = double;
    auto P = [&](int q) { return v3<D>(xyz[3 * q], xyz[3 * q + 1], xyz[3 * q + 2]); };
    auto unit = [](V3<D> v) { D s = 1.0 / sqrt(dot(v, v)); return s * v; };
    const int ft = axe[i];
    const V3<D> xi = P(i);
    V3<D> zv = v3<D>(0, 0, 1), xv = v3<D>(1, 0, 0);
    flip = false;
    planar = false;
    if (ft == AMG_FRAME_ZTHENX && yax[i] != 0) {
        int k = yax[i];
        V3<D> pa = xi, pb = P(zax[i] - 1), pc = P(xax[i] - 1), pd = P(abs(k) - 1);
        D vol = dot(pa - pd, cross(pb - pd, pc - pd));
        flip = (k < 0 && vol > 0) || (k > 0 && vol < 0);
    }
    if (ft == AMG_FRAME_ZONLY) {
        zv = unit(P(zax[i] - 1) - xi);
        V3<D> t = fabs(zv.x) > 0.707 ? v3<D>(0, 1, 0) : v3<D>(1, 0, 0);
        xv = unit(t - dot(t, zv) * zv);
    } else if (ft == AMG_FRAME_ZTHENX) {
        zv = unit(P(zax[i] - 1) - xi);
        V3<D> t = P(xax[i] - 1) - xi;
        xv = unit(t - dot(t, zv) * zv);
    } else if (ft == AMG_FRAME_BISECTOR) {
        V3<D> u1 = unit(P(zax[i] - 1) - xi), u2 = unit(P(xax[i] - 1) - xi);
        zv = unit(u1 + u2);
        xv = unit(u2 - dot(u2, zv) * zv);
    } else if (ft == AMG_FRAME_ZBISECT) {
        zv = unit(P(zax[i] - 1) - xi);
        V3<D> u1 = unit(P(xax[i] - 1) - xi), u2 = unit(P(abs(yax[i]) - 1) - xi);
        V3<D> b = unit(u1 + u2);
        D angle = 180.0 - (180.0 / kPi) * acos(dot(b, zv));
        if (angle < 0.0) {
            planar = true;
            b = cross(u1, u2);
            if (dot(b, zv) < 0) b = (-1.0) * b;
        }
        xv = unit(b - dot(b, zv) * zv);
    } else if (ft == AMG_FRAME_THREEFOLD) {
        V3<D> u1 = unit(P(zax[i] - 1) - xi), u2 = unit(P(xax[i] - 1) - xi), u3 = unit(P(abs(yax[i]) - 1) - xi);
        zv = unit(u1 + u2 + u3);
        xv = unit(u1 - dot(u1, zv) * zv);
    }
    V3<D> yv = cross(zv, xv);
    a[0][0] = xv.x; a[0][1] = xv.y; a[0][2] = xv.z;
    a[1][0] = yv.x; a[1][1] = yv.y; a[1][2] = yv.z;
    a[2][0] = zv.x; a[2][1] = zv.y; a[2][2] = zv.z;
}

// The rotated (global-frame) multipole of site i, compact [q, d, Qxx, Qxy,
// Qxz, Qyy, Qyz, Qzz], as the reference's rotsite (src/md/rotpole.cpp:356-425):
// d_g = A^T d_l, Q_g = A^T Q_l A.
__device__ inline void frame_and_rotate(int i, const double* __restrict__ xyz, const double* __restrict__ pole13,
                                        const int* __restrict__ zax, const int* __restrict__ xax,
                                        const int* __restrict__ yax, const int* __restrict__ axe, double out[10]) {
    double a[3][3];
    bool flip, planar;
    frame_matrix(i, xyz, zax, xax, yax, axe, a, flip, planar);
    double sp[13];
    for (int j = 0; j < 13; j++) sp[j] = pole13[13 * i + j];
    if (flip) {
        sp[2] = -sp[2]; sp[5] = -sp[5]; sp[7] = -sp[7]; sp[9] = -sp[9]; sp[11] = -sp[11];
    }
    if (planar) {
        sp[1] = 0; sp[6] = 0; sp[10] = 0;
        sp[4] = sp[8] = 0.5 * (sp[4] + sp[8]);
    }
    out[0] = sp[0];
    for (int c = 0; c < 3; c++) out[1 + c] = sp[1] * a[0][c] + sp[2] * a[1][c] + sp[3] * a[2][c];
    double qg[3][3];
    for (int p = 0; p < 3; p++)
        for (int q = p; q < 3; q++) {
            double v = 0;
            for (int r = 0; r < 3; r++)
                for (int t = 0; t < 3; t++) v += a[r][p] * a[t][q] * sp[4 + 3 * r + t];
            qg[p][q] = v;
        }
    out[4] = qg[0][0]; out[5] = qg[0][1]; out[6] = qg[0][2];
    out[7] = qg[1][1]; out[8] = qg[1][2]; out[9] = qg[2][2];
}

template <class R>
__global__ void k_rotate(int n, const double* __restrict__ xyz, const double* __restrict__ pole13,
                         const int* __restrict__ zax, const int* __restrict__ xax, const int* __restrict__ yax,
                         const int* __restrict__ axe, const double* __restrict__ pdamp,
                         const double* __restrict__ thole, const double* __restrict__ pol,
                         const double* __restrict__ dq, double* __restrict__ rp10, AtomR<R>* __restrict__ atoms) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double m[10];
    frame_and_rotate(i, xyz, pole13, zax, xax, yax, axe, m);
    if (dq) m[0] += dq[i];  // charge flux: the monopole of the current geometry
    for (int j = 0; j < 10; j++) rp10[10 * i + j] = m[j];
    AtomR<R> A;
    A.a = make_r4<R>((R)xyz[3 * i], (R)xyz[3 * i + 1], (R)xyz[3 * i + 2], (R)m[0]);
    A.b = make_r4<R>((R)m[1], (R)m[2], (R)m[3], (R)m[4]);
    A.c = make_r4<R>((R)m[5], (R)m[6], (R)m[7], (R)m[8]);
    A.e = make_r4<R>((R)m[9], pdamp ? (R)pdamp[i] : R(0), thole ? (R)thole[i] : R(0), pol ? (R)pol[i] : R(0));
    atoms[i] = A;
}

// ---------------------------------------------------------------- cells
struct CellGrid {
    int nc[3];          // cells per axis
    double origin[3];   // lower corner (non-periodic) or 0
    double size[3];     // cell edge
    int periodic;
    int off_lo[3], off_hi[3];  // distinct stencil offsets per axis
    // monoclinic / triclinic cell: cells are the lattice's parallelepipeds,
    // indexed by fractional coordinates s_a = sum_j x_j R[j][a]; A rows are the
    // lattice vectors (x = sum_a s_a A[a])
    int general;
    double R[3][3], A[3][3];
    // truncated octahedron / rhombic dodecahedron: cells of the enclosing
    // prism (edges size * nc, an even count per axis), whose lattice plus the
    // centring translation (half of every edge) is the cell's lattice
    int centred;
};

// fractional coordinates of x in [0, 1) along each lattice vector
__device__ __forceinline__ void frac_wrapped(const CellGrid& cg, double x, double y, double z, double (&f)[3]) {
#pragma unroll
    for (int a = 0; a < 3; a++) {
        f[a] = x * cg.R[0][a] + y * cg.R[1][a] + z * cg.R[2][a];
        f[a] -= floor(f[a]);
    }
}

__global__ void k_cell_index(int n, const double* __restrict__ xyz, CellGrid cg, Box bx, unsigned* __restrict__ keys,
                             int* __restrict__ ids) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int c[3];
    if (cg.general) {
        double f[3];
        frac_wrapped(cg, xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2], f);
        for (int a = 0; a < 3; a++) c[a] = min(cg.nc[a] - 1, (int)(f[a] * cg.nc[a]));
        keys[i] = (unsigned)((c[0] * cg.nc[1] + c[1]) * cg.nc[2] + c[2]);
        ids[i] = i;
        return;
    }
    for (int a = 0; a < 3; a++) {
        double x = xyz[3 * i + a];
        double f;
        if (cg.centred) {  // wrapped into the enclosing prism
            f = x / (cg.size[a] * cg.nc[a]);
            f -= floor(f);
            c[a] = min(cg.nc[a] - 1, (int)(f * cg.nc[a]));
        } else if (cg.periodic) {
            f = x * bx.iL[a];
            f -= floor(f);
            c[a] = min(cg.nc[a] - 1, (int)(f * cg.nc[a]));
        } else {
            c[a] = min(cg.nc[a] - 1, max(0, (int)((x - cg.origin[a]) / cg.size[a])));
        }
    }
    keys[i] = (unsigned)((c[0] * cg.nc[1] + c[1]) * cg.nc[2] + c[2]);
    ids[i] = i;
}

// cell start/end of the sorted keys, the coordinates in cell order and each
// site's position in that order (rank, the inverse of sids); with sdt, the
// sites' (pdamp, thole) in cell order as well
__global__ void k_cell_bounds(int n, const unsigned* __restrict__ skeys, const int* __restrict__ sids,
                              const double* __restrict__ xyz, int* __restrict__ start, int* __restrict__ end,
                              double4* __restrict__ spos, int* __restrict__ rank,
                              const double* __restrict__ pdamp, const double* __restrict__ thole,
                              double2* __restrict__ sdt) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    unsigned k = skeys[i];
    if (i == 0 || skeys[i - 1] != k) start[k] = i;
    if (i == n - 1 || skeys[i + 1] != k) end[k] = i + 1;
    int a = sids[i];
    spos[i] = make_double4(xyz[3 * a], xyz[3 * a + 1], xyz[3 * a + 2], 0.0);
    rank[a] = i;
    if (sdt) sdt[i] = make_double2(pdamp[a], thole[a]);  // damping parameters in cell order
}

// The packed sites in cell order (atS[g] = at[sids[g]]), which the bulk pair
// kernels gather with the cell-order partner indices of the lists: a warp's
// sites share most of their partners, which then sit in a few contiguous runs.
template <class R>
__global__ void k_gather_atoms(int n, const int* __restrict__ sids, const AtomR<R>* __restrict__ at,
                               AtomR<R>* __restrict__ atS) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g < n) atS[g] = at[sids[g]];
}

// Exact neighbour list: all j != i with minimum-image |r| <= cutoff, decided
// in FP64 so the pair set is the same in both precisions, leaving out the
// scaled (1-n / polarization-group) partners of i (xoff/xidx, CSR), which
// the FP64 scaled-pair kernels evaluate.  One warp per site (sites taken in
// cell order); the lanes scan a stencil cell together and compact the hits
// with a ballot, so each list is in cell order, then index order.  Stored
// site-major: nbr[i * cap + s] holds the partner, cnb[i * cap + s] its
// position in cell order (the index the pair kernels gather with).
__global__ void k_neighbors(int n, const double4* __restrict__ spos, const unsigned* __restrict__ skeys,
                            const int* __restrict__ sids, const int* __restrict__ cstart,
                            const int* __restrict__ cend, CellGrid cg, Box bx, double cut2, int cap,
                            const int* __restrict__ xoff, const int* __restrict__ xidx, const int2* __restrict__ xrange,
                            int* __restrict__ nbr, int* __restrict__ cnb, int* __restrict__ nnb,
                            int* __restrict__ overflow) {
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (w >= n) return;  // whole warps exit together
    const int i = sids[w];
    const unsigned key = skeys[w];
    const int c2 = key % cg.nc[2];
    const int c1 = (key / cg.nc[2]) % cg.nc[1];
    const int c0 = key / (cg.nc[2] * cg.nc[1]);
    const double4 pi = spos[w];
    const int x0 = xoff[i], x1 = xoff[i + 1];
    const int2 xr = xrange[i];  // index range of i's scaled partners
    const int limit = cap - (x1 - x0);  // the row's tail holds the scaled partners
    int* row = nbr + (size_t)i * cap;
    int cnt = 0;
    for (int dx = cg.off_lo[0]; dx <= cg.off_hi[0]; dx++) {
        int q0 = c0 + dx;
        if (cg.periodic) q0 = (q0 + cg.nc[0]) % cg.nc[0];
        else if (q0 < 0 || q0 >= cg.nc[0]) continue;
        for (int dy = cg.off_lo[1]; dy <= cg.off_hi[1]; dy++) {
            int q1 = c1 + dy;
            if (cg.periodic) q1 = (q1 + cg.nc[1]) % cg.nc[1];
            else if (q1 < 0 || q1 >= cg.nc[1]) continue;
            for (int dz = cg.off_lo[2]; dz <= cg.off_hi[2]; dz++) {
                int q2 = c2 + dz;
                if (cg.periodic) q2 = (q2 + cg.nc[2]) % cg.nc[2];
                else if (q2 < 0 || q2 >= cg.nc[2]) continue;
                const int cell = (q0 * cg.nc[1] + q1) * cg.nc[2] + q2;
                const int s = cstart[cell], e = cend[cell];
                for (int base = s; base < e; base += 32) {
                    const int p = base + lane;
                    bool hit = false;
                    int j = -1;
                    if (p < e) {
                        j = sids[p];
                        double4 pj = spos[p];
                        V3<double> r = min_image<double>(v3<double>(pj.x - pi.x, pj.y - pi.y, pj.z - pi.z), bx);
                        hit = j != i && dot(r, r) <= cut2;
                        if (hit && j >= xr.x && j <= xr.y)
                            for (int q = x0; q < x1; q++) hit &= (xidx[q] != j);
                    }
                    unsigned m = __ballot_sync(0xffffffffu, hit);
                    if (hit) {
                        int pos = cnt + __popc(m & ((1u << lane) - 1u));
                        if (pos < limit) {
                            row[pos] = j;
                            cnb[(size_t)i * cap + pos] = p;  // the partner's position in cell order
                        }
                    }
                    cnt += __popc(m);
                }
            }
        }
    }
    if (lane == 0) {
        nnb[i] = min(cnt, limit);
        if (cnt > limit) atomicMax(overflow, cnt + (x1 - x0));
    }
}

// The same exact neighbour list, one block per home cell, for boxes with at
// least 3 cells on every periodic axis (orthogonal cells; or the lattice's
// parallelepipeds of a monoclinic or triclinic cell, whose stencil images are
// lattice translations).  The atoms of the (up to) 27 stencil
// cells are staged in shared memory as FP32 positions relative to the home
// cell's corner (periodic coordinates first wrapped into the box, as the
// cell index does), each moved by its stencil cell's periodic image, so
// the inner loop is three FP32 differences and a dot product.  A pair whose
// FP32 squared distance lies within `margin` of cut^2 is decided again by the
// FP64 minimum-image test of k_neighbors, so both kernels give the same pair
// set; candidates are taken in the same order (stencil cells in x, y, z
// order, each in sorted order), so the rows are identical too.  Staging is
// chunked (kNbrChunk candidates, kNbrHome home atoms at a time), so any cell
// occupancy works.
constexpr int kNbrChunk = 1280;
constexpr int kNbrHome = 128;
constexpr int kNbrThreads = 256;

// CENTRED (truncated octahedron, rhombic dodecahedron): the stencil is the 27
// cells around the home cell plus the 27 around the cell half a prism away,
// whose sites reach the home cell by the centring translation; with an even
// count of at least 6 cells per axis the two stencils are disjoint, so each
// site is a candidate at most once, and every candidate within reach is
// decided by the cell's FP64 image().
template <bool GENERAL, bool CENTRED = false>
__global__ void __launch_bounds__(kNbrThreads) k_neighbors_cells(
    const double4* __restrict__ spos, const int* __restrict__ sids, const int* __restrict__ cstart,
    const int* __restrict__ cend, CellGrid cg, Box bx, double cut2, double margin, int cap,
    const int* __restrict__ xoff, const int* __restrict__ xidx, const int2* __restrict__ xrange, int* __restrict__ nbr,
    int* __restrict__ cnb, int* __restrict__ nnb,
    int* __restrict__ overflow) {
    __shared__ float4 cpos[kNbrChunk];
    __shared__ int csrt[kNbrChunk];  // sorted index
    __shared__ int cid[kNbrChunk];   // site index
    __shared__ int hcnt[kNbrHome];
    // home sites of the current chunk: position relative to the cell corner,
    // site index, scaled-partner range (CSR offsets) and index range
    __shared__ float4 hpos[kNbrHome];
    __shared__ int hid[kNbrHome], hx0[kNbrHome], hx1[kNbrHome];
    __shared__ int2 hxr[kNbrHome];
    __shared__ int rstart[54], rpre[55];
    __shared__ double rshift[54][3];
    __shared__ int nst;
    const int cell = blockIdx.x;
    const int hs = cstart[cell], he = cend[cell];
    if (he <= hs) return;  // empty cell: the whole block leaves
    const int c2 = cell % cg.nc[2], c1 = (cell / cg.nc[2]) % cg.nc[1], c0 = cell / (cg.nc[2] * cg.nc[1]);
    const int cc[3] = {c0, c1, c2};
    double corner[3];
#pragma unroll
    for (int a = 0; a < 3; a++) corner[a] = cg.origin[a] + cc[a] * cg.size[a];
    if (GENERAL)  // the cell's lowest lattice point
        for (int a = 0; a < 3; a++)
            corner[a] = (double)cc[0] / cg.nc[0] * cg.A[0][a] + (double)cc[1] / cg.nc[1] * cg.A[1][a] +
                        (double)cc[2] / cg.nc[2] * cg.A[2][a];
    if (threadIdx.x < 32) {
        // stencil cell k = lane (+ 32 in a second round: all of a warp's loads
        // of cstart/cend in flight at once), lengths summed by a warp scan;
        // cells outside an open system's grid count as empty
        const int na0 = cg.off_hi[0] - cg.off_lo[0] + 1, na1 = cg.off_hi[1] - cg.off_lo[1] + 1;
        const int na2 = cg.off_hi[2] - cg.off_lo[2] + 1;
        const int n27 = na0 * na1 * na2, total = CENTRED ? 2 * n27 : n27;
        int carry = 0;
        for (int k0 = 0; k0 < total; k0 += 32) {
            const int k = k0 + (int)threadIdx.x;
            int len = 0;
            if (k < total) {
                const int kk = k < n27 ? k : k - n27;  // the second 27: around the centred cell
                const int d[3] = {cg.off_lo[0] + kk / (na1 * na2), cg.off_lo[1] + (kk / na2) % na1,
                                  cg.off_lo[2] + kk % na2};
                int q[3];
                double sh[3];
                bool skip = false;
                int wrap[3] = {0, 0, 0};
                for (int a = 0; a < 3; a++) {
                    // prism edge: the centred grids' own, else the box's
                    const double La = CENTRED ? cg.size[a] * cg.nc[a] : bx.L[a];
                    const int half = (CENTRED && k >= n27) ? cg.nc[a] / 2 : 0;
                    q[a] = cc[a] + half + d[a];
                    sh[a] = half ? -0.5 * La : 0.0;  // the centring translation
                    if (cg.periodic) {
                        if (q[a] < 0) { q[a] += cg.nc[a]; sh[a] -= La; wrap[a] = -1; }
                        else if (q[a] >= cg.nc[a]) { q[a] -= cg.nc[a]; sh[a] += La; wrap[a] = 1; }
                    } else if (q[a] < 0 || q[a] >= cg.nc[a]) {
                        skip = true;
                    }
                }
                if (GENERAL)  // the periodic image is a lattice translation
                    for (int a = 0; a < 3; a++)
                        sh[a] = wrap[0] * cg.A[0][a] + wrap[1] * cg.A[1][a] + wrap[2] * cg.A[2][a];
                rstart[k] = 0;
                if (!skip) {
                    const int qc = (q[0] * cg.nc[1] + q[1]) * cg.nc[2] + q[2];
                    const int s0 = cstart[qc];
                    len = max(cend[qc] - s0, 0);
                    rstart[k] = s0;
                }
                for (int a = 0; a < 3; a++) rshift[k][a] = sh[a];
            }
            int incl = len;  // inclusive scan over the warp
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int v = __shfl_up_sync(0xffffffffu, incl, o);
                if ((int)threadIdx.x >= o) incl += v;
            }
            if (k < total) rpre[k] = carry + incl - len;
            if (k == total - 1) {
                rpre[total] = carry + incl;
                nst = total;
            }
            carry += __shfl_sync(0xffffffffu, incl, 31);
        }
    }
    __syncthreads();
    const int M = rpre[nst];
    // position in the box (periodic) relative to the home cell's corner;
    // a general cell wraps the fractional coordinates
    auto rel3 = [&](const double4& x, double (&o)[3]) {
        if (GENERAL) {
            double f[3];
            frac_wrapped(cg, x.x, x.y, x.z, f);
            for (int a = 0; a < 3; a++) o[a] = f[0] * cg.A[0][a] + f[1] * cg.A[1][a] + f[2] * cg.A[2][a] - corner[a];
            return;
        }
        const double xs[3] = {x.x, x.y, x.z};
        for (int a = 0; a < 3; a++) {
            double v = xs[a];
            if (CENTRED) {
                const double La = cg.size[a] * cg.nc[a];
                v -= La * floor(v / La);
            } else if (cg.periodic) {
                v -= bx.L[a] * floor(v * bx.iL[a]);
            }
            o[a] = v - corner[a];
        }
    };
    const float lo2 = (float)(cut2 - margin), hi2 = (float)(cut2 + margin);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarp = blockDim.x >> 5;
    const unsigned below = (1u << lane) - 1u;
    for (int h0 = hs; h0 < he; h0 += kNbrHome) {
        const int hn = min(kNbrHome, he - h0);
        for (int t = threadIdx.x; t < hn; t += blockDim.x) {
            // every thread loads one home site: the warps below then start
            // their scans without a chain of dependent global loads
            hcnt[t] = 0;
            const int i = sids[h0 + t];
            double h3[3];
            rel3(spos[h0 + t], h3);
            hpos[t] = make_float4((float)h3[0], (float)h3[1], (float)h3[2], 0.f);
            hid[t] = i;
            hx0[t] = xoff[i];
            hx1[t] = xoff[i + 1];
            hxr[t] = xrange[i];
        }
        for (int m0 = 0; m0 < M; m0 += kNbrChunk) {
            const int mn = min(kNbrChunk, M - m0);
            __syncthreads();  // the previous chunk is consumed and hcnt is initialised
            // stage the chunk one stencil cell at a time (cells overlapping it)
            for (int k = 0; k < nst; k++) {
                const int f0 = max(rpre[k], m0), f1 = min(rpre[k + 1], m0 + mn);
                for (int f = f0 + threadIdx.x; f < f1; f += blockDim.x) {
                    const int p = rstart[k] + (f - rpre[k]);
                    double c3[3];
                    rel3(spos[p], c3);
                    const int t = f - m0;
                    cpos[t] = make_float4((float)(c3[0] + rshift[k][0]), (float)(c3[1] + rshift[k][1]),
                                          (float)(c3[2] + rshift[k][2]), 0.f);
                    csrt[t] = p;
                    cid[t] = sids[p];
                }
            }
            __syncthreads();
            for (int hh = warp; hh < hn; hh += nwarp) {
                const int ph = h0 + hh;
                const int i = hid[hh];
                const float4 hp = hpos[hh];
                const float hx = hp.x, hy = hp.y, hz = hp.z;
                const int x0 = hx0[hh], x1 = hx1[hh];
                const int2 xr = hxr[hh];  // index range of i's scaled partners
                const int limit = cap - (x1 - x0);  // the row's tail holds the scaled partners
                // the first kExcl scaled partners in registers, the rest read when needed
                constexpr int kExcl = 8;
                int ex[kExcl];
#pragma unroll
                for (int q = 0; q < kExcl; q++) ex[q] = x0 + q < x1 ? xidx[x0 + q] : -1;
                int* row = nbr + (size_t)i * cap;
                int cnt = hcnt[hh];
                for (int b = 0; b < mn; b += 32) {
                    const int t = b + lane;
                    bool hit = false;
                    int j = -1;
                    if (t < mn) {
                        const float4 c = cpos[t];
                        const float dx = c.x - hx, dy = c.y - hy, dz = c.z - hz;
                        const float r2 = dx * dx + dy * dy + dz * dz;
                        if (r2 <= hi2) {
                            j = cid[t];
                            hit = j != i;
                            // near the cutoff the FP64 minimum image decides; in a
                            // general cell it decides every pair, so the pair set
                            // is that of the cell's image(), as in k_neighbors
                            if (hit && (r2 > lo2 || GENERAL || CENTRED)) {
                                const double4 xi = spos[ph];
                                const double4 pj = spos[csrt[t]];
                                const V3<double> r = min_image<double, GENERAL || CENTRED>(
                                    v3<double>(pj.x - xi.x, pj.y - xi.y, pj.z - xi.z), bx);
                                hit = dot(r, r) <= cut2;
                            }
                            if (hit && j >= xr.x && j <= xr.y) {  // only then can j be a scaled partner
#pragma unroll
                                for (int q = 0; q < kExcl; q++) hit &= (ex[q] != j);
                                for (int q = x0 + kExcl; q < x1; q++) hit &= (xidx[q] != j);
                            }
                        }
                    }
                    const unsigned m = __ballot_sync(0xffffffffu, hit);
                    if (hit) {
                        const int pos = cnt + __popc(m & below);
                        if (pos < limit) {
                            row[pos] = j;
                            cnb[(size_t)i * cap + pos] = csrt[t];  // the partner's position in cell order
                        }
                    }
                    cnt += __popc(m);
                }
                if (lane == 0) hcnt[hh] = cnt;
            }
        }
        __syncthreads();
        for (int t = threadIdx.x; t < hn; t += blockDim.x) {
            const int i = sids[h0 + t];
            const int nx = xoff[i + 1] - xoff[i];
            const int limit = cap - nx, cnt = hcnt[t];
            nnb[i] = min(cnt, limit);
            if (cnt > limit) atomicMax(overflow, cnt + nx);
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------- B-splines
// Cardinal B-spline weights of order P at the P grid points starting at
// floor(u) - P + 1, and their first three derivatives (Essmann et al. 1995):
//   b_n[s] = ((w + n - 1 - s) b_{n-1}[s-1] + (s + 1 - w) b_{n-1}[s]) / (n - 1)
// with w = u - floor(u); derivatives from the lower orders by differences.
template <class R, int P>
__device__ __forceinline__ void bspline_weights(double w, R (&th)[4][P]) {
    double b[P + 1][P];
    for (int n = 0; n <= P; n++)
        for (int s = 0; s < P; s++) b[n][s] = 0.0;
    b[1][0] = 1.0;
    for (int n = 2; n <= P; n++)
        for (int s = 0; s < n; s++) {
            double lo = s >= 1 ? b[n - 1][s - 1] : 0.0;
            double hi = s < n - 1 ? b[n - 1][s] : 0.0;
            b[n][s] = ((w + n - 1 - s) * lo + (s + 1 - w) * hi) / (n - 1);
        }
    auto B = [&](int n, int s) { return (s >= 0 && s < n) ? b[n][s] : 0.0; };
    for (int s = 0; s < P; s++) {
        th[0][s] = (R)b[P][s];
        th[1][s] = (R)(B(P - 1, s - 1) - B(P - 1, s));
        th[2][s] = (R)(B(P - 2, s - 2) - 2 * B(P - 2, s - 1) + B(P - 2, s));
        th[3][s] = (R)(B(P - 3, s - 3) - 3 * B(P - 3, s - 2) + 3 * B(P - 3, s - 1) - B(P - 3, s));
    }
}

// B-spline stencils (weights and three derivatives per axis, start indices)
// of a block of BS sites, computed once in FP64 and
// written through shared memory, so the block's rows (3 axes x 4 orders x P
// values per site, consecutive sites adjacent) leave as contiguous runs
// instead of 60 scattered words per thread; with WD the FP64 stencils, with
// WF the FP32 copy (the FP32 path rounds the same FP64 values), each with
// its start indices.
template <int P, int BS, bool WD, bool WF>
__global__ void __launch_bounds__(BS) k_bspline_rows(int n, const double* __restrict__ xyz, Box bx, Frac F, int3 K,
                                                    double* __restrict__ thd, int* __restrict__ k0d,
                                                    float* __restrict__ thf, int* __restrict__ k0f) {
    constexpr int W = 3 * 4 * P;
    __shared__ double sd[BS * W];
    const int i0 = blockIdx.x * BS, i = i0 + threadIdx.x;
    if (i < n) {
        const int Ks[3] = {K.x, K.y, K.z};
        const double x = xyz[3 * i], y = xyz[3 * i + 1], z = xyz[3 * i + 2];
        for (int a = 0; a < 3; a++) {
            double f = F.general ? (x * F.m[0][a] + y * F.m[1][a] + z * F.m[2][a]) / Ks[a]
                                 : (a == 0 ? x : a == 1 ? y : z) * bx.iL[a];
            f -= floor(f);
            const double u = f * Ks[a];
            const double fl = floor(u);
            double th[4][P];
            bspline_weights<double, P>(u - fl, th);
            int start = (int)fl - P + 1;
            if (start < 0) start += Ks[a];
            if (WD) k0d[3 * i + a] = start;
            if (WF) k0f[3 * i + a] = start;
            double* o = sd + threadIdx.x * W + a * 4 * P;
            for (int d = 0; d < 4; d++)
                for (int s = 0; s < P; s++) o[d * P + s] = th[d][s];
        }
    }
    __syncthreads();
    const int cnt = min(BS, n - i0) * W;
    for (int t = threadIdx.x; t < cnt; t += BS) {
        const double v = sd[t];
        if (WD) thd[(size_t)i0 * W + t] = v;
        if (WF) thf[(size_t)i0 * W + t] = (float)v;
    }
}

}  // namespace amg
