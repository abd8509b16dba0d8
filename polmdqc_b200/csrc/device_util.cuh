// device_util.cuh -- small device helpers shared by the kernels.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

namespace amg {

template <class R>
struct R4T;
template <>
struct R4T<float> {
    using type = float4;
};
template <>
struct R4T<double> {
    using type = double4;
};
template <class R>
using R4 = typename R4T<R>::type;

template <class R>
__host__ __device__ __forceinline__ R4<R> make_r4(R a, R b, R c, R d) {
    R4<R> v;
    v.x = a; v.y = b; v.z = c; v.w = d;
    return v;
}

// sum over a warp
template <class T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// sum over an aligned group of G consecutive lanes (G = 2..32), the result in
// every lane of the group; all 32 lanes of the warp must take part
template <int G, class T>
__device__ __forceinline__ T group_sum(T v) {
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// block-wide sum of one double per thread; lane 0 of warp 0 adds the result
// to *out (one atomic per block).  blockDim.x must be a multiple of 32.
__device__ __forceinline__ void block_sum_add(double v, double* out) {
    __shared__ double part[32];
    v = warp_sum(v);
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) part[w] = v;
    __syncthreads();
    if (w == 0) {
        int nw = (blockDim.x + 31) >> 5;
        double s = lane < nw ? part[lane] : 0.0;
        s = warp_sum(s);
        if (lane == 0 && s != 0.0) atomicAdd(out, s);
    }
    __syncthreads();
}

__device__ __forceinline__ void block_sum_add_ll(long long v, unsigned long long* out) {
    __shared__ long long part[32];
    v = warp_sum(v);
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) part[w] = v;
    __syncthreads();
    if (w == 0) {
        int nw = (blockDim.x + 31) >> 5;
        long long s = lane < nw ? part[lane] : 0;
        s = warp_sum(s);
        if (lane == 0 && s != 0) atomicAdd(out, (unsigned long long)s);
    }
    __syncthreads();
}

// Virial (dE/d(strain), symmetrised) as six sums: xx yy zz xy xz yz.
// v += s sym(g (x) r): the strain derivative of a term whose gradient with
// respect to the separation r is g.
__device__ __forceinline__ void vir_outer(double (&v)[6], double gx, double gy, double gz, double rx, double ry,
                                          double rz, double s) {
    v[0] += s * gx * rx;
    v[1] += s * gy * ry;
    v[2] += s * gz * rz;
    v[3] += 0.5 * s * (gx * ry + gy * rx);
    v[4] += 0.5 * s * (gx * rz + gz * rx);
    v[5] += 0.5 * s * (gy * rz + gz * ry);
}

// block-wide sums of the six virial components into out[0..5]; every thread
// of the block must call it
__device__ __forceinline__ void block_vir_add(const double (&v)[6], double* out) {
#pragma unroll
    for (int c = 0; c < 6; c++) block_sum_add(v[c], out + c);
}

// minimum image in an orthogonal box (box <= 0 on an axis: no wrapping)
template <class R>
__device__ __forceinline__ R wrap1(R d, R L, R iL) {
    return L > R(0) ? d - L * rint(d * iL) : d;
}

}  // namespace amg
