// Device helpers shared by the two truncated column-pivoted QR kernels
// (rrqr.cu: one reflector applied per pivot step; rrqr_blk.cu: LAPACK dlaqps
// blocking with the trailing update deferred over a block of pivot steps).
#pragma once

#include <cuda_runtime.h>

namespace spq {
namespace rrqr {

template <class T>
__device__ __forceinline__ T wsum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Sum over the CTA; red holds one slot per warp. Every thread gets the sum.
template <class T>
__device__ __forceinline__ T bsum(T v, T* red) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    v = wsum(v);
    __syncthreads();
    if (lane == 0) red[warp] = v;
    __syncthreads();
    if (warp == 0) {
        T r = lane < nw ? red[lane] : T(0);
        r = wsum(r);
        if (lane == 0) red[0] = r;
    }
    __syncthreads();
    return red[0];
}

// The same sum with one barrier: every warp reduces the per-warp slots itself
// (the same butterfly over the same slots as bsum's warp 0, so bitwise the
// same value). The caller guarantees a barrier between two calls on the same
// red (no thread may still be reading the slots of the previous call).
template <class T>
__device__ __forceinline__ T bsum1(T v, T* red) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    v = wsum(v);
    if (lane == 0) red[warp] = v;
    __syncthreads();
    return wsum(lane < nw ? red[lane] : T(0));
}

// LAPACK's tol3z = sqrt(unit roundoff): below it a downdated partial column
// norm is recomputed (dlaqp2 / dlaqps).
template <class T>
struct Tol3z;
template <>
struct Tol3z<double> {
    static __device__ __forceinline__ double v() { return 1.0536712127723509e-08; }  // sqrt(2^-53)
};
template <>
struct Tol3z<float> {
    static __device__ __forceinline__ float v() { return 2.44140625e-04f; }  // sqrt(2^-24)
};

__device__ __forceinline__ double dhypot(double a, double b) { return hypot(a, b); }
__device__ __forceinline__ float dhypot(float a, float b) { return hypotf(a, b); }

// 16-byte vector of adjacent row elements (columns of a row-major matrix).
template <class T>
struct Vec;
template <>
struct Vec<float> {
    using type = float4;
    static constexpr int n = 4;
};
template <>
struct Vec<double> {
    using type = double2;
    static constexpr int n = 2;
};

// Pivot candidates (value, position): the larger value wins, then the smaller
// position (the first index idamax returns).
template <class T>
__device__ __forceinline__ bool better(T v, int p, T bv, int bp) {
    return v > bv || (v == bv && p < bp);
}

// One pivot candidate as a 16-byte record (one DSMEM load).
template <class T>
struct __align__(16) Cand {
    T v;
    int p, c;
};

// Warp arg-max of (value, position, column) candidates; every lane gets the winner.
template <class T>
__device__ __forceinline__ void warp_best(T& v, int& p, int& c) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const T ov = __shfl_xor_sync(0xffffffffu, v, o);
        const int op = __shfl_xor_sync(0xffffffffu, p, o);
        const int oc = __shfl_xor_sync(0xffffffffu, c, o);
        if (better(ov, op, v, p)) {
            v = ov;
            p = op;
            c = oc;
        }
    }
}

}  // namespace rrqr
}  // namespace spq
