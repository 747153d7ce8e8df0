// Householder panel factorization on a thread-block cluster (elimination and
// scaling panels, src/tree.cpp:263-276 via LAPACK dgeqrf / dlarft).
//
// A task's panel (R = m - p rows, w <= kNB columns) is cut into CL row slabs,
// one per CTA of a cluster, each held in shared memory for the whole panel
// (row-major, row stride kNB + 1). Column j of the panel costs:
//   A. one pass over the slab: g[c] = sum_{r > j} P[r, j] P[r, c] for all c
//      (g[j] is the squared norm below the diagonal), warp transpose-sums and
//      a CTA reduction into this CTA's partial (double-buffered by column
//      parity), CTA 0 also publishing row j;
//   B. one cluster barrier;
//   C. every CTA sums the CL partials (DSMEM, fixed order: identical results in
//      all CTAs) and forms the reflector (LAPACK dlarfg: beta, tau, scale) and
//      d[c] = P[j, c] + scale g[c] = v_j^T P[:, c], which is also the Gram entry
//      v_c^T v_j of the panel's T factor for c < j;
//   D. one pass that scales v_j and applies the rank-1 update to the later
//      columns.
// A final cluster barrier keeps every CTA alive until the last DSMEM reads of
// its partials are done. CTA 0 then builds T (forward, columnwise) and every
// CTA writes its slab back.
#include <cooperative_groups.h>

#include <algorithm>

#include "kernels.hpp"

namespace spq {

namespace cg = cooperative_groups;

namespace {

constexpr int kPThreads = 256;
constexpr int kPS = kNB + 1;  // shared row stride

template <class T>
__device__ __forceinline__ T hyp(T a, T b);
template <>
__device__ __forceinline__ double hyp<double>(double a, double b) { return hypot(a, b); }
template <>
__device__ __forceinline__ float hyp<float>(float a, float b) { return hypotf(a, b); }

template <class T>
__device__ __forceinline__ T tsum32(T (&a)[kNB]) {  // lane q returns sum over lanes of a[q]
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int s = 16; s >= 1; s >>= 1) {
        const bool upper = (lane & s) != 0;
#pragma unroll
        for (int q = 0; q < s; ++q) {
            const T send = upper ? a[q] : a[q + s];
            const T keep = upper ? a[q + s] : a[q];
            a[q] = keep + __shfl_xor_sync(0xffffffffu, send, s);
        }
    }
    return a[0];
}

template <class T>
__global__ void __launch_bounds__(kPThreads) k_panel_cl(const QRTask<T>* tasks, const int* ids, int p) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* P = reinterpret_cast<T*>(smem_raw);  // slab rows x kPS
    __shared__ T part[2][kNB];              // this CTA's column sums
    __shared__ T rowj[2][kNB];              // row j of the panel (CTA 0)
    __shared__ T wred[(kPThreads / 32) * kNB];
    __shared__ T s_d[kNB];
    __shared__ T G[kNB * kPS];
    __shared__ T Ts[kNB * kPS];
    __shared__ T s_tau[kNB];
    cg::cluster_group cl = cg::this_cluster();
    const int CL = (int)cl.num_blocks();
    const int cr = (int)cl.block_rank();
    const QRTask<T> t = tasks[ids[blockIdx.x / CL]];
    const int m = t.m, k = t.k;
    if (p >= k) return;  // the same for every CTA of the cluster
    const int w = min(kNB, k - p);
    const int R = m - p;
    const int S = (R + CL - 1) / CL;  // slab height; the launcher keeps S >= kNB when CL > 1
    const int r0 = min(R, cr * S), r1 = min(R, r0 + S);
    const int nr = r1 - r0;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5, nth = blockDim.x;
    T* gp = t.fac + p + (size_t)p * m;  // panel origin (column-major, ld m)
    for (int e = tid; e < nr * kNB; e += nth) {
        const int i = e % nr, c = e / nr;
        P[i * kPS + c] = c < w ? gp[(r0 + i) + (size_t)c * m] : T(0);
    }
    __syncthreads();
    for (int j = 0; j < w; ++j) {
        const int buf = j & 1;
        if (j >= R) {  // more columns than rows: nothing below, tau = 0 (uniform over the cluster)
            if (tid < j) G[tid * kPS + j] = T(0);
            if (tid == 0) s_tau[j] = T(0);
            continue;
        }
        // A. column sums of this slab over the rows below j
        T acc[kNB];
#pragma unroll
        for (int c = 0; c < kNB; ++c) acc[c] = T(0);
        for (int i = tid; i < nr; i += nth) {
            const int r = r0 + i;
            const T* row = P + i * kPS;
            const T x = r > j ? row[j] : T(0);
            T pv[kNB];
#pragma unroll
            for (int c = 0; c < kNB; ++c) pv[c] = row[c];
#pragma unroll
            for (int c = 0; c < kNB; ++c) acc[c] += x * pv[c];
        }
        const T ws = tsum32(acc);
        wred[warp * kNB + lane] = ws;
        __syncthreads();
        if (tid < kNB) {
            T s = T(0);
            for (int q = 0; q < nw; ++q) s += wred[q * kNB + tid];
            part[buf][tid] = s;
            if (cr == 0) rowj[buf][tid] = P[j * kPS + tid];
        }
        // B.
        cl.sync();
        // C. reflector and d (all CTAs, identical arithmetic)
        if (tid < kNB) {
            T g = T(0);
            for (int q = 0; q < CL; ++q) g += *cl.map_shared_rank(&part[buf][tid], q);
            s_d[tid] = g;  // g for now
        }
        __syncthreads();
        const T alpha = *cl.map_shared_rank(&rowj[buf][j], 0);
        const T xn2 = s_d[j];
        T tau, beta, scal;
        if (xn2 == T(0)) {
            tau = T(0);
            beta = alpha;
            scal = T(1);
        } else {
            const T nrm = hyp(alpha, (T)sqrt(xn2));
            beta = alpha >= T(0) ? -nrm : nrm;
            tau = (beta - alpha) / beta;
            scal = T(1) / (alpha - beta);
        }
        T dmine = T(0);
        if (tid < kNB) dmine = *cl.map_shared_rank(&rowj[buf][tid], 0) + scal * s_d[tid];
        __syncthreads();
        if (tid < kNB) {
            s_d[tid] = dmine;
            if (tid < j) G[tid * kPS + j] = dmine;  // v_tid^T v_j
            if (tid == 0) s_tau[j] = tau;
        }
        __syncthreads();
        // D. scale v_j and update the later columns
        for (int i = tid; i < nr; i += nth) {
            const int r = r0 + i;
            T* row = P + i * kPS;
            if (r > j) {
                T pv[kNB];
#pragma unroll
                for (int c = 0; c < kNB; ++c) pv[c] = row[c];
                const T xj = row[j];
                const T v = tau != T(0) ? xj * scal : xj;
                if (tau != T(0)) {
                    row[j] = v;
#pragma unroll
                    for (int c = 0; c < kNB; ++c)
                        if (c > j && c < w) row[c] = pv[c] - (tau * s_d[c]) * v;
                }
            } else if (r == j) {
                row[j] = beta;
                if (tau != T(0))
                    for (int c = j + 1; c < w; ++c) row[c] -= tau * s_d[c];
            }
        }
        __syncthreads();
    }
    // no CTA leaves while another may still read its partials
    cl.sync();
    if (cr == 0) {
        for (int j = tid; j < w; j += nth) t.tau[p + j] = s_tau[j];
        if (warp == 0) {  // T(0:j, j) = -tau_j T(0:j, 0:j) G(0:j, j)
            for (int j = 0; j < kNB; ++j) {
                if (j < w) {
                    const T tj = s_tau[j];
                    T tmp = T(0);
                    if (lane < j)
                        for (int l = lane; l < j; ++l) tmp += Ts[lane * kPS + l] * G[l * kPS + j];
                    if (lane < j) Ts[lane * kPS + j] = -tj * tmp;
                    if (lane == j) Ts[j * kPS + j] = tj;
                    if (lane > j) Ts[lane * kPS + j] = T(0);
                } else {
                    Ts[lane * kPS + j] = T(0);
                }
                __syncwarp();
            }
        }
        __syncthreads();
        T* Tout = t.tp + (size_t)(p / kNB) * kNB * kNB;
        for (int e = tid; e < kNB * kNB; e += nth) Tout[e] = Ts[(e % kNB) * kPS + (e / kNB)];
    }
    for (int e = tid; e < nr * w; e += nth) {
        const int i = e % nr, c = e / nr;
        gp[(r0 + i) + (size_t)c * m] = P[i * kPS + c];
    }
}

}  // namespace

template <class T>
size_t panel_cl_max_rows(int cluster) {
    return (size_t)cluster * ((200 * 1024) / (kPS * sizeof(T)));
}

template <class T>
cudaError_t launch_panel_cl(const QRTask<T>* tasks, const int* ids, int ntasks, int cluster, int max_rows, int p,
                            cudaStream_t s) {
    if (ntasks <= 0) return cudaSuccess;
    const int slab = (max_rows + cluster - 1) / cluster;
    const size_t smem = (size_t)std::max(slab, 1) * kPS * sizeof(T);
    if (smem > 200 * 1024) return cudaErrorInvalidValue;
    once_per_device(reinterpret_cast<const void*>(&k_panel_cl<T>), [] {
        cudaFuncSetAttribute(k_panel_cl<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
        cudaFuncSetAttribute(k_panel_cl<T>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    });
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(ntasks * cluster), 1, 1);
    cfg.blockDim = dim3(kPThreads, 1, 1);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = (unsigned)cluster;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, k_panel_cl<T>, tasks, ids, p);
}

template size_t panel_cl_max_rows<double>(int);
template size_t panel_cl_max_rows<float>(int);
template cudaError_t launch_panel_cl<double>(const QRTask<double>*, const int*, int, int, int, int, cudaStream_t);
template cudaError_t launch_panel_cl<float>(const QRTask<float>*, const int*, int, int, int, int, cudaStream_t);

}  // namespace spq
