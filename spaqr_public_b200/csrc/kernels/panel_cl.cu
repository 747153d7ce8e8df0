// Householder panel factorization on a thread-block cluster (elimination and
// scaling panels, src/tree.cpp:263-276 via LAPACK dgeqrf / dlarft).
//
// One launch serves tasks of different heights: the launch's cluster has the
// largest size any listed task needs, and a task of cluster size CLt < CL uses
// its first CLt CTAs (the others only take part in the cluster barriers). A
// task's panel (R = m - p rows, w <= kNB columns) is cut into CLt row slabs,
// one per CTA, each held in shared memory for the whole panel (row-major, row
// stride kNB + 1). Column j costs:
//   1. one pass over the slab that first applies reflector j-1 to each row
//      (held in registers) and then adds the row's products into
//      g[c] = sum_{r > j} P[r, j] P[r, c] for all c (g[j] is the squared norm
//      below the diagonal); warp transpose-sums into shared memory;
//   2. one CTA barrier, after which every warp sums the warp partials (fixed
//      order) and stores this CTA's column sums into slot `cr` of every CTA of
//      the task (DSMEM stores, double-buffered by column parity); CTA 0 also
//      stores row j of the panel;
//   3. one cluster barrier (release / acquire: the stores are visible);
//   4. every warp of every CTA sums the slots in rank order from its own
//      shared memory and forms the reflector (LAPACK dlarfg: beta, tau, scale)
//      and d[c] = P[j, c] + scale g[c] = v_j^T P[:, c] (also the Gram entry
//      v_c^T v_j of the panel's T factor for c < j): the same arithmetic
//      everywhere, so every thread holds the same reflector.
// No CTA reads another's shared memory, so nothing waits at the end. CTA 0
// builds T (forward, columnwise) and every CTA writes its slab back. The sums
// are taken in the order of a per-column two-barrier form (rows of a thread,
// lanes, warps, CTAs), so the result depends only on CLt.
#include <cooperative_groups.h>

#include <algorithm>

#include "kernels.hpp"
#include "pdl.cuh"
#include "status.cuh"

namespace spq {

namespace cg = cooperative_groups;

namespace {

constexpr int kPThreads = 256;
constexpr int kPWarps = kPThreads / 32;
constexpr int kPS = kNB + 1;  // shared row stride
constexpr int kMaxCl = 16;
constexpr size_t kPanelDynSmem = 200 * 1024;

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

// ids[0:n] task indices, ids[n:2n] their cluster sizes (1 <= CLt <= cluster)
template <class T>
__global__ void __launch_bounds__(kPThreads) k_panel_cl(const QRTask<T>* tasks, const int* ids, int n, int p) {
    pdl_enter();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* P = reinterpret_cast<T*>(smem_raw);  // slab rows x kPS
    // column sums by sender rank (2 x kMaxCl x kNB), then the warp partials
    // (kPWarps x kNB); after the column loop the same words hold T
    __shared__ __align__(16) T xbuf[2 * kMaxCl * kNB + kPWarps * kNB];
    __shared__ T rowj[2][kNB];       // row j of the panel (stored by CTA 0)
    __shared__ T s_d[kPWarps][kNB];  // each warp's copy of d for the pending reflector
    __shared__ T G[kNB * kPS];
    __shared__ T s_tau[kNB];
    static_assert(2 * kMaxCl * kNB + kPWarps * kNB >= kNB * kPS, "T must fit the reduction buffers");
    T* const part = xbuf;                     // [buf][sender][c]
    T* const wred = xbuf + 2 * kMaxCl * kNB;  // [warp][c]
    cg::cluster_group cl = cg::this_cluster();
    const int CL = (int)cl.num_blocks();
    const int cr = (int)cl.block_rank();
    const int slot = blockIdx.x / CL;
    const QRTask<T> t = tasks[ids[slot]];
    const int CLt = ids[n + slot];
    const int m = t.m, k = t.k;
    if (p >= k) return;  // the same for every CTA of the cluster
    const int w = min(kNB, k - p);
    const int R = m - p;
    const int jn = min(w, R);  // columns with rows below the diagonal
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nth = blockDim.x;
    if (cr >= CLt) {  // not used by this task: the task's cluster barriers only
        for (int j = 0; j < jn; ++j) cl.sync();
        return;
    }
    const int S = (R + CLt - 1) / CLt;  // slab height; the launcher keeps S >= kNB when CLt > 1
    const int r0 = min(R, cr * S), r1 = min(R, r0 + S);
    const int nr = r1 - r0;
    T* gp = t.fac + p + (size_t)p * m;  // panel origin (column-major, ld m)
    for (int e = tid; e < nr * kNB; e += nth) {
        const int i = e % nr, c = e / nr;
        P[i * kPS + c] = c < w ? gp[(r0 + i) + (size_t)c * m] : T(0);
    }
    __syncthreads();
    T tau = T(0), scal = T(1), beta = T(0);  // reflector j - 1
    const T* dw = s_d[warp];
    for (int j = 0; j <= jn; ++j) {
        const int buf = j & 1;
        const int jj = j - 1;
        const bool red = j < jn;
        T acc[kNB];
#pragma unroll
        for (int c = 0; c < kNB; ++c) acc[c] = T(0);
        for (int i = tid; i < nr; i += nth) {
            const int r = r0 + i;
            T* row = P + i * kPS;
            T pv[kNB];
#pragma unroll
            for (int c = 0; c < kNB; ++c) pv[c] = row[c];
            if (j > 0) {  // reflector j - 1 on this row
                if (r > jj) {
                    if (tau != T(0)) {
                        const T v = row[jj] * scal;
#pragma unroll
                        for (int c = 0; c < kNB; ++c) {
                            if (c == jj) pv[c] = v;
                            if (c > jj && c < w) pv[c] = pv[c] - (tau * dw[c]) * v;
                        }
                    }
                } else if (r == jj) {
#pragma unroll
                    for (int c = 0; c < kNB; ++c) {
                        if (c == jj) pv[c] = beta;
                        if (tau != T(0) && c > jj && c < w) pv[c] -= tau * dw[c];
                    }
                }
#pragma unroll
                for (int c = 0; c < kNB; ++c) row[c] = pv[c];
            }
            if (red) {
                T x = T(0);
#pragma unroll
                for (int c = 0; c < kNB; ++c)
                    if (c == j && r > j) x = pv[c];
#pragma unroll
                for (int c = 0; c < kNB; ++c) acc[c] += x * pv[c];
            }
        }
        if (!red) break;
        wred[warp * kNB + lane] = tsum32(acc);
        __syncthreads();
        {
            T s = T(0);
            for (int q = 0; q < kPWarps; ++q) s += wred[q * kNB + lane];
            for (int q = warp; q < CLt; q += kPWarps) *cl.map_shared_rank(&part[(buf * kMaxCl + cr) * kNB + lane], q) = s;
            if (cr == 0) {
                const T rv = P[j * kPS + lane];
                for (int q = warp; q < CLt; q += kPWarps) *cl.map_shared_rank(&rowj[buf][lane], q) = rv;
            }
        }
        cl.sync();
        T g = T(0);
        for (int q = 0; q < CLt; ++q) g += part[(buf * kMaxCl + q) * kNB + lane];
        const T alpha = rowj[buf][j];
        const T xn2 = __shfl_sync(0xffffffffu, g, j);
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
        const T dm = rowj[buf][lane] + scal * g;
        s_d[warp][lane] = dm;
        if (cr == 0 && warp == 0) {
            if (lane < j) G[lane * kPS + j] = dm;  // v_lane^T v_j
            if (lane == 0) {
                s_tau[j] = tau;
                note_qr_pivot(t.status, beta);
            }
        }
        __syncwarp();
    }
    __syncthreads();  // every warp is past its last read of the column sums
    if (cr == 0) {
        T* Ts = xbuf;
        for (int j = max(jn, 0) + tid; j < w; j += nth) {  // no rows below: tau = 0
            s_tau[j] = T(0);
            for (int l = 0; l < j; ++l) G[l * kPS + j] = T(0);
        }
        __syncthreads();
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


// Register-resident panel for slabs of at most 32 * kRPL rows (one CTA per
// slab, a cluster of CLt CTAs per task as above; kCl: the launch has
// clusters of more than one CTA). Rows past the slab hold zeros, so the
// result does not depend on kRPL. Warp w owns panel columns 4w .. 4w+3; lane
// l holds slab rows l + 32 i (i < kRPL) of them in registers. Column j costs:
//   1. the warp owning column j stores it below the diagonal (x, unscaled)
//      to shared memory; CTA barrier;
//   2. every warp forms g[c] = x^T P[:, c] for its four columns (kRPL FMAs
//      per lane, then a transposed reduction: two exchange steps leave lane
//      group q (lanes 8q .. 8q+7) with column q, three more sum the group);
//      g[j] is the squared norm;
//   3. the per-CTA sums go to slot `cr` of every CTA of the task, and CTA 0
//      sends row j of the panel (DSMEM stores); one cluster barrier (a CTA
//      barrier without clusters);
//   4. every warp sums the slots in rank order, forms the reflector (LAPACK
//      dlarfg) and d[c] = P[j, c] + scale g[c] = v_j^T P[:, c] (the Gram entry
//      v_c^T v_j for c < j), and updates its columns in registers with one
//      FMA per element, P[r, c] += (-tau d[c]) v[r] (coefficient zero for the
//      finished columns), the owner then writing v and beta into column j.
template <class T, bool kCl, int kRPL>
__global__ void __launch_bounds__(kPThreads, ((sizeof(T) == 4 && kRPL < 16) || kRPL < 8) ? 2 : 1) k_panel_reg(const QRTask<T>* tasks, const int* ids, int n, int p) {
    pdl_enter();
    constexpr int CPW = kNB / kPWarps;  // columns per warp
    constexpr int SR = 32 * kRPL;       // slab rows
    static_assert(CPW == 4, "the transposed reduction assumes four columns per warp");
    __shared__ T xs[2][SR];
    __shared__ T part[2][kCl ? kMaxCl : 1][kNB];
    __shared__ T rowj[2][kNB];
    __shared__ T G[kNB * kPS];
    __shared__ T Ts[kNB * kPS];
    __shared__ T s_tau[kNB];
    cg::cluster_group cl = cg::this_cluster();
    const int CL = kCl ? (int)cl.num_blocks() : 1;
    const int cr = kCl ? (int)cl.block_rank() : 0;
    const int slot = blockIdx.x / CL;
    const QRTask<T> t = tasks[ids[slot]];
    const int CLt = kCl ? ids[n + slot] : 1;
    const int m = t.m, k = t.k;
    if (p >= k) return;  // the same for every CTA of the cluster
    const int w = min(kNB, k - p);
    const int R = m - p;
    const int jn = min(w, R);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (kCl && cr >= CLt) {
        for (int j = 0; j < jn; ++j) cl.sync();
        return;
    }
    const int S = (R + CLt - 1) / CLt;  // <= SR; >= kNB when CLt > 1 (row j < kNB lies in CTA 0)
    const int r0 = min(R, cr * S);
    const int nr = min(R, r0 + S) - r0;
    T* gp = t.fac + p + (size_t)p * m;
    T a[kRPL][CPW];
#pragma unroll
    for (int i = 0; i < kRPL; ++i) {
        const int r = lane + 32 * i;
#pragma unroll
        for (int q = 0; q < CPW; ++q) {
            const int c = warp * CPW + q;
            a[i][q] = (r < nr && c < w) ? gp[(r0 + r) + (size_t)c * m] : T(0);
        }
    }
    const bool u16 = (lane & 16) != 0, u8 = (lane & 8) != 0;
    const int qi = (u16 ? 2 : 0) + (u8 ? 1 : 0);  // the column this lane's reduction ends with
    const int cq = warp * CPW + qi;
    for (int j = 0; j < jn; ++j) {
        const int buf = j & 1;
        const int ow = j / CPW, oq = j % CPW;
        if (warp == ow) {
#pragma unroll
            for (int i = 0; i < kRPL; ++i) {
                T xv = a[i][0];
#pragma unroll
                for (int q = 1; q < CPW; ++q)
                    if (q == oq) xv = a[i][q];
                xs[buf][lane + 32 * i] = r0 + lane + 32 * i > j ? xv : T(0);
            }
        }
        __syncthreads();
        T xr[kRPL];
        T g[CPW];
#pragma unroll
        for (int q = 0; q < CPW; ++q) g[q] = T(0);
#pragma unroll
        for (int i = 0; i < kRPL; ++i) {
            xr[i] = xs[buf][lane + 32 * i];
#pragma unroll
            for (int q = 0; q < CPW; ++q) g[q] += xr[i] * a[i][q];
        }
        const T h0 = (u16 ? g[2] : g[0]) + __shfl_xor_sync(0xffffffffu, u16 ? g[0] : g[2], 16);
        const T h1 = (u16 ? g[3] : g[1]) + __shfl_xor_sync(0xffffffffu, u16 ? g[1] : g[3], 16);
        T gs = (u8 ? h1 : h0) + __shfl_xor_sync(0xffffffffu, u8 ? h0 : h1, 8);
        gs += __shfl_xor_sync(0xffffffffu, gs, 4);
        gs += __shfl_xor_sync(0xffffffffu, gs, 2);
        gs += __shfl_xor_sync(0xffffffffu, gs, 1);
        T rq = T(0);  // P[j, cq] (CTA 0: row j is lane j's register row 0)
        if (cr == 0) {
#pragma unroll
            for (int q = 0; q < CPW; ++q) {
                const T v = __shfl_sync(0xffffffffu, a[0][q], j);
                if (q == qi) rq = v;
            }
        }
        if (kCl) {
            for (int dst = lane & 7; dst < CLt; dst += 8) {
                *cl.map_shared_rank(&part[buf][cr][cq], dst) = gs;
                if (cr == 0) *cl.map_shared_rank(&rowj[buf][cq], dst) = rq;
            }
            cl.sync();
        } else {
            if ((lane & 7) == 0) {
                part[buf][0][cq] = gs;
                rowj[buf][cq] = rq;
            }
            __syncthreads();
        }
        T xn2 = part[buf][0][j];
        if (kCl)
            for (int u = 1; u < CLt; ++u) xn2 += part[buf][u][j];
        const T alpha = rowj[buf][j];
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
        if (threadIdx.x == 0 && (!kCl || cr == 0)) note_qr_pivot(t.status, beta);
        T coef[CPW];
#pragma unroll
        for (int q = 0; q < CPW; ++q) {
            const int c = warp * CPW + q;
            T gsum = part[buf][0][c];
            if (kCl)
                for (int u = 1; u < CLt; ++u) gsum += part[buf][u][c];
            const T dq = rowj[buf][c] + scal * gsum;
            if (cr == 0 && lane == 0 && c < j) G[c * kPS + j] = dq;  // v_c^T v_j
            coef[q] = (c > j && c < w) ? -(tau * dq) : T(0);
        }
        if (cr == 0 && tid == 0) s_tau[j] = tau;
        if (tau != T(0)) {
            T v[kRPL];
#pragma unroll
            for (int i = 0; i < kRPL; ++i) v[i] = xr[i] * scal;  // zero at and above the diagonal
            if (cr == 0 && lane == j) v[0] = T(1);                // row j (unit diagonal of v_j)
#pragma unroll
            for (int i = 0; i < kRPL; ++i)
#pragma unroll
                for (int q = 0; q < CPW; ++q) a[i][q] += coef[q] * v[i];
            if (warp == ow) {
#pragma unroll
                for (int i = 0; i < kRPL; ++i) {
                    const int gr = r0 + lane + 32 * i;
#pragma unroll
                    for (int q = 0; q < CPW; ++q)
                        if (q == oq && gr >= j) a[i][q] = gr > j ? v[i] : beta;
                }
            }
        }
    }
#pragma unroll
    for (int i = 0; i < kRPL; ++i) {
        const int r = lane + 32 * i;
#pragma unroll
        for (int q = 0; q < CPW; ++q) {
            const int c = warp * CPW + q;
            if (r < nr && c < w) gp[(r0 + r) + (size_t)c * m] = a[i][q];
        }
    }
    if (cr == 0) {
        for (int j = max(jn, 0) + tid; j < w; j += kPThreads) {  // no rows below: tau = 0
            s_tau[j] = T(0);
            for (int l = 0; l < j; ++l) G[l * kPS + j] = T(0);
        }
        __syncthreads();
        for (int j = tid; j < w; j += kPThreads) t.tau[p + j] = s_tau[j];
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
        for (int e = tid; e < kNB * kNB; e += kPThreads) Tout[e] = Ts[(e % kNB) * kPS + (e / kNB)];
    }
}

}  // namespace

template <class T>
size_t panel_cl_max_rows(int cluster) {
    return (size_t)cluster * (kPanelDynSmem / (kPS * sizeof(T)));
}

template <class T>
cudaError_t launch_panel_cl(const QRTask<T>* tasks, const int* ids, int ntasks, int cluster, int max_slab, int p,
                            cudaStream_t s) {
    if (ntasks <= 0) return cudaSuccess;
    if (cluster < 1 || cluster > kMaxCl) return cudaErrorInvalidValue;
    const size_t smem = (size_t)std::max(max_slab, 1) * kPS * sizeof(T);
    if (smem > kPanelDynSmem) return cudaErrorInvalidValue;
    once_per_device(reinterpret_cast<const void*>(&k_panel_cl<T>), [] {
        cudaFuncSetAttribute(k_panel_cl<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kPanelDynSmem);
        cudaFuncSetAttribute(k_panel_cl<T>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    });
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(ntasks * cluster), 1, 1);
    cfg.blockDim = dim3(kPThreads, 1, 1);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute at[2];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = (unsigned)cluster;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    at[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;  // the kernel starts with pdl_enter()
    at[1].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 2;
    return cudaLaunchKernelEx(&cfg, k_panel_cl<T>, tasks, ids, ntasks, p);
}

template <class T, int RPL>
cudaError_t launch_panel_reg_rpl(const QRTask<T>* tasks, const int* ids, int ntasks, int cluster, int p,
                                 cudaStream_t s) {
    if (cluster == 1) {
        return launch_pdl(k_panel_reg<T, false, RPL>, dim3(ntasks), dim3(kPThreads), 0, s, 0, tasks, ids, ntasks, p);
    }
    once_per_device(reinterpret_cast<const void*>(&k_panel_reg<T, true, RPL>), [] {
        cudaFuncSetAttribute(k_panel_reg<T, true, RPL>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    });
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(ntasks * cluster), 1, 1);
    cfg.blockDim = dim3(kPThreads, 1, 1);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute at[2];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = (unsigned)cluster;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    at[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;  // the kernel starts with pdl_enter()
    at[1].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 2;
    return cudaLaunchKernelEx(&cfg, k_panel_reg<T, true, RPL>, tasks, ids, ntasks, p);
}

template <class T>
cudaError_t launch_panel_reg(const QRTask<T>* tasks, const int* ids, int ntasks, int cluster, int max_slab, int p,
                             cudaStream_t s) {
    if (ntasks <= 0) return cudaSuccess;
    if (cluster < 1 || cluster > kMaxCl || max_slab > 2 * kPanelRegRows) return cudaErrorInvalidValue;
    if (max_slab <= 64) return launch_panel_reg_rpl<T, 2>(tasks, ids, ntasks, cluster, p, s);
    if (max_slab <= 128) return launch_panel_reg_rpl<T, 4>(tasks, ids, ntasks, cluster, p, s);
    if (max_slab <= kPanelRegRows) return launch_panel_reg_rpl<T, 8>(tasks, ids, ntasks, cluster, p, s);
    if (sizeof(T) != 4) return cudaErrorInvalidValue;
    return launch_panel_reg_rpl<T, 16>(tasks, ids, ntasks, cluster, p, s);
}

template cudaError_t launch_panel_reg<double>(const QRTask<double>*, const int*, int, int, int, int, cudaStream_t);
template cudaError_t launch_panel_reg<float>(const QRTask<float>*, const int*, int, int, int, int, cudaStream_t);
template size_t panel_cl_max_rows<double>(int);
template size_t panel_cl_max_rows<float>(int);
template cudaError_t launch_panel_cl<double>(const QRTask<double>*, const int*, int, int, int, int, cudaStream_t);
template cudaError_t launch_panel_cl<float>(const QRTask<float>*, const int*, int, int, int, int, cudaStream_t);

}  // namespace spq
