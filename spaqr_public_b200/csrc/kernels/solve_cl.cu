// Tall Q applications of the preconditioner sweeps on thread-block clusters
// (the Q^T / Q steps of Tree::solve, src/tree.cpp:1360-1460, for the
// elimination, scaling and sparsification reflectors).
//
// One SK_APPLYQ op of m rows (x(0:m) <- Q^T x for dir 0, Q x for dir 1, Q
// from unit-lower V with one kNB x kNB T factor per panel) runs on a cluster
// of CL CTAs, CTA cr holding rows [cr S, (cr + 1) S) with S = ceil(m / CL) <=
// 256: one row per thread, its x value in a register. A panel costs one pass
// that takes the row's kNB entries of V from registers and forms the kNB
// products v x, a warp transpose-sum and a CTA sum, the CTA's kNB sums stored
// into slot cr of every CTA of the cluster (DSMEM, double-buffered by panel
// parity) and released by a fence, then the next panel's V and T loads, one
// relaxed cluster barrier (the loads stay in flight through it: a releasing
// arrive would first wait for them), then in every warp y = the slots summed
// in rank order, z = T^T y (dir 0) or T y (dir 1) by lane shuffles, and
// x -= v^T z from the registers. V is read once per panel (the one-CTA form
// reads it twice and walks m / 256 rows per thread in each pass).
#include <cooperative_groups.h>

#include "kernels.hpp"
#include "pdl.cuh"

namespace spq {

namespace cg = cooperative_groups;

namespace {

constexpr int kAThreads = 256;
constexpr int kAWarps = kAThreads / 32;
constexpr int kAMaxCl = 16;

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
__global__ void __launch_bounds__(kAThreads) k_applyq_cl(const SolveOp* ops, const XSeg* segs, T* x) {
    pdl_enter();
    __shared__ T part[2][kAMaxCl][kNB];
    __shared__ T wred[kAWarps][kNB];
    __shared__ T tsh[2][kNB][kNB + 1];
    __shared__ T zw[kAWarps][kNB];
    cg::cluster_group cl = cg::this_cluster();
    const int CL = (int)cl.num_blocks();
    const int cr = (int)cl.block_rank();
    const SolveOp op = ops[blockIdx.x / CL];
    const int m = op.a, kq = op.b, ldv = op.c, dir = op.dir;
    const T* V = reinterpret_cast<const T*>(op.p0);
    const T* Tf = reinterpret_cast<const T*>(op.p1);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int S = (m + CL - 1) / CL;
    const int r0 = min(m, cr * S);
    const int nr = min(m, r0 + S) - r0;
    const int r = r0 + tid;
    const bool has = tid < nr;
    T* xp = nullptr;
    if (has) {
        if (op.nseg > 0) {
            int cur = 0;
            for (int s = 0; s < op.nseg; ++s) {
                const XSeg sg = segs[op.seg0 + s];
                if (r < cur + sg.len) {
                    xp = x + sg.xoff + (r - cur);
                    break;
                }
                cur += sg.len;
            }
        } else {
            xp = x + op.x0 + r;
        }
    }
    T xr = has ? *xp : T(0);
    const int rl = has ? r : 0;  // a row that exists, for the unconditional loads
    const int np = (kq + kNB - 1) / kNB;
    constexpr int TPT = kNB * kNB / kAThreads;  // T entries per thread
    // raw V entries and T entries of panel pi (loaded one panel ahead)
    T vraw[kNB], traw[TPT];
    auto load_panel = [&](int pi, T (&vd)[kNB], T (&td)[TPT]) {
        const int pidx = dir == 0 ? pi : np - 1 - pi;
        const int p0 = pidx * kNB;
        const int wl = min(kNB, kq - p0) - 1;
        const T* vr = V + (size_t)p0 * ldv + rl;
#pragma unroll
        for (int q = 0; q < kNB; ++q) vd[q] = vr[(size_t)min(q, wl) * ldv];
        const T* Tp = Tf + (size_t)pidx * kNB * kNB;
#pragma unroll
        for (int u = 0; u < TPT; ++u) td[u] = Tp[tid + u * kAThreads];
    };
    if (np > 0) load_panel(0, vraw, traw);
    for (int pi = 0; pi < np; ++pi) {
        const int buf = pi & 1;
        const int pidx = dir == 0 ? pi : np - 1 - pi;
        const int p0 = pidx * kNB;
        const int w = min(kNB, kq - p0);
#pragma unroll
        for (int u = 0; u < TPT; ++u) {
            const int e = tid + u * kAThreads;
            tsh[buf][e % kNB][e / kNB] = traw[u];
        }
        const int rr = r - p0;
        T v[kNB];
#pragma unroll
        for (int q = 0; q < kNB; ++q) {  // unit diagonal, zeros above it and past the panel
            const T vq = q < rr ? vraw[q] : (q == rr ? T(1) : T(0));
            v[q] = (has && q < w) ? vq : T(0);
        }
        T a[kNB];
#pragma unroll
        for (int q = 0; q < kNB; ++q) a[q] = v[q] * xr;
        wred[warp][lane] = tsum32(a);
        __syncthreads();
        {
            T s = T(0);
#pragma unroll
            for (int q = 0; q < kAWarps; ++q) s += wred[q][lane];
            for (int dst = warp; dst < CL; dst += kAWarps) *cl.map_shared_rank(&part[buf][cr][lane], dst) = s;
        }
        asm volatile("fence.acq_rel.cluster;" ::: "memory");
        if (pi + 1 < np) load_panel(pi + 1, vraw, traw);
        asm volatile("barrier.cluster.arrive.relaxed.aligned;" ::: "memory");
        asm volatile("barrier.cluster.wait.aligned;" ::: "memory");
        T y = T(0);
        for (int q = 0; q < CL; ++q) y += part[buf][q][lane];
        T z = T(0);  // lane j: z_j = sum_l T(l, j) y_l (dir 0) or T(j, l) y_l (dir 1); zero past w
        if (dir == 0) {
#pragma unroll
            for (int l = 0; l < kNB; ++l) {
                const T yl = __shfl_sync(0xffffffffu, y, l);
                if (l <= lane) z += tsh[buf][l][lane] * yl;
            }
        } else {
#pragma unroll
            for (int l = 0; l < kNB; ++l) {
                const T yl = __shfl_sync(0xffffffffu, y, l);
                if (l >= lane && l < w) z += tsh[buf][lane][l] * yl;
            }
        }
        zw[warp][lane] = lane < w ? z : T(0);
        __syncwarp();
        T s = T(0);
#pragma unroll
        for (int q = 0; q < kNB; ++q) s += v[q] * zw[warp][q];
        xr -= s;
    }
    if (has) *xp = xr;
}


// One backward triangular op (SK_TRI, dir 0: x_c <- R^-1 (x_c - sum_b B_b x_b),
// the R^-1 solve of Tree::solve after the neighbour products, src/tree.cpp:
// 1440-1466 with the QR / ScaleD operations' backward steps) or one ScaleD /
// OrthD step whose Q^T was formed (SK_APPLYQ with p2 = Q^T, m x m column-major:
// x_c <- Q^T x_c for dir 0, x_c <- Q x_c as the transposed product for dir 1;
// the Q^T / Q steps of the scaling and the sparsification, src/tree.cpp:557,
// src/operations.cpp) on a cluster of CL CTAs, for ops whose matrices are too
// large for one CTA's load stream:
//   1. CTA cr sums B(:, j) x_j over its slice of the op's neighbour columns
//      (the blocks' columns concatenated, ceil(gc / CL) per CTA) for all k
//      rows into its shared memory;
//   2. one cluster barrier; every CTA forms xs = x_c - (p_0 + ... + p_{CL-1})
//      from the slices' partials read over DSMEM in rank order (the same
//      values in every CTA); a second barrier, after which no CTA reads
//      another's shared memory and x_c may be written;
//   3. CTA cr writes rows [cr S, (cr + 1) S) of R^-1 xs, Q^T xs or Q xs (S =
//      ceil(k / CL)), or of xs itself where R is the identity (p0 == 0); Q xs
//      reads columns of Q^T, a warp per row with the lanes along the column.
// Results are deterministic for a given cluster size; they differ from the
// one-CTA form only by the order of the neighbour sums.
constexpr int kTThreads = 256;
constexpr int kTGU = 16;  // loads in flight per thread in the products

template <class T>
__global__ void __launch_bounds__(kTThreads) k_tri_cl(const SolveOp* ops, const GemvRef<T>* gemv, T* x) {
    pdl_enter();
    extern __shared__ __align__(16) unsigned char tri_raw[];
    __shared__ GemvRef<T> refs[kTriMaxRefs];
    __shared__ int cstart[kTriMaxRefs + 1];
    __shared__ T red[kTThreads];
    cg::cluster_group cl = cg::this_cluster();
    const int CL = (int)cl.num_blocks();
    const int cr = (int)cl.block_rank();
    const SolveOp op = ops[blockIdx.x / CL];
    const bool dense = op.kind == SK_APPLYQ;  // Q^T, full; else R^-1, upper triangular
    const int k = op.a, nb = dense ? 0 : op.nseg;
    T* part = reinterpret_cast<T*>(tri_raw);  // this CTA's partial sums (k)
    T* xs = part + k;                         // the reduced right-hand side (k)
    T* xc = x + op.x0;
    const int tid = threadIdx.x;
    for (int b = tid; b < nb; b += kTThreads) refs[b] = gemv[op.seg0 + b];
    __syncthreads();
    if (tid == 0) {
        int c = 0;
        for (int b = 0; b < nb; ++b) {
            cstart[b] = c;
            c += refs[b].s;
        }
        cstart[nb] = c;
    }
    __syncthreads();
    // 1. partial neighbour products over this CTA's column slice
    const int gc = cstart[nb];
    const int sc = (gc + CL - 1) / CL;
    const int c0 = min(gc, cr * sc), c1 = min(gc, c0 + sc);
    {
        const int RT = min(kTThreads, (k + 31) & ~31);
        const int G = kTThreads / RT;
        const int ri = tid % RT, g = tid / RT;
        for (int i0 = 0; i0 < k; i0 += RT) {
            const int i = i0 + ri;
            const int ic = min(i, k - 1);
            T a[4] = {T(0), T(0), T(0), T(0)};
            if (g < G) {
                for (int b = 0; b < nb; ++b) {
                    const int lo = max(c0, cstart[b]) - cstart[b], hi = min(c1, cstart[b + 1]) - cstart[b];
                    if (lo >= hi) continue;
                    const GemvRef<T> r = refs[b];
                    const T* B = reinterpret_cast<const T*>(r.boff) + ic;
                    const T* xn = x + r.xoff;
                    const size_t ld = (size_t)r.ld;
                    const int last = hi - 1;
                    for (int j = lo + g; j < hi; j += kTGU * G) {
                        T bv[kTGU], xv[kTGU];
#pragma unroll
                        for (int u = 0; u < kTGU; ++u) {
                            const int jj = min(j + u * G, last);
                            bv[u] = B[(size_t)jj * ld];
                            xv[u] = xn[jj];
                        }
#pragma unroll
                        for (int u = 0; u < kTGU; ++u)
                            if (j + u * G <= last) a[u & 3] += bv[u] * xv[u];
                    }
                }
            }
            red[tid] = (a[0] + a[1]) + (a[2] + a[3]);
            __syncthreads();
            if (g == 0 && i < k) {
                T sum = T(0);
                for (int q = 0; q < G; ++q) sum += red[q * RT + ri];
                part[i] = sum;
            }
            __syncthreads();
        }
    }
    cl.sync();
    // 2. xs = x_c - the partials in rank order
    if (gc == 0) {
        for (int i = tid; i < k; i += kTThreads) xs[i] = xc[i];
    } else {
        for (int i = tid; i < k; i += kTThreads) {
            T sum = T(0);
            for (int q = 0; q < CL; ++q) sum += *cl.map_shared_rank(part + i, q);
            xs[i] = xc[i] - sum;
        }
    }
    cl.sync();
    // 3. this CTA's rows of R^-1 xs (column-major, exactly zero below the
    //    diagonal: a warp starts at its first row) or of Q^T xs
    const int S = (k + CL - 1) / CL;
    const int r0 = min(k, cr * S), r1 = min(k, r0 + S);
    const T* Ri = dense ? reinterpret_cast<const T*>(op.p2)
                        : op.p1 != 0 ? reinterpret_cast<const T*>(op.p1) : nullptr;
    if (!Ri) {
        for (int i = r0 + tid; i < r1; i += kTThreads) xc[i] = xs[i];
        return;
    }
    const int nr = r1 - r0;
    if (nr <= 0) return;
    if (dense && op.dir == 1) {
        const int lane = tid & 31, warp = tid >> 5;
        for (int i = r0 + warp; i < r1; i += kTThreads / 32) {
            const T* col = Ri + (size_t)i * k;
            T a[4] = {T(0), T(0), T(0), T(0)};
            int j = lane;
            for (; j + 32 * (kTGU - 1) < k; j += 32 * kTGU) {
                T cv[kTGU];
#pragma unroll
                for (int u = 0; u < kTGU; ++u) cv[u] = col[j + 32 * u];
#pragma unroll
                for (int u = 0; u < kTGU; ++u) a[u & 3] += cv[u] * xs[j + 32 * u];
            }
            for (; j < k; j += 32) a[0] += col[j] * xs[j];
            T sum = (a[0] + a[1]) + (a[2] + a[3]);
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
            if (lane == 0) xc[i] = sum;
        }
        return;
    }
    const int RT = min(kTThreads, (nr + 31) & ~31);
    const int G = kTThreads / RT;
    const int ri = tid % RT, g = tid / RT;
    for (int i0 = r0; i0 < r1; i0 += RT) {
        const int i = i0 + ri;
        const int ic = min(i, k - 1);
        const int jb = dense ? 0 : min(i0 + (ri & ~31), k - 1);
        T a[4] = {T(0), T(0), T(0), T(0)};
        if (g < G) {
            int j = jb + g;
            for (; j + (kTGU - 1) * G < k; j += kTGU * G) {
                T rv[kTGU];
#pragma unroll
                for (int u = 0; u < kTGU; ++u) rv[u] = Ri[ic + (size_t)(j + u * G) * k];
#pragma unroll
                for (int u = 0; u < kTGU; ++u) a[u & 3] += rv[u] * xs[j + u * G];
            }
            for (; j < k; j += G) a[0] += Ri[ic + (size_t)j * k] * xs[j];
        }
        red[tid] = (a[0] + a[1]) + (a[2] + a[3]);
        __syncthreads();
        if (g == 0 && i < r1) {
            T sum = T(0);
            for (int q = 0; q < G; ++q) sum += red[q * RT + ri];
            xc[i] = sum;
        }
        __syncthreads();
    }
}

}  // namespace

template <class T>
cudaError_t launch_applyq_cl(const SolveOp* ops, int nops, int cluster, const XSeg* segs, T* x, cudaStream_t s) {
    if (nops <= 0) return cudaSuccess;
    if (cluster < 1 || cluster > kAMaxCl) return cudaErrorInvalidValue;
    once_per_device(reinterpret_cast<const void*>(&k_applyq_cl<T>), [] {
        cudaFuncSetAttribute(k_applyq_cl<T>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    });
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(nops * cluster), 1, 1);
    cfg.blockDim = dim3(kAThreads, 1, 1);
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
    return cudaLaunchKernelEx(&cfg, k_applyq_cl<T>, ops, segs, x);
}

template cudaError_t launch_applyq_cl<double>(const SolveOp*, int, int, const XSeg*, double*, cudaStream_t);
template cudaError_t launch_applyq_cl<float>(const SolveOp*, int, int, const XSeg*, float*, cudaStream_t);

template <class T>
cudaError_t launch_tri_cl(const SolveOp* ops, int nops, int cluster, int kmax, const GemvRef<T>* gemv, T* x,
                          cudaStream_t s) {
    if (nops <= 0) return cudaSuccess;
    if (cluster < 1 || cluster > kTriMaxCl || kmax < 1 || kmax > kRinvMax) return cudaErrorInvalidValue;
    once_per_device(reinterpret_cast<const void*>(&k_tri_cl<T>), [] {
        cudaFuncSetAttribute(k_tri_cl<T>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    });
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(nops * cluster), 1, 1);
    cfg.blockDim = dim3(kTThreads, 1, 1);
    cfg.dynamicSmemBytes = 2 * (size_t)kmax * sizeof(T);
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
    return cudaLaunchKernelEx(&cfg, k_tri_cl<T>, ops, gemv, x);
}

template cudaError_t launch_tri_cl<double>(const SolveOp*, int, int, int, const GemvRef<double>*, double*,
                                           cudaStream_t);
template cudaError_t launch_tri_cl<float>(const SolveOp*, int, int, int, const GemvRef<float>*, float*,
                                          cudaStream_t);

}  // namespace spq
