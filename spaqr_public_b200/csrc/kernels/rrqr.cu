// Truncated column-pivoted Householder QR of the sparsification matrices
// (sparsifyD, src/tree.cpp:1022-1049; dgeqp3 + choose_rank, src/util.cpp:466-477,
// 795-816), one thread-block cluster per interface.
//
// Layout: C (m x n, m = interface columns, n = total neighbour width) is stored
// ROW-major with row stride ldc, so a thread that owns a column streams it
// with warp-coalesced accesses. Columns are never moved: the pivot order is
// kept as pos[column] / colat[position] exactly as LAPACK's swaps would leave
// it, so ties in the partial norms are broken by the current position (first
// index of idamax), and the norms travel with their columns.
//
// Per pivot step k, with the columns split in contiguous slabs over the CTAs
// of the cluster:
//   1. every CTA finds the largest partial norm of its active columns;
//      cluster barrier; every CTA reduces the candidates through DSMEM;
//   2. the CTA owning the pivot column builds the reflector (LAPACK dlarfg)
//      into its shared memory; cluster barrier; the others copy it through
//      DSMEM and all stop together if |R_kk| < tol |R_00|;
//   3. every CTA applies the reflector to its active columns and downdates
//      their norms (LAPACK dlaqp2 rule with recomputation below sqrt(eps)).
// The loop stops at the rank, so only rank steps of the O(m n r) work run.
#include <cooperative_groups.h>

#include <cfloat>
#include <algorithm>
#include <climits>

#include "kernels.hpp"
#include "pdl.cuh"

#include <stdexcept>
#include <string>
#include "rrqr_common.cuh"
#include "status.cuh"

namespace cg = cooperative_groups;

namespace spq {
namespace {

constexpr int kRRThreads = 512;
constexpr int kU = 4;  // column tiles per lane in the update passes

using namespace rrqr;

template <class T>
__global__ void __launch_bounds__(kRRThreads) k_rrqr_rm(const RRQRTaskRM<T>* tasks, const int* ids,
                                                         size_t smem_bytes) {
    pdl_enter();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* vsh = reinterpret_cast<T*>(smem_raw);
    __shared__ T red[32];
    __shared__ T wv[32];
    __shared__ int wp[32], wc[32];
    __shared__ T s_val, s_beta, s_tau;
    __shared__ int s_pos, s_col, s_gp, s_gc;

    cg::cluster_group cl = cg::this_cluster();
    const int CL = (int)cl.num_blocks();
    const int cr = (int)cl.block_rank();
    const RRQRTaskRM<T> t = tasks[ids[blockIdx.x / CL]];
    const int m = t.m, n = t.n;
    const size_t ld = (size_t)t.ldc;
    T* C = t.C;
    // slabs start on 32-column boundaries, so 16-byte column vectors never
    // straddle two CTAs (the row stride ldc is a multiple of 4)
    const int W = (((n + CL - 1) / CL) + 31) & ~31;
    const int j0 = min(n, cr * W), j1 = min(n, j0 + W);
    const int tid = threadIdx.x, nth = blockDim.x, lane = tid & 31, warp = tid >> 5, nw = nth >> 5;
    // shared memory: reflector (m) | dot partials (G x Wp) | per-column scale (Wp)
    const int mpad = (m + 7) & ~7;
    const int Wp = ((j1 - j0) + 32 * Vec<T>::n - 1) / (32 * Vec<T>::n) * (32 * Vec<T>::n);
    const int avail = (int)(smem_bytes / sizeof(T)) - mpad - Wp;
    const int G = max(1, min(16, Wp > 0 ? avail / Wp : 1));
    T* part = vsh + mpad;
    T* svec = part + (size_t)G * Wp;

    for (int j = j0 + tid; j < j1; j += nth) {
        T s = T(0);
#pragma unroll 8
        for (int i = 0; i < m; ++i) {
            const T v = C[i * ld + j];
            s += v * v;
        }
        const T nv = sqrt(s);
        t.vn1[j] = nv;
        t.vn2[j] = nv;
        t.pos[j] = j;
        t.colat[j] = j;
    }
    cl.sync();

    const int kmax = min(m, n);
    const double tol = t.tol;
    int rank = kmax;
    const int ksteps = (tol != 0.0 && tol >= 1.0) ? 0 : kmax;
    if (ksteps == 0) rank = (tol != 0.0 && tol >= 1.0) ? 0 : kmax;
    T r00 = T(0);
    for (int k = 0; k < ksteps; ++k) {
        // 1. pivot: largest partial norm, ties to the smallest position
        T bv = T(-1);
        int bp = INT_MAX, bc = -1;
        for (int j = j0 + tid; j < j1; j += nth) {
            const int p = t.pos[j];
            if (p < k) continue;
            const T v = t.vn1[j];
            if (better(v, p, bv, bp)) { bv = v; bp = p; bc = j; }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const T ov = __shfl_xor_sync(0xffffffffu, bv, o);
            const int op = __shfl_xor_sync(0xffffffffu, bp, o);
            const int oc = __shfl_xor_sync(0xffffffffu, bc, o);
            if (better(ov, op, bv, bp)) { bv = ov; bp = op; bc = oc; }
        }
        if (lane == 0) { wv[warp] = bv; wp[warp] = bp; wc[warp] = bc; }
        __syncthreads();
        if (warp == 0) {
            bv = lane < nw ? wv[lane] : T(-1);
            bp = lane < nw ? wp[lane] : INT_MAX;
            bc = lane < nw ? wc[lane] : -1;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const T ov = __shfl_xor_sync(0xffffffffu, bv, o);
                const int op = __shfl_xor_sync(0xffffffffu, bp, o);
                const int oc = __shfl_xor_sync(0xffffffffu, bc, o);
                if (better(ov, op, bv, bp)) { bv = ov; bp = op; bc = oc; }
            }
            if (lane == 0) { s_val = bv; s_pos = bp; s_col = bc; }
        }
        cl.sync();
        // every CTA reduces the cluster's candidates in parallel (lane r reads CTA r)
        if (warp == 0) {
            T v = T(-1);
            int p = INT_MAX, c = -1;
            if (lane < CL) {
                c = *cl.map_shared_rank(&s_col, lane);
                if (c >= 0) {
                    v = *cl.map_shared_rank(&s_val, lane);
                    p = *cl.map_shared_rank(&s_pos, lane);
                }
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const T ov = __shfl_xor_sync(0xffffffffu, v, o);
                const int op = __shfl_xor_sync(0xffffffffu, p, o);
                const int oc = __shfl_xor_sync(0xffffffffu, c, o);
                if (better(ov, op, v, p)) { v = ov; p = op; c = oc; }
            }
            if (lane == 0) { s_gp = p; s_gc = c; }
        }
        __syncthreads();
        const int gp = s_gp, gc = s_gc;
        const int pc = gc;
        if (pc < 0) {  // no finite partial norm left (NaN input): stop here, uniformly over the cluster
            rank = k;
            if (cr == 0 && tid == 0) note_rrqr_nan(t.status);
            break;
        }
        const int owner = pc / W;
        // 2. reflector of the pivot column (rows k..m-1) by its owner
        if (cr == owner) {
            T acc = T(0);
            for (int i = k + 1 + tid; i < m; i += nth) {
                const T v = C[i * ld + pc];
                acc += v * v;
            }
            const T xn2 = bsum(acc, red);
            const T alpha = C[k * ld + pc];
            T tau, beta, scal;
            if (xn2 == T(0)) {
                tau = T(0);
                beta = alpha;
                scal = T(1);
            } else {
                const T nrm = dhypot(alpha, (T)sqrt(xn2));
                beta = alpha >= T(0) ? -nrm : nrm;
                tau = (beta - alpha) / beta;
                scal = T(1) / (alpha - beta);
            }
            for (int i = k + 1 + tid; i < m; i += nth) {
                T v = C[i * ld + pc];
                if (tau != T(0)) {
                    v *= scal;
                    C[i * ld + pc] = v;
                }
                vsh[i] = v;
            }
            if (tid == 0) {
                vsh[k] = T(1);
                s_beta = beta;
                s_tau = tau;
                C[k * ld + pc] = beta;
                t.tau[k] = tau;
            }
            note_rrqr_pivot(tid == 0 ? t.status : nullptr, beta);
        }
        cl.sync();
        const T beta = *cl.map_shared_rank(&s_beta, owner);
        const T tau = *cl.map_shared_rank(&s_tau, owner);
        if (cr != owner) {
            const T* ov = cl.map_shared_rank(vsh, owner);
            for (int i = k + tid; i < m; i += nth) vsh[i] = ov[i];
        }
        if (tol != 0.0 && kmax > 1) {
            if (k == 0) {
                r00 = fabs(beta);
            } else if (!((double)fabs(beta) / (double)r00 >= tol)) {
                rank = k;
                break;  // uniform over the cluster: every CTA read the same beta
            }
        }
        if (cr == 0 && tid == 0) {  // LAPACK's column swap, as positions
            const int pvt = gp;
            const int c0 = t.colat[k];
            t.colat[pvt] = c0;
            t.pos[c0] = pvt;
            t.colat[k] = pc;
            t.pos[pc] = k;
        }
        __syncthreads();
        // 3. apply H_k to the active columns and downdate their norms. The slab
        //    is cut in 32-column tiles (lane = column: coalesced rows) and the
        //    rows below k in G chunks; warps take (chunk, tile) items so that no
        //    thread walks a whole column, and the chunk partials of each dot
        //    product meet in shared memory.
        // 3. apply H_k to the active columns and downdate their norms. Lanes own
        //    16-byte vectors of VEC adjacent columns (coalesced row segments),
        //    kU vectors per lane at once; the rows below k are cut into Gs chunks
        //    handled by different warps, whose dot partials meet in shared memory.
        constexpr int VEC = Vec<T>::n;
        constexpr int kRowUnroll = sizeof(T) == 4 ? 4 : 2;  // rows in flight per lane (registers)
        using VT = typename Vec<T>::type;
        const int Wc = j1 - j0;
        const int nvt = (Wc + 32 * VEC - 1) / (32 * VEC);  // 32-vector tiles in the slab
        const int ntg = (nvt + kU - 1) / kU;                 // groups of kU tiles per lane
        const int Gs = max(1, min(G, (m - k - 1 + 31) / 32));  // >= 32 rows per chunk
        const int Lr = (m - k - 1 + Gs - 1) / Gs;
        if (tau != T(0)) {
            for (int item = warp; item < Gs * ntg; item += nw) {
                const int g = item % Gs, tg = item / Gs;
                const int i0 = k + 1 + g * Lr, i1 = min(m, i0 + Lr);
                // vectors past the slab read its first vector instead (loads stay
                // unconditional, so all of a row's loads are in flight together);
                // their sums land in the unused tail of the partials
                T s[kU][VEC];
                const T* cp[kU];
#pragma unroll
                for (int u = 0; u < kU; ++u) {
#pragma unroll
                    for (int q = 0; q < VEC; ++q) s[u][q] = T(0);
                    const int jl = ((tg * kU + u) * 32 + lane) * VEC;
                    cp[u] = C + j0 + (jl < Wc ? jl : 0);
                }
#pragma unroll kRowUnroll
                for (int i = i0; i < i1; ++i) {
                    const T vi = vsh[i];
                    VT x[kU];
#pragma unroll
                    for (int u = 0; u < kU; ++u) x[u] = *reinterpret_cast<const VT*>(cp[u] + i * ld);
#pragma unroll
                    for (int u = 0; u < kU; ++u) {
                        const T* xs = reinterpret_cast<const T*>(&x[u]);
#pragma unroll
                        for (int q = 0; q < VEC; ++q) s[u][q] += vi * xs[q];
                    }
                }
#pragma unroll
                for (int u = 0; u < kU; ++u) {
                    const int jl = ((tg * kU + u) * 32 + lane) * VEC;
                    if (jl < Wp) {
#pragma unroll
                        for (int q = 0; q < VEC; ++q) part[g * Wp + jl + q] = s[u][q];
                    }
                }
            }
        }
        __syncthreads();
        for (int jl = tid; jl < Wc; jl += nth) {
            const int j = j0 + jl;
            T s = T(0);
            if (tau != T(0) && j != pc && t.pos[j] >= k) {
                s = C[k * ld + j];
                for (int g = 0; g < Gs; ++g) s += part[g * Wp + jl];
                s *= tau;
                C[k * ld + j] -= s;
            }
            svec[jl] = s;
        }
        for (int jl = Wc + tid; jl < Wp; jl += nth) svec[jl] = T(0);  // vector tail past the slab
        __syncthreads();
        if (tau != T(0)) {
            for (int item = warp; item < Gs * ntg; item += nw) {
                const int g = item % Gs, tg = item / Gs;
                const int i0 = k + 1 + g * Lr, i1 = min(m, i0 + Lr);
                T sc[kU][VEC];
                T* cp[kU];
                bool st[kU];  // vector inside the slab with a nonzero scale: store it
#pragma unroll
                for (int u = 0; u < kU; ++u) {
                    const int jl = ((tg * kU + u) * 32 + lane) * VEC;
                    bool any = false;
#pragma unroll
                    for (int q = 0; q < VEC; ++q) {
                        sc[u][q] = jl < Wc ? svec[jl + q] : T(0);
                        any = any || sc[u][q] != T(0);
                    }
                    st[u] = jl < Wc && any;
                    cp[u] = C + j0 + (jl < Wc ? jl : 0);
                }
#pragma unroll kRowUnroll
                for (int i = i0; i < i1; ++i) {
                    const T vi = vsh[i];
                    VT x[kU];
#pragma unroll
                    for (int u = 0; u < kU; ++u) x[u] = *reinterpret_cast<const VT*>(cp[u] + i * ld);
#pragma unroll
                    for (int u = 0; u < kU; ++u) {
                        T* xs = reinterpret_cast<T*>(&x[u]);
#pragma unroll
                        for (int q = 0; q < VEC; ++q) xs[q] -= sc[u][q] * vi;
                        if (st[u]) *reinterpret_cast<VT*>(cp[u] + i * ld) = x[u];
                    }
                }
            }
        }
        __syncthreads();
        for (int j = j0 + tid; j < j1; j += nth) {
            if (j == pc || t.pos[j] < k) continue;
            T* cj = C + j;
            const T n1 = t.vn1[j];
            if (n1 != T(0)) {
                const T rk = fabs(cj[k * ld]) / n1;
                T temp = T(1) - rk * rk;
                temp = temp < T(0) ? T(0) : temp;
                const T q = n1 / t.vn2[j];
                const T temp2 = temp * q * q;
                if (temp2 <= Tol3z<T>::v()) {
                    T ss = T(0);
                    for (int i = k + 1; i < m; ++i) ss += cj[i * ld] * cj[i * ld];
                    const T nv = (k + 1 < m) ? (T)sqrt(ss) : T(0);
                    t.vn1[j] = nv;
                    t.vn2[j] = nv;
                } else {
                    t.vn1[j] = n1 * (T)sqrt(temp);
                }
            }
        }
        cl.sync();  // positions of step k visible to every CTA before the next pivot search
    }
    // No CTA may exit while another still reads its shared memory (the early
    // exit at the rank leaves right after the DSMEM reads of that step).
    cl.sync();
    if (cr == 0 && tid == 0) *t.rank = rank;
}

// Write-back of a sparsified interface (sparsifyD, src/tree.cpp:1082-1110):
// Crank = R(0:r, :) un-permuted: Crank(i, c) = C(i, c) if i <= pos[c] else 0.
// CTA (task, y) of a (tasks x ny) grid takes the blocks b = y mod ny, the
// 32-column groups of V and the T panels with index = y mod ny. Row-major C
// is transposed into column-major blocks and V through 32 x 32 shared tiles;
// each panel's Gram matrix V_p^T V_p is accumulated over staged row tiles and
// turned into the panel's T factor (LAPACK dlarft, forward, columnwise).
template <class T>
__global__ void __launch_bounds__(256) k_spars_wb_rm(const SparsWBRM<T>* tasks, const SpBlock<T>* blocks) {
    pdl_enter();
    constexpr int P = kNB + 1;
    __shared__ T G[kNB * P];
    __shared__ T Ts[kNB * P];
    __shared__ T tile[32][33];
    __shared__ T s_tau[kNB];
    __shared__ int s_col[32];
    const SparsWBRM<T> t = tasks[blockIdx.x];
    const int r = t.r, m = t.m, ny = gridDim.y, y = blockIdx.y;
    const size_t ld = (size_t)t.ldc;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
    // 1. interface blocks
    for (int b = y; b < t.nblk; b += ny) {
        const SpBlock<T> B = blocks[t.blk0 + b];
        if (B.kind == 0) {  // column block A(n2, c): rows x r, element (i, j) = Crank(j, coff + i)
            for (int j = warp; j < r; j += nw) {
                T* dcol = B.p + (size_t)j * B.ld;
                const T* crow = t.C + (size_t)j * ld + B.coff;
                for (int i = lane; i < B.rows; i += 32) dcol[i] = (j <= t.pos[B.coff + i]) ? crow[i] : T(0);
            }
        } else {  // row block A(c, n1): r x cols, element (i, j) = Crank(i, coff + j)
            for (int j0 = 0; j0 < B.cols; j0 += 32) {
                for (int i0 = 0; i0 < r; i0 += 32) {
                    const int j = j0 + lane;
                    const int pc = j < B.cols ? t.pos[B.coff + j] : -1;
                    for (int ii = warp; ii < 32; ii += nw) {
                        const int i = i0 + ii;
                        tile[ii][lane] = (i < r && i <= pc) ? t.C[(size_t)i * ld + B.coff + j] : T(0);
                    }
                    __syncthreads();
                    for (int jj = warp; jj < 32; jj += nw) {
                        const int jc = j0 + jj, i = i0 + lane;
                        if (jc < B.cols && i < r) B.p[i + (size_t)jc * B.ld] = tile[lane][jj];
                    }
                    __syncthreads();
                }
            }
        }
    }
    // the compression of extra rows (sparsify_extra) keeps no reflectors
    if (t.V == nullptr) return;
    // 2. V(:, q) = column colat[q] of C (reflector below the diagonal), tau
    for (int q0 = y * 32; q0 < r; q0 += ny * 32) {
        if (tid < 32) s_col[tid] = (q0 + tid < r) ? t.colat[q0 + tid] : 0;
        __syncthreads();
        for (int i0 = 0; i0 < m; i0 += 32) {
            for (int ii = warp; ii < 32; ii += nw) {
                const int i = i0 + ii;
                tile[ii][lane] = (i < m && q0 + lane < r) ? t.C[(size_t)i * ld + s_col[lane]] : T(0);
            }
            __syncthreads();
            for (int qq = warp; qq < 32; qq += nw) {
                const int q = q0 + qq, i = i0 + lane;
                if (q < r && i < m) t.V[i + (size_t)q * m] = tile[lane][qq];
            }
            __syncthreads();
        }
    }
    if (y == 0)
        for (int q = tid; q < r; q += blockDim.x) t.tau[q] = t.tau_in[q];
    // 3. T factor of each 32-reflector panel
    const int gi = tid & 31, gj = tid >> 5;  // G rows gi, columns gj + 8k
    for (int pi = y; pi * kNB < r; pi += ny) {
        const int p0 = pi * kNB;
        const int w = min(kNB, r - p0);
        const int R = m - p0;
        if (tid < kNB) {
            s_col[tid] = t.colat[p0 + (tid < w ? tid : 0)];
            s_tau[tid] = tid < w ? t.tau_in[p0 + tid] : T(0);
        }
        __syncthreads();
        T acc[4] = {T(0), T(0), T(0), T(0)};
        for (int r0 = 0; r0 < R; r0 += 32) {
            for (int ii = warp; ii < 32; ii += nw) {
                const int rr = r0 + ii;  // row p0 + rr of the panel; v_q: 1 at rr == q, 0 above
                T v = T(0);
                if (rr < R && lane < w) v = rr > lane ? t.C[(size_t)(p0 + rr) * ld + s_col[lane]] : (rr == lane ? T(1) : T(0));
                tile[ii][lane] = v;
            }
            __syncthreads();
#pragma unroll 8
            for (int ii = 0; ii < 32; ++ii) {
                const T a = tile[ii][gi];
#pragma unroll
                for (int k = 0; k < 4; ++k) acc[k] += a * tile[ii][gj + 8 * k];
            }
            __syncthreads();
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) G[gi * P + gj + 8 * k] = acc[k];
        __syncthreads();
        if (warp == 0) {
            for (int j = 0; j < kNB; ++j) {
                if (j < w) {
                    const T tj = s_tau[j];
                    T tmp = T(0);
                    if (lane < j)
                        for (int l = lane; l < j; ++l) tmp += Ts[lane * P + l] * G[l * P + j];
                    if (lane < j) Ts[lane * P + j] = -tj * tmp;
                    if (lane == j) Ts[j * P + j] = tj;
                    if (lane > j) Ts[lane * P + j] = T(0);
                } else {
                    Ts[lane * P + j] = T(0);
                }
                __syncwarp();
            }
        }
        __syncthreads();
        T* Tout = t.tp + (size_t)pi * kNB * kNB;
        for (int e = tid; e < kNB * kNB; e += blockDim.x) Tout[e] = Ts[(e % kNB) * P + (e / kNB)];
        __syncthreads();
    }
}

}  // namespace

template <class T>
cudaError_t launch_rrqr_rm(const RRQRTaskRM<T>* tasks, const int* ids, int ntasks, int cluster, int max_m,
                           int max_n, cudaStream_t s) {
    if (ntasks <= 0) return cudaSuccess;
    // reflector + up to 16 row-chunk partials of the widest slab + per-column scales
    const size_t mpad = (size_t)((max_m + 7) & ~7);
    const size_t wp = (size_t)(((max_n + cluster - 1) / cluster + 127) & ~127);
    size_t smem_bytes = (mpad + 17 * wp) * sizeof(T);
    const size_t cap = 160 * 1024;
    if (smem_bytes > cap) smem_bytes = std::max(cap, (mpad + 2 * wp) * sizeof(T));
    if (smem_bytes > 200 * 1024) return cudaErrorInvalidValue;  // interface too wide for this launch shape
    once_per_device(reinterpret_cast<const void*>(&k_rrqr_rm<T>), [] {
        cudaFuncSetAttribute(k_rrqr_rm<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
        cudaFuncSetAttribute(k_rrqr_rm<T>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    });
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(ntasks * cluster), 1, 1);
    cfg.blockDim = dim3(kRRThreads, 1, 1);
    cfg.dynamicSmemBytes = smem_bytes;
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
    return cudaLaunchKernelEx(&cfg, k_rrqr_rm<T>, tasks, ids, smem_bytes);
}

template <class T>
void launch_spars_wb_rm(const SparsWBRM<T>* tasks, const SpBlock<T>* blocks, int ntasks, int parts, cudaStream_t s) {
    if (ntasks <= 0) return;
    const int ny = parts < 1 ? 1 : (parts > 32 ? 32 : parts);
    const cudaError_t e = launch_pdl(k_spars_wb_rm<T>, dim3(ntasks, ny), dim3(256), 0, s, 0, tasks, blocks);
    if (e != cudaSuccess) throw std::runtime_error(std::string("k_spars_wb_rm launch: ") + cudaGetErrorString(e));
}

template cudaError_t launch_rrqr_rm<double>(const RRQRTaskRM<double>*, const int*, int, int, int, int,
                                            cudaStream_t);
template cudaError_t launch_rrqr_rm<float>(const RRQRTaskRM<float>*, const int*, int, int, int, int, cudaStream_t);
template void launch_spars_wb_rm<double>(const SparsWBRM<double>*, const SpBlock<double>*, int, int,
                                          cudaStream_t);
template void launch_spars_wb_rm<float>(const SparsWBRM<float>*, const SpBlock<float>*, int, int, cudaStream_t);

}  // namespace spq
