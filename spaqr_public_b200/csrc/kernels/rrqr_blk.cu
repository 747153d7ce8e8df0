// Blocked truncated column-pivoted Householder QR of the sparsification
// matrices (sparsifyD, src/tree.cpp:1022-1049; dgeqp3 + choose_rank,
// src/util.cpp:466-477, 795-816), one thread-block cluster per interface.
//
// dgeqp3 factors in blocks of NB pivot steps (LAPACK dlaqps): inside a block
// only the pivot column and the pivot row of each step are brought up to date;
// the rest of the matrix waits for one rank-NB update at the end of the block,
// C(k:m, :) -= V_b F^T, with
//     V_b  the block's reflectors (m x NB),
//     F    (n x NB), F(c, j) = tau_j v_j^T C_j(:, c), C_j = C as left by reflectors < j,
// built column by column from the block-start matrix C_bs:
//     F(:, j) = tau_j (C_bs(k:m, :)^T v_j - F(:, 0:j) (V_b(k:m, 0:j)^T v_j)).
// A pivot step therefore reads C once (the product C_bs^T v_j) instead of
// twice plus a write (the reflector applied at once), which is what bounds
// the unblocked kernel on the many-interface levels.
//
// Layout as in the unblocked kernel: C (m x n) row-major with stride ldc, the
// columns split in contiguous 32-aligned slabs over the CTAs of the cluster;
// pivoting is kept as positions (pos / colat), so ties break on the current
// position exactly as LAPACK's swaps would. Each CTA keeps in shared memory
// the F rows of its slab (l-major: F(l, c) at l * Wp + c), its own copy of V_b
// (m x NB, row-major, rows padded to NB + 1), and the partial norms and
// positions of its slab's columns.
//
// Per pivot step k (block column jb), with ONE cluster barrier:
//   1. arg-max of the partial norms over the slab; the CTAs publish their
//      candidates in alternating slots, cluster barrier, each CTA reduces the
//      candidates through DSMEM;
//   2. every CTA brings the pivot column up to date (C_bs(k:m, pc) -
//      V_b F(pc, :)^T, reading F(pc, :) from the owner's shared memory) and,
//      in the same pass and one block reduction, its norm and V_b^T of it;
//      the reflector (dlarfg) is v = (1, scal x) and s_aux = V_b(k:m, 0:jb)^T v
//      follows from those sums: same inputs and arithmetic give bitwise the
//      same v in every CTA, so nothing is broadcast; the swap is applied to the
//      positions each CTA keeps;
//   3. every CTA forms F(jb, c) over its slab (one pass over C_bs(k+1:m, slab),
//      row chunks whose count depends only on m and k, so the result does not
//      depend on the cluster size), updates pivot row k of its columns and
//      downdates their norms; a norm whose downdate lost accuracy (dlaqps's
//      tol3z test) is recomputed at once from C_bs - V_b F^T of its column.
// At the end of a block (cluster barrier) the owners store R_kk and the
// reflector of each pivot in its column, and the rows below the block get
// C -= V_b F^T (active columns only; cluster barrier). The loop stops at the
// rank (|R_kk| < tol |R_00|); the rows of R above it are already final, so no
// trailing update follows the last block.
#include <cooperative_groups.h>

#include <algorithm>
#include <climits>

#include "kernels.hpp"
#include "pdl.cuh"
#include "rrqr_common.cuh"
#include "status.cuh"

namespace cg = cooperative_groups;

// Phase clocks of the pivot steps (built only with -DSPQ_RRQR_CLOCKS, as the
// separate library libspaqr_b200_rrqrclk.so): thread 0 of every CTA adds the
// clock64() span of each phase of each pivot step to a device counter.
#ifdef SPQ_RRQR_CLOCKS
__device__ unsigned long long g_rrqr_clocks[16];
#define SPQ_CLK(name) const long long name = clock64()
#define SPQ_CLK_ADD(slot, v) atomicAdd(&g_rrqr_clocks[slot], (unsigned long long)(v))
// Reads (and with reset != 0 zeroes) the 16 counters: slots 0-6 the phase
// spans (arg-max, cluster barrier, candidate reduction, pivot column and
// reflector, partial products, row update and norms, norm recomputation), 7 the
// block ends, 8 the CTA steps, 9 the CTA blocks.
extern "C" int spq_rrqr_phase_clocks(unsigned long long* out16, int reset) {
    if (cudaDeviceSynchronize() != cudaSuccess) return 1;
    if (cudaMemcpyFromSymbol(out16, g_rrqr_clocks, sizeof(unsigned long long) * 16) != cudaSuccess) return 1;
    if (reset) {
        const unsigned long long z[16] = {0};
        if (cudaMemcpyToSymbol(g_rrqr_clocks, z, sizeof(z)) != cudaSuccess) return 1;
    }
    return 0;
}
#else
#define SPQ_CLK(name)
#define SPQ_CLK_ADD(slot, v)
#endif

namespace spq {
namespace {

using namespace rrqr;

constexpr int kBT = 512;                    // threads per CTA
constexpr int kGMax = 8;                    // row chunks of the per-step product (fixed: cluster-independent)
constexpr int kBU = 4;                      // 16-byte column vectors per lane in the per-step product
constexpr int kTRows = 64;                  // rows of a trailing-update tile (16 row groups of 4)
constexpr size_t kBlkSmemCap = 216 * 1024;  // dynamic shared memory of one CTA (static use is ~3 KB)

// Pivot steps per block: 32 in FP32, 16 in FP64 (the F and V_b copies of a CTA
// stay within shared memory for slabs of a few hundred columns).
template <class T>
struct BlkNB {
    static constexpr int v = sizeof(T) == 4 ? 32 : 16;
};

// Shared-memory elements of one CTA for slab width Wp (a multiple of the
// vector tile 32 * VEC) and m rows: F, partials, the slab's norms and
// positions, reflector, V_b (rows padded).
template <class T>
__host__ __device__ constexpr size_t blk_smem_elems(int Wp, int m) {
    return (size_t)(BlkNB<T>::v + kGMax + 3) * Wp + (size_t)((m + 7) & ~7) * (BlkNB<T>::v + 2);
}

// Partial products of pivot step k (3a below): part[g * Wp + c] = sum over the
// rows of chunk g of C_bs(i, c) v(i), lanes owning KBU 16-byte column vectors.
template <class T, int KBU>
__device__ __forceinline__ void rrqr_partials(const T* C, size_t ld, int j0, int Wc, int Wp, int k, int m, int Gs,
                                              int Lr, const T* vsh, T* part, int warp, int nw, int lane) {
    constexpr int VEC = Vec<T>::n;
    using VT = typename Vec<T>::type;
    constexpr int kRowUnroll = sizeof(T) == 4 ? 4 : 2;
    const int nvt = (Wc + 32 * VEC - 1) / (32 * VEC);
    const int ntg = (nvt + KBU - 1) / KBU;
    for (int item = warp; item < Gs * ntg; item += nw) {
        const int g = item % Gs, tg = item / Gs;
        const int i0 = k + 1 + g * Lr, i1 = min(m, i0 + Lr);
        T sv[KBU][VEC];
        const T* cp[KBU];
#pragma unroll
        for (int u = 0; u < KBU; ++u) {
#pragma unroll
            for (int q = 0; q < VEC; ++q) sv[u][q] = T(0);
            const int jl = ((tg * KBU + u) * 32 + lane) * VEC;
            cp[u] = C + j0 + (jl < Wc ? jl : 0);  // past the slab: reads its first vector
        }
#pragma unroll kRowUnroll
        for (int i = i0; i < i1; ++i) {
            const T vi = vsh[i];
            VT x[KBU];
#pragma unroll
            for (int u = 0; u < KBU; ++u) x[u] = *reinterpret_cast<const VT*>(cp[u] + i * ld);
#pragma unroll
            for (int u = 0; u < KBU; ++u) {
                const T* xs = reinterpret_cast<const T*>(&x[u]);
#pragma unroll
                for (int q = 0; q < VEC; ++q) sv[u][q] += vi * xs[q];
            }
        }
#pragma unroll
        for (int u = 0; u < KBU; ++u) {
            const int jl = ((tg * KBU + u) * 32 + lane) * VEC;
            if (jl < Wp) {
#pragma unroll
                for (int q = 0; q < VEC; ++q) part[g * Wp + jl + q] = sv[u][q];
            }
        }
    }
}

template <class T>
__global__ void __launch_bounds__(kBT) k_rrqr_blk(const RRQRTaskRM<T>* tasks, const int* ids, int Wp, int mpad) {
    pdl_enter();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int VEC = Vec<T>::n;
    constexpr int kBNB = BlkNB<T>::v;
    constexpr int VP = kBNB + 1;  // padded V_b row: conflict-free row-parallel reads
    using VT = typename Vec<T>::type;
    T* F = reinterpret_cast<T*>(smem_raw);            // kBNB x Wp, l-major
    T* part = F + (size_t)kBNB * Wp;                  // kGMax x Wp: row-chunk partials of C_bs^T v
    T* vn1 = part + (size_t)kGMax * Wp;               // Wp: partial column norms of the slab
    T* vn2 = vn1 + Wp;                                // Wp: norms at their last recomputation
    int* pos = reinterpret_cast<int*>(vn2 + Wp);      // Wp: current position of each slab column
    T* vsh = vn2 + 2 * (size_t)Wp;                    // mpad: the current reflector (pos takes <= Wp elements)
    T* Vs = vsh + mpad;                               // mpad x VP: V_b(i, l) at i * VP + l
    __shared__ T red[32];
    __shared__ Cand<T> wcand[2][32];  // per-warp pivot candidates, alternating slots by step parity
    __shared__ int s_gp, s_gc;
    __shared__ T s_fp[kBNB];  // F(l, pivot column), zero for l >= jb
    __shared__ T s_alpha;
    __shared__ int s_c0, s_nflag;
    __shared__ T s_aux[kBNB];    // V_b(k:m, l)^T v for l < jb, zero after
    __shared__ int s_pcs[kBNB];  // pivot column of each step of the block
    __shared__ T s_betas[kBNB];  // R_kk of each step of the block
    __shared__ T s_wpart[(kBT / 32) * kBNB];

    cg::cluster_group cl = cg::this_cluster();
    const int CL = (int)cl.num_blocks();
    const int cr = (int)cl.block_rank();
    const RRQRTaskRM<T> t = tasks[ids[blockIdx.x / CL]];
    const int m = t.m, n = t.n;
    const size_t ld = (size_t)t.ldc;
    T* C = t.C;
    const int W = (((n + CL - 1) / CL) + 31) & ~31;
    const int j0 = min(n, cr * W), j1 = min(n, j0 + W);
    const int Wc = j1 - j0;
    const int tid = threadIdx.x, nth = blockDim.x, lane = tid & 31, warp = tid >> 5, nw = nth >> 5;

    for (int jl = tid; jl < Wc; jl += nth) {
        T s = T(0);
#pragma unroll 8
        for (int i = 0; i < m; ++i) {
            const T v = C[i * ld + j0 + jl];
            s += v * v;
        }
        const T nv = sqrt(s);
        vn1[jl] = nv;
        vn2[jl] = nv;
        pos[jl] = j0 + jl;
    }
    if (tid == 0) s_c0 = -1;
    __syncthreads();

    const int kmax = min(m, n);
    const double tol = t.tol;
    int rank = kmax;
    const int ksteps = (tol != 0.0 && tol >= 1.0) ? 0 : kmax;
    if (ksteps == 0) rank = 0;
    T r00 = T(0);
    bool done = false;
    int k = 0;
    while (k < ksteps && !done) {
        const int k0 = k;
        const int nbk = min(kBNB, ksteps - k0);
        // a block starts from zero F and V_b: entries past the current step are
        // exact zeros, so the products below run over all kBNB columns unmasked
        for (int e = tid; e < kBNB * Wp; e += nth) F[e] = T(0);
        for (int e = tid; e < m * VP; e += nth) Vs[e] = T(0);
        __syncthreads();
        int steps = 0;
        for (int jb = 0; jb < nbk; ++jb) {
            k = k0 + jb;
            SPQ_CLK(tq0);
            const int buf = k & 1;  // candidate slots alternate, so one cluster barrier per step suffices
            // 1. pivot: largest partial norm, ties to the smallest position; the
            //    column now at position k is noted for the swap (s_c0 is -1 here:
            //    set before the first step, reset by its reader at every step)
            T bv = T(-1);
            int bp = INT_MAX, bc = -1;
            for (int jl = tid; jl < Wc; jl += nth) {
                const int p = pos[jl];
                if (p < k) continue;
                if (p == k) s_c0 = j0 + jl;
                const T v = vn1[jl];
                if (better(v, p, bv, bp)) {
                    bv = v;
                    bp = p;
                    bc = j0 + jl;
                }
            }
            warp_best(bv, bp, bc);
            if (lane == 0) wcand[buf][warp] = Cand<T>{bv, bp, bc};
            SPQ_CLK(tq1);
            // the cluster barrier also orders this CTA's warps: every warp's candidate
            // of every CTA is visible to all after it
            cl.sync();
            SPQ_CLK(tq2);
            // every CTA reduces all warps' candidates of the cluster (candidate q: CTA
            // q / nw, warp q % nw, one 16-byte record; the order is immaterial,
            // (value, position) is a strict order), then warp 0 fetches F(:, pc) from
            // the pivot's owner
            if (warp == 0) {
                // all of a lane's candidate loads are issued before any is used,
                // so the DSMEM round trips overlap
                constexpr int kCand = (16 * (kBT / 32) + 31) / 32;  // <= 16 CTAs x warps per CTA, per lane
                constexpr int kBatch = 4;
                T v = T(-1);
                int p = INT_MAX, c = -1;
#pragma unroll
                for (int u0 = 0; u0 < kCand; u0 += kBatch) {
                    if (32 * u0 >= CL * nw) break;  // uniform over the warp: no candidate left
                    Cand<T> cq[kBatch];
#pragma unroll
                    for (int u = 0; u < kBatch; ++u) {
                        const int q = lane + 32 * (u0 + u);
                        const bool in = q < CL * nw;
                        const int rk = in ? q / nw : 0, wq = in ? q % nw : 0;
                        cq[u] = *cl.map_shared_rank(&wcand[buf][wq], rk);
                        if (!in) cq[u].c = -1;
                    }
#pragma unroll
                    for (int u = 0; u < kBatch; ++u)
                        if (cq[u].c >= 0 && better(cq[u].v, cq[u].p, v, p)) {
                            v = cq[u].v;
                            p = cq[u].p;
                            c = cq[u].c;
                        }
                }
                warp_best(v, p, c);
                if (c >= 0 && lane < kBNB) {
                    const int ow = c / W;
                    s_fp[lane] = *cl.map_shared_rank(&F[lane * Wp + (c - ow * W)], ow);
                }
                if (lane == 0) {
                    s_gp = p;
                    s_gc = c;
                }
            }
            __syncthreads();
            const int gp = s_gp, pc = s_gc;
            SPQ_CLK(tq3);
            if (pc < 0) {  // no finite partial norm left (NaN input): stop, uniformly over the cluster
                rank = k;
                done = true;
                if (cr == 0 && tid == 0) note_rrqr_nan(t.status);
                break;
            }
            // 2. every CTA brings the pivot column up to date (C_bs - V_b F(pc, :)^T, F
            //    from the owner's shared memory) and builds the same reflector: the
            //    same inputs and the same arithmetic give bitwise the same v in every
            //    CTA, so v needs no broadcast. The owner stores the column at the end
            //    of the block, once no CTA reads its block-start values any more.
            // One pass and one block reduction: the pivot column x (kept unscaled in
            //    vsh), its squared norm below row k and the sums V_b(k+1:m, l)^T x;
            //    after the reduction the reflector is v = (1, scal x(k+1:m)), so
            //    s_aux = V_b(k, :) + scal V_b(k+1:m, :)^T x, and the partial products
            //    of 3a run on x and are scaled in 3b.
            T acc = T(0);
            T sa[kBNB];
#pragma unroll
            for (int l = 0; l < kBNB; ++l) sa[l] = T(0);
            for (int i = k + tid; i < m; i += nth) {
                T x = C[i * ld + pc];
#pragma unroll
                for (int l = 0; l < kBNB; ++l) x -= Vs[i * VP + l] * s_fp[l];  // zero past jb
                vsh[i] = x;
                if (i == k) {
                    s_alpha = x;
                } else {
                    acc += x * x;
#pragma unroll
                    for (int l = 0; l < kBNB; ++l) sa[l] += Vs[i * VP + l] * x;  // columns >= jb are zero
                }
            }
            // warp transpose-sum: lane l (mod kBNB) ends with the warp's sum of sa[l]
#pragma unroll
            for (int sft = kBNB / 2; sft >= 1; sft >>= 1) {
                const bool upper = (lane & sft) != 0;
#pragma unroll
                for (int q = 0; q < sft; ++q) {
                    const T send = upper ? sa[q] : sa[q + sft];
                    const T keep = upper ? sa[q + sft] : sa[q];
                    sa[q] = keep + __shfl_xor_sync(0xffffffffu, send, sft);
                }
            }
            // with kBNB < 32, lanes l and l + kBNB hold halves of the same sum
            T part0 = sa[0];
            if (kBNB < 32) part0 += __shfl_xor_sync(0xffffffffu, part0, kBNB);
            acc = wsum(acc);
            if (lane < kBNB) s_wpart[warp * kBNB + lane] = part0;
            if (lane == 0) red[warp] = acc;
            __syncthreads();
            T xn2 = T(0);
            for (int q = 0; q < nw; ++q) xn2 += red[q];
            const T alpha = s_alpha;
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
            const T sc = tau != T(0) ? scal : T(1);  // v(k+1:m) = sc x(k+1:m)
            if (tid < kBNB) {
                T sacc = T(0);
                for (int q = 0; q < nw; ++q) sacc += s_wpart[q * kBNB + tid];
                s_aux[tid] = tid < jb ? Vs[k * VP + tid] + sc * sacc : T(0);
            }
            // V_b(:, jb) = v (read after the barriers that follow)
            for (int i = k + tid; i < m; i += nth) Vs[i * VP + jb] = i == k ? T(1) : sc * vsh[i];
            if (cr == 0 && tid == 0) note_rrqr_pivot(t.status, beta);
            if (tol != 0.0 && kmax > 1) {
                if (k == 0) {
                    r00 = fabs(beta);
                } else if (!((double)fabs(beta) / (double)r00 >= tol)) {
                    rank = k;
                    done = true;
                    break;  // uniform over the cluster: every CTA computed the same beta
                }
            }
            if (tid == 0) {
                s_pcs[jb] = pc;
                s_betas[jb] = beta;
                if (cr == 0) t.tau[k] = tau;
                // LAPACK's column swap, as positions of the slab's own columns
                if (s_c0 >= 0) pos[s_c0 - j0] = gp;
                if (pc >= j0 && pc < j1) pos[pc - j0] = k;
                s_c0 = -1;
            }
            steps = jb + 1;
            SPQ_CLK(tq4);
            // no barrier here: 3a reads only x (complete since the reduction
            // barrier) and C; the positions, s_aux, V_b(:, jb) and the partials are
            // read in 3b, after the barrier that closes 3a
            // 3a. partials of C_bs(k+1:m, slab)^T x (v / sc): lanes own 16-byte column vectors,
            //     the rows are cut in Gs chunks of about 16 rows taken by different
            //     warps; narrow slabs give each lane one vector (kBU = 1) so that more
            //     warps share the pass. Each column's chunk sum runs over its rows in
            //     order in one lane either way (bitwise the same), and Gs depends on
            //     (m, k) only, so the result does not depend on the cluster size.
            const int Gs = max(1, min(kGMax, (m - k - 1 + 15) / 16));
            const int Lr = (m - k - 1 + Gs - 1) / Gs;
            if (tau != T(0)) {
                const int nvt = (Wc + 32 * VEC - 1) / (32 * VEC);
                if (Gs * ((nvt + kBU - 1) / kBU) >= nw)
                    rrqr_partials<T, kBU>(C, ld, j0, Wc, Wp, k, m, Gs, Lr, vsh, part, warp, nw, lane);
                else
                    rrqr_partials<T, 1>(C, ld, j0, Wc, Wp, k, m, Gs, Lr, vsh, part, warp, nw, lane);
            }
            if (tid == 0) s_nflag = 0;
            __syncthreads();
            SPQ_CLK(tq5);
            // 3b. F(jb, c), pivot row k, partial norms
            T vk[kBNB];  // V_b(k, 0:jb], zero after
#pragma unroll
            for (int l = 0; l < kBNB; ++l) vk[l] = Vs[k * VP + l];
            for (int jl = tid; jl < Wc; jl += nth) {
                const int c = j0 + jl;
                if (c == pc || pos[jl] < k) continue;
                const T ck0 = C[k * ld + c];
                T upd = T(0);
                if constexpr (sizeof(T) == 4) {
                    // F(:, c) read once: F(jb, c) is still zero, and V_b(k, jb) = 1,
                    // so the update is the sum over l != jb plus the new entry (the
                    // same sum term by term, zeros included). FP64 reads F twice
                    // (its 16 entries in registers would spill).
                    T fr[kBNB];
#pragma unroll
                    for (int l = 0; l < kBNB; ++l) fr[l] = F[l * Wp + jl];
                    T fnew = T(0);
                    if (tau != T(0)) {
                        T g = T(0);
                        for (int q = 0; q < Gs; ++q) g += part[q * Wp + jl];
                        g = ck0 + sc * g;
                        T corr = T(0);
#pragma unroll
                        for (int l = 0; l < kBNB; ++l) corr += fr[l] * s_aux[l];
                        fnew = tau * (g - corr);
                        F[jb * Wp + jl] = fnew;
                    }
#pragma unroll
                    for (int l = 0; l < kBNB; ++l) upd += vk[l] * fr[l];
                    upd += fnew;
                } else {
                    if (tau != T(0)) {
                        T g = T(0);
                        for (int q = 0; q < Gs; ++q) g += part[q * Wp + jl];
                        g = ck0 + sc * g;
                        T corr = T(0);
#pragma unroll
                        for (int l = 0; l < kBNB; ++l) corr += F[l * Wp + jl] * s_aux[l];
                        F[jb * Wp + jl] = tau * (g - corr);
                    }
#pragma unroll
                    for (int l = 0; l < kBNB; ++l) upd += vk[l] * F[l * Wp + jl];
                }
                const T ck = ck0 - upd;
                C[k * ld + c] = ck;
                const T n1 = vn1[jl];
                if (n1 != T(0)) {
                    const T rk = fabs(ck) / n1;
                    T temp = T(1) - rk * rk;
                    temp = temp < T(0) ? T(0) : temp;
                    const T qq = n1 / vn2[jl];
                    const T temp2 = temp * qq * qq;
                    if (temp2 <= Tol3z<T>::v()) {
                        vn2[jl] = T(-1);  // recomputed below from the up-to-date column
                        atomicAdd(&s_nflag, 1);
                    } else {
                        vn1[jl] = n1 * (T)sqrt(temp);
                    }
                }
            }
            __syncthreads();
            SPQ_CLK(tq6);
            // 3c. norms whose downdate lost accuracy, from C_bs(k+1:m, c) - V_b F(:, c)^T
            //     (one warp per column)
            if (s_nflag > 0) {
                for (int jl = warp; jl < Wc; jl += nw) {
                    const int c = j0 + jl;
                    if (!(vn2[jl] < T(0)) || c == pc || pos[jl] < k) continue;
                    T fr[kBNB];
#pragma unroll
                    for (int l = 0; l < kBNB; ++l) fr[l] = F[l * Wp + jl];
                    T ss = T(0);
                    for (int i = k + 1 + lane; i < m; i += 32) {
                        T x = C[i * ld + c];
#pragma unroll
                        for (int l = 0; l < kBNB; ++l) x -= Vs[i * VP + l] * fr[l];
                        ss += x * x;
                    }
                    ss = wsum(ss);
                    if (lane == 0) {
                        const T nv = (k + 1 < m) ? (T)sqrt(ss) : T(0);
                        vn1[jl] = nv;
                        vn2[jl] = nv;
                    }
                }
                __syncthreads();
            }
#ifdef SPQ_RRQR_CLOCKS
            if (tid == 0) {
                SPQ_CLK(tq7);
                SPQ_CLK_ADD(0, tq1 - tq0);
                SPQ_CLK_ADD(1, tq2 - tq1);
                SPQ_CLK_ADD(2, tq3 - tq2);
                SPQ_CLK_ADD(3, tq4 - tq3);
                SPQ_CLK_ADD(4, tq5 - tq4);
                SPQ_CLK_ADD(5, tq6 - tq5);
                SPQ_CLK_ADD(6, tq7 - tq6);
                SPQ_CLK_ADD(8, 1);
            }
#endif
        }
        // every CTA is past its last read of this block's block-start pivot columns
        // and of the owners' F: the owners store R_kk and the reflector of each
        // accepted pivot in its column
        SPQ_CLK(tb0);
        cl.sync();
        for (int j = 0; j < steps; ++j) {
            const int pcj = s_pcs[j], kj = k0 + j;
            if (pcj < j0 || pcj >= j1) continue;
            for (int i = kj + tid; i < m; i += nth) C[i * ld + pcj] = i == kj ? s_betas[j] : Vs[i * VP + j];
        }
        if (done) break;
        k = k0 + steps;
        if (k >= ksteps) break;  // full rank reached: rows of R final, nothing below to update
        // 4. C(k:m, c) -= V_b(k:m, :) F(:, c) for the active columns of the slab: a thread
        //    owns 4 rows x one 16-byte column vector of each 64 x (32 VEC) tile
        const int rg = tid >> 5;  // 16 row groups of 4 rows
        for (int r0 = k; r0 < m; r0 += kTRows) {
            for (int c0 = 0; c0 < Wc; c0 += 32 * VEC) {
                const int cl0 = c0 + lane * VEC;
                if (cl0 >= Wc) continue;
                VT x[4];
#pragma unroll
                for (int r = 0; r < 4; ++r) {
                    const int i = min(r0 + rg * 4 + r, m - 1);
                    x[r] = *reinterpret_cast<const VT*>(C + i * ld + j0 + cl0);
                }
                T acc[4][VEC];
#pragma unroll
                for (int r = 0; r < 4; ++r)
#pragma unroll
                    for (int q = 0; q < VEC; ++q) acc[r][q] = T(0);
#pragma unroll 4
                for (int l = 0; l < kBNB; ++l) {
                    const VT b = *reinterpret_cast<const VT*>(F + l * Wp + cl0);
                    const T* bs = reinterpret_cast<const T*>(&b);
#pragma unroll
                    for (int r = 0; r < 4; ++r) {
                        const T a = Vs[min(r0 + rg * 4 + r, m - 1) * VP + l];
#pragma unroll
                        for (int q = 0; q < VEC; ++q) acc[r][q] += a * bs[q];
                    }
                }
                bool act[VEC];
                bool all = true;
#pragma unroll
                for (int q = 0; q < VEC; ++q) {
                    act[q] = cl0 + q < Wc && pos[cl0 + q] >= k;
                    all = all && act[q];
                }
#pragma unroll
                for (int r = 0; r < 4; ++r) {
                    const int i = r0 + rg * 4 + r;
                    if (i >= m) break;
                    T* xs = reinterpret_cast<T*>(&x[r]);
                    T* px = C + i * ld + j0 + cl0;
                    if (all) {
#pragma unroll
                        for (int q = 0; q < VEC; ++q) xs[q] -= acc[r][q];
                        *reinterpret_cast<VT*>(px) = x[r];
                    } else {
#pragma unroll
                        for (int q = 0; q < VEC; ++q)
                            if (act[q]) px[q] = xs[q] - acc[r][q];
                    }
                }
            }
        }
        // the next block's first pivot columns are read (global) by every CTA
        cl.sync();
#ifdef SPQ_RRQR_CLOCKS
        if (tid == 0) {
            SPQ_CLK(tb1);
            SPQ_CLK_ADD(7, tb1 - tb0);
            SPQ_CLK_ADD(9, 1);
        }
#endif
    }
    __syncthreads();
    // positions out: pos, and colat as their inverse (positions are a permutation)
    for (int jl = tid; jl < Wc; jl += nth) {
        const int p = pos[jl];
        t.pos[j0 + jl] = p;
        t.colat[p] = j0 + jl;
        t.vn1[j0 + jl] = vn1[jl];
        t.vn2[j0 + jl] = vn2[jl];
    }
    if (cr == 0 && tid == 0) *t.rank = rank;
}

}  // namespace

template <class T>
bool rrqr_blk_fits(int max_m, int max_n, int cluster) {
    constexpr int tile = 32 * Vec<T>::n;
    if (cluster < 1 || max_m < 1) return false;
    const int W = (((max_n + cluster - 1) / cluster) + 31) & ~31;
    const int Wp = (W + tile - 1) / tile * tile;
    return blk_smem_elems<T>(Wp, max_m) * sizeof(T) <= kBlkSmemCap;
}

template <class T>
cudaError_t launch_rrqr_blk(const RRQRTaskRM<T>* tasks, const int* ids, int ntasks, int cluster, int max_m,
                            int max_n, cudaStream_t s) {
    if (ntasks <= 0) return cudaSuccess;
    if (!rrqr_blk_fits<T>(max_m, max_n, cluster)) return cudaErrorInvalidValue;
    constexpr int tile = 32 * Vec<T>::n;
    const int W = (((max_n + cluster - 1) / cluster) + 31) & ~31;
    const int Wp = (W + tile - 1) / tile * tile;
    const int mpad = (max_m + 7) & ~7;
    const size_t smem_bytes = blk_smem_elems<T>(Wp, max_m) * sizeof(T);
    once_per_device(reinterpret_cast<const void*>(&k_rrqr_blk<T>), [] {
        cudaFuncSetAttribute(k_rrqr_blk<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kBlkSmemCap);
        cudaFuncSetAttribute(k_rrqr_blk<T>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    });
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(ntasks * cluster), 1, 1);
    cfg.blockDim = dim3(kBT, 1, 1);
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
    return cudaLaunchKernelEx(&cfg, k_rrqr_blk<T>, tasks, ids, Wp, mpad);
}

template bool rrqr_blk_fits<double>(int, int, int);
template bool rrqr_blk_fits<float>(int, int, int);
template cudaError_t launch_rrqr_blk<double>(const RRQRTaskRM<double>*, const int*, int, int, int, int,
                                             cudaStream_t);
template cudaError_t launch_rrqr_blk<float>(const RRQRTaskRM<float>*, const int*, int, int, int, int, cudaStream_t);

}  // namespace spq
