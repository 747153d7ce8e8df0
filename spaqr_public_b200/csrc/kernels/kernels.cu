// sm_100a kernels of the spaQR factorization (elimination, scaling,
// sparsification, merge) and of the solve sweeps and Krylov vector work.
//
// Layout: every dense block is column-major in HBM; a batched launch receives a
// device array of task descriptors and serves one descriptor per CTA (or one
// tile of a descriptor per CTA). Householder conventions follow LAPACK
// (dgeqrf/dlarfg/dlarft forward-columnwise, dgeqp3 with Drmac-Bujanovic norm
// downdating) so that ranks and reflectors agree with the reference's LAPACK
// calls up to rounding.
#include "kernels.hpp"
#include "pdl.cuh"
#include "status.cuh"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <mutex>
#include <set>
#include <stdexcept>
#include <string>
#include <utility>

namespace spq {

namespace {

constexpr int kThreads = 256;
constexpr int kRC = 64;  // row chunk of the trailing update

template <class T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Deterministic block sum; red must hold 32 elements of shared memory.
template <class T>
__device__ T block_sum(T v, T* red) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    v = warp_sum(v);
    __syncthreads();
    if (lane == 0) red[warp] = v;
    __syncthreads();
    if (warp == 0) {
        T r = lane < nw ? red[lane] : T(0);
        r = warp_sum(r);
        if (lane == 0) red[0] = r;
    }
    __syncthreads();
    return red[0];
}

template <class T>
__device__ __forceinline__ T dev_hypot(T a, T b);
template <>
__device__ __forceinline__ double dev_hypot<double>(double a, double b) { return hypot(a, b); }
template <>
__device__ __forceinline__ float dev_hypot<float>(float a, float b) { return hypotf(a, b); }

// Elementary reflector (LAPACK dlarfg): given alpha and the squared norm of
// the tail, returns tau, beta and the tail scale 1/(alpha - beta).
template <class T>
__device__ __forceinline__ void make_reflector(T alpha, T xn2, T& tau, T& beta, T& scal) {
    if (xn2 == T(0)) {
        tau = T(0);
        beta = alpha;
        scal = T(1);
    } else {
        T nrm = dev_hypot(alpha, (T)sqrt(xn2));
        beta = alpha >= T(0) ? -nrm : nrm;
        tau = (beta - alpha) / beta;
        scal = T(1) / (alpha - beta);
    }
}

// Triangular factor of one panel of unit-lower reflectors (LAPACK dlarft,
// forward, columnwise). Vp points at the panel's diagonal element (local row
// 0, column 0); R rows, w <= kNB columns. G and Ts are shared scratch of
// kNB x (kNB+1). Result written to Tout (kNB x kNB, column-major, zero padded).
template <class T>
__device__ void build_tfac(const T* Vp, int ldv, int R, int w, const T* taus, T* Tout, T* G, T* Ts) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    constexpr int P = kNB + 1;
    // G(i, j) = v_i^T v_j for i < j.
    int pair = 0;
    for (int j = 1; j < w; ++j) {
        for (int i = 0; i < j; ++i, ++pair) {
            if ((pair % nw) != warp) continue;
            T s = T(0);
            for (int r = j + 1 + lane; r < R; r += 32) s += Vp[r + (size_t)i * ldv] * Vp[r + (size_t)j * ldv];
            s = warp_sum(s);
            if (lane == 0) G[i * P + j] = s + (j < R ? Vp[j + (size_t)i * ldv] : T(0));
        }
    }
    __syncthreads();
    if (warp == 0) {
        for (int j = 0; j < kNB; ++j) {
            if (j < w) {
                T tj = taus[j];
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
    for (int e = threadIdx.x; e < kNB * kNB; e += blockDim.x) {
        int i = e % kNB, j = e / kNB;
        Tout[e] = Ts[i * P + j];
    }
    __syncthreads();
}

// ------------------------------------------------------------------ copies
// CTA (d, y) copies 32-column chunks y, y + gridDim.y, ... of descriptor d.
// Modes 0/1 (plain / identity): each warp owns columns of the chunk, lanes
// walk the rows (coalesced on both sides). Mode 2 (dst = src^T): 32 x 32
// tiles through shared memory, so reads run along src columns and writes
// along dst columns.
template <class T>
__global__ void __launch_bounds__(256) k_copy(const CopyDesc<T>* descs, int n) {
    pdl_enter();
    __shared__ T tile[32][33];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int d = blockIdx.x; d < n; d += gridDim.x) {
        const CopyDesc<T> c = descs[d];
        for (int j0 = blockIdx.y * 32; j0 < c.cols; j0 += gridDim.y * 32) {
            if (c.mode == 2) {
                for (int i0 = 0; i0 < c.rows; i0 += 32) {
                    const int i = i0 + lane;
#pragma unroll
                    for (int jj = warp; jj < 32; jj += 8) {
                        const int j = j0 + jj;
                        tile[jj][lane] = (i < c.rows && j < c.cols) ? c.src[i + (size_t)j * c.sld] : T(0);
                    }
                    __syncthreads();
                    const int j = j0 + lane;
#pragma unroll
                    for (int ii = warp; ii < 32; ii += 8) {
                        const int r = i0 + ii;
                        if (r < c.rows && j < c.cols) c.dst[j + (size_t)r * c.dld] = tile[lane][ii];
                    }
                    __syncthreads();
                }
                continue;
            }
            for (int jj = warp; jj < 32; jj += 8) {
                const int j = j0 + jj;
                if (j >= c.cols) break;
                T* dcol = c.dst + (size_t)j * c.dld;
                if (c.mode == 1) {
                    for (int i = lane; i < c.rows; i += 32) dcol[i] = (i == j) ? T(1) : T(0);
                } else if (!c.src) {
                    for (int i = lane; i < c.rows; i += 32) dcol[i] = T(0);
                } else {
                    const T* scol = c.src + (size_t)j * c.sld;
                    int i = lane;
                    for (; i + 96 < c.rows; i += 128) {
                        const T a = scol[i], b = scol[i + 32], e = scol[i + 64], f = scol[i + 96];
                        dcol[i] = a;
                        dcol[i + 32] = b;
                        dcol[i + 64] = e;
                        dcol[i + 96] = f;
                    }
                    for (; i < c.rows; i += 32) dcol[i] = scol[i];
                }
            }
        }
    }
}

// ------------------------------------------------------------------ panel QR
// One CTA factors one panel of <= kNB columns (rows p..m-1) of one task. Each
// column step is one row-parallel pass: every thread walks its rows and
// accumulates, in registers, the dot products of the new reflector with all
// other panel columns (coalesced loads, ~31 independent per row). The products
// with the later columns drive the rank-1 update; those with the earlier
// reflectors are the Gram entries v_i^T v_j of the panel's T factor (LAPACK
// dlarft, forward columnwise), so T needs no extra pass.
template <class T>
__global__ void __launch_bounds__(kThreads) k_panel(const QRTask<T>* tasks, const int* ids, int p, int smem_rows) {
    pdl_enter();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* sm = reinterpret_cast<T*>(smem_raw);
    __shared__ T red[32];
    __shared__ T s_tau[kNB];
    __shared__ T dots[kNB];
    __shared__ T wred[(kThreads / 32) * kNB];
    __shared__ T G[kNB * (kNB + 1)];
    __shared__ T Ts[kNB * (kNB + 1)];
    constexpr int GP = kNB + 1;
    const QRTask<T> t = tasks[ids[blockIdx.x]];
    const int m = t.m, k = t.k;
    if (p >= k) return;
    const int w = min(kNB, k - p);
    const int R = m - p;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
    T* gp = t.fac + p + (size_t)p * m;
    const bool in_smem = R <= smem_rows;
    T* P = in_smem ? sm : gp;
    const int ldp = in_smem ? R : m;
    if (in_smem) {
        for (int e = tid; e < R * w; e += blockDim.x) {
            const int i = e % R, j = e / R;
            P[i + j * ldp] = gp[i + (size_t)j * m];
        }
        __syncthreads();
    }
    for (int j = 0; j < w; ++j) {
        if (j >= R) {
            if (tid == 0) s_tau[j] = T(0);
            for (int c = tid; c < j; c += blockDim.x) G[c * GP + j] = T(0);
            continue;
        }
        T* pj = P + (size_t)j * ldp;
        T part = T(0);
        for (int i = j + 1 + tid; i < R; i += blockDim.x) part += pj[i] * pj[i];
        const T xn2 = block_sum(part, red);
        const T alpha = pj[j];
        T tau, beta, scal;
        make_reflector(alpha, xn2, tau, beta, scal);
        if (tau != T(0))
            for (int i = j + 1 + tid; i < R; i += blockDim.x) pj[i] *= scal;
        __syncthreads();
        if (tid == 0) {
            pj[j] = beta;
            s_tau[j] = tau;
            note_qr_pivot(t.status, beta);
        }
        // d[c] = P[j, c] + sum_{r > j} v_j[r] P[r, c] for every panel column c != j
        // (loads issued unconditionally from columns clamped to the panel, so
        // that a row's kNB loads are in flight together; masked by selects)
        const int wl = w - 1;
        T acc[kNB];
#pragma unroll
        for (int c = 0; c < kNB; ++c) acc[c] = T(0);
        for (int r = j + 1 + tid; r < R; r += blockDim.x) {
            const T vr = pj[r];
            T pv[kNB];
#pragma unroll
            for (int c = 0; c < kNB; ++c) pv[c] = P[r + (size_t)min(c, wl) * ldp];
#pragma unroll
            for (int c = 0; c < kNB; ++c) acc[c] += (c < w && c != j) ? vr * pv[c] : T(0);
        }
#pragma unroll
        for (int c = 0; c < kNB; ++c) {
            const T v = warp_sum(acc[c]);
            if (lane == c) wred[warp * kNB + c] = v;
        }
        __syncthreads();
        if (tid < w && tid != j) {
            T d = P[j + (size_t)tid * ldp];
            for (int q = 0; q < nw; ++q) d += wred[q * kNB + tid];
            dots[tid] = d;
            if (tid < j) G[tid * GP + j] = d;  // v_tid^T v_j
        }
        __syncthreads();
        if (tau != T(0)) {
            for (int r = j + 1 + tid; r < R; r += blockDim.x) {
                const T vr = pj[r];
                T pv[kNB];
#pragma unroll
                for (int c = 0; c < kNB; ++c) pv[c] = P[r + (size_t)min(c, wl) * ldp];
#pragma unroll
                for (int c = 0; c < kNB; ++c)
                    if (c > j && c < w) P[r + (size_t)c * ldp] = pv[c] - (tau * dots[c]) * vr;
            }
            if (tid > j && tid < w) P[j + (size_t)tid * ldp] -= tau * dots[tid];
        }
        __syncthreads();
    }
    for (int j = tid; j < w; j += blockDim.x) t.tau[p + j] = s_tau[j];
    // T factor from the Gram entries (warp 0): T(0:j, j) = -tau_j T(0:j, 0:j) G(0:j, j)
    if (warp == 0) {
        for (int j = 0; j < kNB; ++j) {
            if (j < w) {
                const T tj = s_tau[j];
                T tmp = T(0);
                if (lane < j)
                    for (int l = lane; l < j; ++l) tmp += Ts[lane * GP + l] * G[l * GP + j];
                if (lane < j) Ts[lane * GP + j] = -tj * tmp;
                if (lane == j) Ts[j * GP + j] = tj;
                if (lane > j) Ts[lane * GP + j] = T(0);
            } else {
                Ts[lane * GP + j] = T(0);
            }
            __syncwarp();
        }
    }
    __syncthreads();
    T* Tout = t.tp + (size_t)(p / kNB) * kNB * kNB;
    for (int e = tid; e < kNB * kNB; e += blockDim.x) Tout[e] = Ts[(e % kNB) * GP + (e / kNB)];
    if (in_smem) {
        for (int e = tid; e < R * w; e += blockDim.x) {
            const int i = e % R, j = e / R;
            gp[i + (size_t)j * m] = P[i + j * ldp];
        }
    }
}

// ------------------------------------------------------------------ trailing update on tensor cores
// The same C <- C - V (T^T (V^T C)) on one tile of kTN columns, with both
// products on the tensor pipe (warp-level mma.sync):
//   FP32: 3xTF32 (each operand split into a TF32 head and a TF32 tail,
//         hi*hi + hi*lo + lo*hi accumulated in FP32: FP32-level accuracy);
//   FP64: DMMA m8n8k4 (IEEE FP64 products and sums).
// Rows are staged in kRC-row chunks, column-major in shared memory (stride
// kTCS: the fragment loads of both products and the coalesced staging and
// write-back hit distinct banks). Y^T = C^T V: every warp owns fixed output
// tiles and sums its tiles over all rows in order (no cross-warp reduction,
// deterministic). Z = T^T Y on SIMT. C -= V Z per chunk: every warp owns
// fixed tiles of the chunk, subtracted from the staged C, written back.
constexpr int kTCS = kRC + 4;  // 68: column stride of the staged chunk (elements)

__device__ __forceinline__ uint32_t to_tf32(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;\n" : "=r"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ void split_tf32(float x, uint32_t& hi, uint32_t& lo) {
    hi = to_tf32(x);
    lo = to_tf32(x - __uint_as_float(hi));
}
__device__ __forceinline__ void mma_tf32(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}
// acc += A B in 3xTF32: the two small cross terms first, then the head product
__device__ __forceinline__ void mma_3xtf32(float (&d)[4], const uint32_t (&ah)[4], const uint32_t (&al)[4],
                                           uint32_t bh0, uint32_t bh1, uint32_t bl0, uint32_t bl1) {
    mma_tf32(d, al, bh0, bh1);
    mma_tf32(d, ah, bl0, bl1);
    mma_tf32(d, ah, bh0, bh1);
}
__device__ __forceinline__ void mma_f64(double (&d)[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(d[0]), "+d"(d[1])
                 : "d"(a), "d"(b));
}

// Y^T(j, i) = sum over the chunk's rows r of C(r, j) V(r, i), accumulated into
// the warp's tiles. Cs, Vs: column-major chunk (stride kTCS).
// FP32: warp w owns the 16 x 8 tile (j0 = 16 (w >> 2), i0 = 8 (w & 3)).
__device__ __forceinline__ void tc_yt_chunk(float (&acc)[4], const float* Cs, const float* Vs, int warp, int lane) {
    const int g = lane >> 2, t = lane & 3;
    const int j0 = 16 * (warp >> 2), i0 = 8 * (warp & 3);
#pragma unroll 2
    for (int k0 = 0; k0 < kRC; k0 += 8) {
        uint32_t ah[4], al[4], bh0, bl0, bh1, bl1;
        split_tf32(Cs[(j0 + g) * kTCS + k0 + t], ah[0], al[0]);
        split_tf32(Cs[(j0 + g + 8) * kTCS + k0 + t], ah[1], al[1]);
        split_tf32(Cs[(j0 + g) * kTCS + k0 + t + 4], ah[2], al[2]);
        split_tf32(Cs[(j0 + g + 8) * kTCS + k0 + t + 4], ah[3], al[3]);
        split_tf32(Vs[(i0 + g) * kTCS + k0 + t], bh0, bl0);
        split_tf32(Vs[(i0 + g) * kTCS + k0 + t + 4], bh1, bl1);
        mma_3xtf32(acc, ah, al, bh0, bh1, bl0, bl1);
    }
}
// FP64: warp w owns the two 8 x 8 tiles (j0 = 8 (w >> 1), i0 = 16 (w & 1) + {0, 8}).
__device__ __forceinline__ void tc_yt_chunk(double (&acc)[4], const double* Cs, const double* Vs, int warp,
                                            int lane) {
    const int g = lane >> 2, t = lane & 3;
    const int j0 = 8 * (warp >> 1), i0 = 16 * (warp & 1);
    double d0[2] = {acc[0], acc[1]}, d1[2] = {acc[2], acc[3]};
#pragma unroll 4
    for (int k0 = 0; k0 < kRC; k0 += 4) {
        const double a = Cs[(j0 + g) * kTCS + k0 + t];
        mma_f64(d0, a, Vs[(i0 + g) * kTCS + k0 + t]);
        mma_f64(d1, a, Vs[(i0 + 8 + g) * kTCS + k0 + t]);
    }
    acc[0] = d0[0];
    acc[1] = d0[1];
    acc[2] = d1[0];
    acc[3] = d1[1];
}
// The warp's accumulated Y^T tiles into Ys as Y(i, j) = Ys[i * (kTN + 1) + j].
__device__ __forceinline__ void tc_yt_store(const float (&acc)[4], float* Ys, int warp, int lane) {
    constexpr int CP = kTN + 1;
    const int g = lane >> 2, t = lane & 3;
    const int j0 = 16 * (warp >> 2), i0 = 8 * (warp & 3);
    Ys[(i0 + 2 * t) * CP + j0 + g] = acc[0];
    Ys[(i0 + 2 * t + 1) * CP + j0 + g] = acc[1];
    Ys[(i0 + 2 * t) * CP + j0 + g + 8] = acc[2];
    Ys[(i0 + 2 * t + 1) * CP + j0 + g + 8] = acc[3];
}
__device__ __forceinline__ void tc_yt_store(const double (&acc)[4], double* Ys, int warp, int lane) {
    constexpr int CP = kTN + 1;
    const int g = lane >> 2, t = lane & 3;
    const int j0 = 8 * (warp >> 1), i0 = 16 * (warp & 1);
    Ys[(i0 + 2 * t) * CP + j0 + g] = acc[0];
    Ys[(i0 + 2 * t + 1) * CP + j0 + g] = acc[1];
    Ys[(i0 + 8 + 2 * t) * CP + j0 + g] = acc[2];
    Ys[(i0 + 8 + 2 * t + 1) * CP + j0 + g] = acc[3];
}

// Z operand fragments of C -= V Z, kept in registers across the chunks.
// FP32: warp w owns rows m0 = 16 (w >> 1) of the chunk and columns
// n0 = 16 (w & 1) + {0, 8}; zf[nt][ks][0..3] = {hi(k0+t), hi(k0+t+4), lo(k0+t), lo(k0+t+4)}.
struct ZFragF32 {
    uint32_t z[2][4][4];
};
__device__ __forceinline__ void tc_z_load(ZFragF32& f, const float* Zs, int warp, int lane) {
    constexpr int CP = kTN + 1;
    const int g = lane >> 2, t = lane & 3;
    const int n0 = 16 * (warp & 1);
#pragma unroll
    for (int nt = 0; nt < 2; ++nt)
#pragma unroll
        for (int ks = 0; ks < 4; ++ks) {
            const int c = n0 + 8 * nt + g, k0 = 8 * ks;
            split_tf32(Zs[(k0 + t) * CP + c], f.z[nt][ks][0], f.z[nt][ks][2]);
            split_tf32(Zs[(k0 + t + 4) * CP + c], f.z[nt][ks][1], f.z[nt][ks][3]);
        }
}
// Cs(r, c) -= (V Z)(r, c) over the chunk (Vs, Cs column-major, stride kTCS).
__device__ __forceinline__ void tc_cvz_chunk(float* Cs, const float* Vs, const ZFragF32& f, const float*, int warp,
                                             int lane) {
    const int g = lane >> 2, t = lane & 3;
    const int m0 = 16 * (warp >> 1), n0 = 16 * (warp & 1);
    float d[2][4] = {};
#pragma unroll
    for (int ks = 0; ks < 4; ++ks) {
        const int k0 = 8 * ks;
        uint32_t ah[4], al[4];
        split_tf32(Vs[(k0 + t) * kTCS + m0 + g], ah[0], al[0]);
        split_tf32(Vs[(k0 + t) * kTCS + m0 + g + 8], ah[1], al[1]);
        split_tf32(Vs[(k0 + t + 4) * kTCS + m0 + g], ah[2], al[2]);
        split_tf32(Vs[(k0 + t + 4) * kTCS + m0 + g + 8], ah[3], al[3]);
#pragma unroll
        for (int nt = 0; nt < 2; ++nt)
            mma_3xtf32(d[nt], ah, al, f.z[nt][ks][0], f.z[nt][ks][1], f.z[nt][ks][2], f.z[nt][ks][3]);
    }
#pragma unroll
    for (int nt = 0; nt < 2; ++nt) {
        const int c = n0 + 8 * nt + 2 * t;
        Cs[c * kTCS + m0 + g] -= d[nt][0];
        Cs[(c + 1) * kTCS + m0 + g] -= d[nt][1];
        Cs[c * kTCS + m0 + g + 8] -= d[nt][2];
        Cs[(c + 1) * kTCS + m0 + g + 8] -= d[nt][3];
    }
}
struct ZFragF64 {};
__device__ __forceinline__ void tc_z_load(ZFragF64&, const double*, int, int) {}
// FP64: warp w owns rows m0 = 8 w of the chunk and all four 8-column tiles;
// the Z fragments are read from shared memory (Zs = Y(i, j) layout).
__device__ __forceinline__ void tc_cvz_chunk(double* Cs, const double* Vs, const ZFragF64&, const double* Zs,
                                             int warp, int lane) {
    constexpr int CP = kTN + 1;
    const int g = lane >> 2, t = lane & 3;
    const int m0 = 8 * warp;
    double d[4][2] = {};
#pragma unroll
    for (int k0 = 0; k0 < kNB; k0 += 4) {
        const double a = Vs[(k0 + t) * kTCS + m0 + g];
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) mma_f64(d[nt], a, Zs[(k0 + t) * CP + 8 * nt + g]);
    }
#pragma unroll
    for (int nt = 0; nt < 4; ++nt) {
        const int c = 8 * nt + 2 * t;
        Cs[c * kTCS + m0 + g] -= d[nt][0];
        Cs[(c + 1) * kTCS + m0 + g] -= d[nt][1];
    }
}

template <class T>
struct TcTraits;
template <>
struct TcTraits<float> {
    using ZF = ZFragF32;
};
template <>
struct TcTraits<double> {
    using ZF = ZFragF64;
};

template <class T>
__global__ void __launch_bounds__(kThreads) k_trailing_tc(const QRTask<T>* tasks, const TileRef* tiles, int p) {
    pdl_enter();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int CP = kTN + 1, TP = kNB + 1;
    constexpr int EPT = kRC * kNB / kThreads;  // 8 elements per thread per chunk (V and C each)
    T* Vs = reinterpret_cast<T*>(smem_raw);  // kNB columns x kTCS, column-major
    T* Cs = Vs + kNB * kTCS;                  // kTN columns x kTCS
    T* Ys = Cs + kTN * kTCS;                  // kNB x CP: Y, then Z
    T* Tsh = Ys + kNB * CP;                   // kNB x TP
    __shared__ T* colp[kTN];
    const TileRef tr = tiles[blockIdx.x];
    const QRTask<T> t = tasks[tr.task];
    const int m = t.m, k = t.k;
    const int w = min(kNB, k - p);
    const int R = m - p;
    const int nf = t.tr_only ? 0 : k - p - w;
    const int ntot = nf + t.ntr;
    const int c0 = tr.tile * kTN;
    const int tn = min(kTN, ntot - c0);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (tid < kTN) {
        int vc = c0 + tid;
        T* ptr = nullptr;
        if (tid < tn) ptr = vc < nf ? t.fac + (size_t)(p + w + vc) * m : t.tr + (size_t)(vc - nf) * m;
        colp[tid] = ptr;
    }
    const T* V0 = t.fac + (size_t)p * m;
    for (int e = tid; e < kNB * kNB; e += blockDim.x) {
        int i = e % kNB, j = e / kNB;
        Tsh[i * TP + j] = (i < w && j < w) ? t.tp[(size_t)(p / kNB) * kNB * kNB + e] : T(0);
    }
    __syncthreads();
    T vr[EPT], cr[EPT];
    // element u of thread tid: row r = e % kRC, column q = e / kRC (coalesced along rows)
    auto fetch = [&](int r0) {
        const int rc = min(kRC, R - r0);
#pragma unroll
        for (int u = 0; u < EPT; ++u) {
            const int e = tid + u * kThreads;
            const int r = e % kRC, q = e / kRC;
            const int gr = r0 + r;
            const T x = V0[p + min(gr, R - 1) + (size_t)min(q, w - 1) * m];
            vr[u] = (r < rc && q < w) ? (gr < q ? T(0) : (gr == q ? T(1) : x)) : T(0);
            const T y = colp[min(q, tn - 1)][p + r0 + min(r, rc - 1)];
            cr[u] = (r < rc && q < tn) ? y : T(0);
        }
    };
    auto stash = [&]() {
#pragma unroll
        for (int u = 0; u < EPT; ++u) {
            const int e = tid + u * kThreads;
            const int r = e % kRC, q = e / kRC;
            Vs[q * kTCS + r] = vr[u];
            Cs[q * kTCS + r] = cr[u];
        }
    };
    // Y^T = C^T V over all rows
    T acc[4] = {T(0), T(0), T(0), T(0)};
    fetch(0);
    for (int r0 = 0; r0 < R; r0 += kRC) {
        stash();
        __syncthreads();
        if (r0 + kRC < R) fetch(r0 + kRC);
        tc_yt_chunk(acc, Cs, Vs, warp, lane);
        __syncthreads();
    }
    tc_yt_store(acc, Ys, warp, lane);
    __syncthreads();
    // Z = T^T Y (SIMT, 32 x 32 x 32)
    {
        const int c = tid % kTN, jq = tid / kTN;
        constexpr int QPT = kNB / (kThreads / kTN);
        T z[QPT];
#pragma unroll
        for (int u = 0; u < QPT; ++u) {
            const int i = jq * QPT + u;
            T s = T(0);
            for (int l = 0; l <= i; ++l) s += Tsh[l * TP + i] * Ys[l * CP + c];
            z[u] = s;
        }
        __syncthreads();
#pragma unroll
        for (int u = 0; u < QPT; ++u) Ys[(jq * QPT + u) * CP + c] = z[u];
        __syncthreads();
    }
    typename TcTraits<T>::ZF zf;
    tc_z_load(zf, Ys, warp, lane);
    // C -= V Z chunk by chunk, written back after each chunk
    fetch(0);
    for (int r0 = 0; r0 < R; r0 += kRC) {
        const int rc = min(kRC, R - r0);
        stash();
        __syncthreads();
        if (r0 + kRC < R) fetch(r0 + kRC);
        tc_cvz_chunk(Cs, Vs, zf, Ys, warp, lane);
        __syncthreads();
        for (int e = tid; e < kRC * kTN; e += blockDim.x) {
            const int r = e % kRC, cc = e / kRC;
            if (r < rc && cc < tn) colp[cc][p + r0 + r] = Cs[cc * kTCS + r];
        }
        __syncthreads();
    }
}

// One element global -> shared without registers; src_ok false writes zero.
template <class T>
__device__ __forceinline__ void cp_async_el(T* dst, const T* src, bool src_ok) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;\n" ::"r"(d), "l"(src), "n"(sizeof(T)),
                 "r"(src_ok ? (int)sizeof(T) : 0)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// ------------------------------------------------------------------ TRSM on tensor cores
// X(rows x k) <- X R^-1 (R upper k x k) on 128-row tiles, blocked by 32
// columns: for block J, S = X(:, 0:J) R(0:J, J) on the tensor pipe (3xTF32 /
// DMMA mma.sync, the finished blocks of X staged 32 columns at a time), then
// each thread solves its row of (X(:, J) - S) against the 32 x 32 diagonal
// block of R and stores it (the next blocks read it back).
constexpr int kTrXS = 136;  // column stride of the staged X chunk (128 rows + pad)
// Stages of the chunk pipeline: 3 in FP32 (89 KB of shared memory with S and the
// diagonal block), 2 in FP64 (111 KB): two CTAs per SM either way.
template <class T>
struct TrsmStages {
    static constexpr int v = sizeof(T) == 4 ? 3 : 2;
};
constexpr int kTrRS = 40;   // row stride of the staged R chunk (32 columns + pad)

// S(32 rows of the warp, 32 columns) += Xc(:, 0:32) Rc(0:32, :)
__device__ __forceinline__ void trsm_mma_chunk(float (&acc)[2][4][4], const float* Xs, const float* Rs, int warp,
                                               int lane) {
    const int g = lane >> 2, t = lane & 3;
    const int r0 = 32 * warp;
#pragma unroll
    for (int k0 = 0; k0 < 32; k0 += 8) {
        uint32_t ah[2][4], al[2][4];
#pragma unroll
        for (int mt = 0; mt < 2; ++mt) {
            const int r = r0 + 16 * mt + g;
            split_tf32(Xs[(k0 + t) * kTrXS + r], ah[mt][0], al[mt][0]);
            split_tf32(Xs[(k0 + t) * kTrXS + r + 8], ah[mt][1], al[mt][1]);
            split_tf32(Xs[(k0 + t + 4) * kTrXS + r], ah[mt][2], al[mt][2]);
            split_tf32(Xs[(k0 + t + 4) * kTrXS + r + 8], ah[mt][3], al[mt][3]);
        }
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) {
            uint32_t bh0, bl0, bh1, bl1;
            split_tf32(Rs[(k0 + t) * kTrRS + 8 * nt + g], bh0, bl0);
            split_tf32(Rs[(k0 + t + 4) * kTrRS + 8 * nt + g], bh1, bl1);
#pragma unroll
            for (int mt = 0; mt < 2; ++mt) mma_3xtf32(acc[mt][nt], ah[mt], al[mt], bh0, bh1, bl0, bl1);
        }
    }
}
__device__ __forceinline__ void trsm_mma_store(const float (&acc)[2][4][4], float* Ss, int warp, int lane) {
    const int g = lane >> 2, t = lane & 3;
#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) {
            const int r = 32 * warp + 16 * mt + g, c = 8 * nt + 2 * t;
            Ss[r * (kNB + 1) + c] = acc[mt][nt][0];
            Ss[r * (kNB + 1) + c + 1] = acc[mt][nt][1];
            Ss[(r + 8) * (kNB + 1) + c] = acc[mt][nt][2];
            Ss[(r + 8) * (kNB + 1) + c + 1] = acc[mt][nt][3];
        }
}
// FP64: 4 x 4 tiles of 8 x 8 per warp (acc[mt][nt][2] viewed through the same shape)
__device__ __forceinline__ void trsm_mma_chunk(double (&acc)[2][4][4], const double* Xs, const double* Rs, int warp,
                                               int lane) {
    const int g = lane >> 2, t = lane & 3;
    const int r0 = 32 * warp;
#pragma unroll
    for (int k0 = 0; k0 < 32; k0 += 4) {
        double a[4], b[4];
#pragma unroll
        for (int mt = 0; mt < 4; ++mt) a[mt] = Xs[(k0 + t) * kTrXS + r0 + 8 * mt + g];
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) b[nt] = Rs[(k0 + t) * kTrRS + 8 * nt + g];
#pragma unroll
        for (int mt = 0; mt < 4; ++mt)
#pragma unroll
            for (int nt = 0; nt < 4; ++nt) {
                double* d = &acc[mt >> 1][nt][2 * (mt & 1)];
                double dd[2] = {d[0], d[1]};
                mma_f64(dd, a[mt], b[nt]);
                d[0] = dd[0];
                d[1] = dd[1];
            }
    }
}
__device__ __forceinline__ void trsm_mma_store(const double (&acc)[2][4][4], double* Ss, int warp, int lane) {
    const int g = lane >> 2, t = lane & 3;
#pragma unroll
    for (int mt = 0; mt < 4; ++mt)
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) {
            const int r = 32 * warp + 8 * mt + g, c = 8 * nt + 2 * t;
            const double* d = &acc[mt >> 1][nt][2 * (mt & 1)];
            Ss[r * (kNB + 1) + c] = d[0];
            Ss[r * (kNB + 1) + c + 1] = d[1];
        }
}

template <class T>
size_t trsm_tc_smem() {
    return sizeof(T) * ((size_t)TrsmStages<T>::v * (kNB * kTrXS + kNB * kTrRS) + (size_t)128 * (kNB + 1) +
                        (size_t)kNB * (kNB + 1));
}

template <class T>
__global__ void __launch_bounds__(128) k_trsm_tc(const TrsmTask<T>* tasks, const TileRef* tiles) {
    pdl_enter();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int S = TrsmStages<T>::v;
    constexpr int STG = kNB * kTrXS + kNB * kTrRS;  // one stage: X chunk, then R chunk
    T* stg = reinterpret_cast<T*>(smem_raw);       // S stages
    T* Ss = stg + S * STG;                          // 128 x (kNB + 1): S, row-major
    T* Rd = Ss + 128 * (kNB + 1);                   // kNB x (kNB + 1): diagonal block
    const TileRef tr = tiles[blockIdx.x];
    const TrsmTask<T> t = tasks[tr.task];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int row = tr.tile * 128 + tid;
    const bool active = row < t.rows;
    const int rclamp = min(row, t.rows - 1);
    for (int J0 = 0; J0 < t.k; J0 += kNB) {
        const int wj = min(kNB, t.k - J0);
        T acc[2][4][4];
#pragma unroll
        for (int a = 0; a < 2; ++a)
#pragma unroll
            for (int b = 0; b < 4; ++b)
#pragma unroll
                for (int c = 0; c < 4; ++c) acc[a][b][c] = T(0);
        // chunks i0 = 32 ch < J0 (every chunk full), S - 1 in flight: X(tile
        // rows, i0:i0+32) with thread = row (coalesced along rows; this thread
        // wrote those entries itself), R(i0:i0+32, J0:J0+wj), zero-filled past
        const int nch = J0 / kNB;
        auto issue = [&](int ch) {
            if (ch < nch) {
                T* Xs = stg + (ch % S) * STG;
                T* Rs = Xs + kNB * kTrXS;
                const int i0 = ch * kNB;
#pragma unroll 8
                for (int c = 0; c < kNB; ++c)
                    cp_async_el(Xs + c * kTrXS + tid, t.X + rclamp + (size_t)(i0 + c) * t.ldx, active);
                for (int e = tid; e < kNB * kNB; e += 128) {
                    const int i = e % kNB, jj = e / kNB;
                    cp_async_el(Rs + i * kTrRS + jj, t.R + (i0 + i) + (size_t)(J0 + min(jj, wj - 1)) * t.ldr,
                                jj < wj);
                }
            }
            cp_async_commit();
        };
#pragma unroll
        for (int ch = 0; ch < S - 1; ++ch) issue(ch);
        for (int ch = 0; ch < nch; ++ch) {
            cp_async_wait<S - 2>();
            __syncthreads();  // chunk ch landed for every thread; stage (ch - 1) % S is free
            issue(ch + S - 1);
            const T* Xs = stg + (ch % S) * STG;
            trsm_mma_chunk(acc, Xs, Xs + kNB * kTrXS, warp, lane);
        }
        cp_async_wait<0>();
        __syncthreads();
        trsm_mma_store(acc, Ss, warp, lane);
        for (int e = tid; e < kNB * kNB; e += 128) {
            const int i = e % kNB, jj = e / kNB;
            Rd[i * (kNB + 1) + jj] = (i < wj && jj < wj) ? t.R[(J0 + i) + (size_t)(J0 + jj) * t.ldr] : T(1);
        }
        __syncthreads();
        T x[kNB];
#pragma unroll
        for (int jj = 0; jj < kNB; ++jj)
            x[jj] = (jj < wj ? t.X[rclamp + (size_t)(J0 + min(jj, wj - 1)) * t.ldx] : T(0)) - Ss[tid * (kNB + 1) + jj];
#pragma unroll
        for (int jj = 0; jj < kNB; ++jj) {
            x[jj] = x[jj] / Rd[jj * (kNB + 1) + jj];
#pragma unroll
            for (int ll = jj + 1; ll < kNB; ++ll) x[ll] -= x[jj] * Rd[jj * (kNB + 1) + ll];
        }
        if (active) {
#pragma unroll
            for (int jj = 0; jj < kNB; ++jj)
                if (jj < wj) t.X[row + (size_t)(J0 + jj) * t.ldx] = x[jj];
        }
        __syncthreads();
    }
}

// X(i, i) = 1 for i < k of every task (X zeroed before): the identity that the
// TRSM turns into R^-1.
template <class T>
__global__ void k_unit_diag(const TrsmTask<T>* tasks) {
    pdl_enter();
    const TrsmTask<T> t = tasks[blockIdx.x];
    for (int i = threadIdx.x; i < t.k; i += blockDim.x) t.X[i + (size_t)i * t.ldx] = T(1);
}

// One CTA per fill candidate: the squared entries of A1^T A2 (each entry a
// dot product over the rows), summed over the CTA, square-rooted.
template <class T>
__global__ void __launch_bounds__(256) k_product_norm(const ProdNormTask<T>* tasks, double* out) {
    pdl_enter();
    __shared__ double red[32];
    const ProdNormTask<T> t = tasks[blockIdx.x];
    double s = 0.0;
    const int pairs = t.c1 * t.c2;
    for (int q = threadIdx.x; q < pairs; q += blockDim.x) {
        const int a = q % t.c1, b = q / t.c1;
        const T* x = t.a1 + (size_t)a * t.ld1;
        const T* y = t.a2 + (size_t)b * t.ld2;
        double dot = 0.0;
        for (int r = 0; r < t.rows; ++r) dot += (double)x[r] * (double)y[r];
        s += dot * dot;
    }
    s = block_sum(s, red);
    if (threadIdx.x == 0) out[blockIdx.x] = sqrt(s);
}

// ------------------------------------------------------------------ --scale 0 helpers
// One-sided (Hestenes) Jacobi on the columns of a copy W of R: round-robin
// pairs (i, j), one pair per warp at a time, rotated until every pair is
// orthogonal to working precision (or 30 sweeps); the singular values are then
// the column norms. Writes 1 / sigma_min (sum of squares in FP64).
template <class T>
__global__ void __launch_bounds__(256) k_sigma_min(const SigmaTask<T>* tasks) {
    pdl_enter();
    __shared__ double red[32];
    __shared__ int s_rot;
    const SigmaTask<T> t = tasks[blockIdx.x];
    const int n = t.n, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
    T* W = t.work;
    for (int e = tid; e < n * n; e += blockDim.x) {
        const int i = e % n, j = e / n;
        W[e] = i <= j ? t.R[i + (size_t)j * t.ld] : T(0);
    }
    __syncthreads();
    const int np = n + (n & 1);  // players of the round-robin (a dummy when n is odd)
    const double eps = sizeof(T) == 8 ? 1e-15 : 1e-7;
    for (int sweep = 0; sweep < 30 && n > 1; ++sweep) {
        if (tid == 0) s_rot = 0;
        __syncthreads();
        for (int round = 0; round < np - 1; ++round) {
            for (int pr = warp; pr < np / 2; pr += nw) {
                // circle method: player np-1 fixed, the others rotate
                int a = pr == 0 ? np - 1 : (round + pr) % (np - 1);
                int b = (round + np - 1 - pr) % (np - 1);
                if (a >= n || b >= n) continue;
                if (a > b) { const int x = a; a = b; b = x; }
                T* x = W + (size_t)a * n;
                T* y = W + (size_t)b * n;
                double al = 0, be = 0, ga = 0;
                for (int r = lane; r < n; r += 32) {
                    const double xr = x[r], yr = y[r];
                    al += xr * xr;
                    be += yr * yr;
                    ga += xr * yr;
                }
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) {
                    al += __shfl_xor_sync(0xffffffffu, al, o);
                    be += __shfl_xor_sync(0xffffffffu, be, o);
                    ga += __shfl_xor_sync(0xffffffffu, ga, o);
                }
                if (fabs(ga) <= eps * sqrt(al * be) || ga == 0.0) continue;
                const double zeta = (be - al) / (2.0 * ga);
                const double tt = (zeta >= 0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
                const double cs = 1.0 / sqrt(1.0 + tt * tt), sn = cs * tt;
                for (int r = lane; r < n; r += 32) {
                    const double xr = x[r], yr = y[r];
                    x[r] = (T)(cs * xr - sn * yr);
                    y[r] = (T)(sn * xr + cs * yr);
                }
                if (lane == 0) s_rot = 1;
            }
            __syncthreads();
        }
        if (!s_rot) break;
        __syncthreads();
    }
    double mn = 1e308;
    for (int j = warp; j < n; j += nw) {
        const T* x = W + (size_t)j * n;
        double ss = 0;
        for (int r = lane; r < n; r += 32) ss += (double)x[r] * (double)x[r];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) ss += __shfl_xor_sync(0xffffffffu, ss, o);
        mn = fmin(mn, sqrt(ss));
    }
    if (lane == 0) red[warp] = mn;
    __syncthreads();
    if (tid == 0) {
        double m2 = red[0];
        for (int q = 1; q < nw; ++q) m2 = fmin(m2, red[q]);
        *t.sinv = 1.0 / m2;
    }
}

// One CTA per (task, 32-column tile of B): thread (i, jj) sums over the rows.
template <class T>
__global__ void __launch_bounds__(256) k_atb_scaled(const AtbTask<T>* tasks, const TileRef* tiles) {
    pdl_enter();
    const TileRef tr = tiles[blockIdx.x];
    const AtbTask<T> t = tasks[tr.task];
    const int j0 = tr.tile * 32;
    const T sc = (T)*t.sinv;
    for (int e = threadIdx.x; e < t.ni * 32; e += blockDim.x) {
        const int jj = e / t.ni, i = e % t.ni;
        const int j = j0 + jj;
        if (j >= t.nj) continue;
        const T* a = t.A + (size_t)i * t.lda;
        const T* b = t.B + (size_t)j * t.ldb;
        T acc = T(0);
        for (int r = 0; r < t.rows; ++r) acc += a[r] * b[r];
        t.C[(size_t)i * t.ldc + t.off + j] = sc * acc;
    }
}

// ------------------------------------------------------------------ assembly scatter
template <class T>
__global__ void k_scatter_values(const uint64_t* addr, const double* vals, int64_t n) {
    pdl_enter();
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x)
        *reinterpret_cast<T*>(addr[e]) = (T)vals[e];
}

// ------------------------------------------------------------------ solve sweeps
template <class T>
__device__ __forceinline__ const T* aptr(int64_t v) {
    return reinterpret_cast<const T*>(v);
}

// Warp transpose-sum: lane q returns sum over the 32 lanes of a[q] (31
// shuffles, recursive halving of the index range).
template <class T>
__device__ __forceinline__ T warp_transpose_sum(T (&a)[32]) {
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

// Scratch of the solve-step CTA (static shared memory).
constexpr int kGemvRefs = 48;  // neighbour-block descriptors a triangular op stages in shared memory
template <class T>
struct SolveShared {
    T wred[(kThreads / 32) * kNB];  // per-warp partials
    T y[kNB], z[kNB];
    T tsh[kNB * (kNB + 1)];         // panel T factor / diagonal block of R
    GemvRef<T> gref[kGemvRefs];
};

// x(0:m) <- Q^T x (dir 0) or Q x (dir 1), Q from unit-lower V (ld ldv) with
// one kNB x kNB T factor per panel (H_panel = I - V T V^T). Per panel, each
// thread walks its rows once for the kNB products V^T x and once for the
// update x -= V z. Every row issues its kNB loads unconditionally (columns
// past the panel's width are clamped to its last column and weighted by zero)
// so that they are all in flight together.
template <class T>
__device__ void apply_q(T* xs, int m, int kq, const T* V, int ldv, const T* tp, int dir, SolveShared<T>& sh) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5, nth = blockDim.x;
    constexpr int TP = kNB + 1;
    const int np = (kq + kNB - 1) / kNB;
    for (int pi = 0; pi < np; ++pi) {
        const int pidx = dir == 0 ? pi : np - 1 - pi;
        const int p0 = pidx * kNB;
        const int w = min(kNB, kq - p0);
        const int wl = w - 1;
        const T* Vp = V + (size_t)p0 * ldv;
        const T* Tp = tp + (size_t)pidx * kNB * kNB;
        for (int e = tid; e < kNB * kNB; e += nth) sh.tsh[(e % kNB) * TP + e / kNB] = Tp[e];
        T acc[kNB];
#pragma unroll
        for (int q = 0; q < kNB; ++q) acc[q] = T(0);
        for (int r = p0 + tid; r < m; r += nth) {
            const T xr = xs[r];
            const int rr = r - p0;
            const T* vr = Vp + r;
            T v[kNB];
#pragma unroll
            for (int q = 0; q < kNB; ++q) v[q] = vr[(size_t)min(q, wl) * ldv];
            if (rr < kNB) {  // unit diagonal, zeros above it
#pragma unroll
                for (int q = 0; q < kNB; ++q) v[q] = q < rr ? v[q] : (q == rr ? T(1) : T(0));
            }
#pragma unroll
            for (int q = 0; q < kNB; ++q) acc[q] += v[q] * xr;
        }
        const T part = warp_transpose_sum(acc);
        sh.wred[warp * kNB + lane] = part;
        __syncthreads();
        if (tid < kNB) {
            T y = T(0);
            for (int q = 0; q < nw; ++q) y += sh.wred[q * kNB + tid];
            sh.y[tid] = y;
        }
        __syncthreads();
        if (tid < kNB) {  // z = T^T y (dir 0) or T y (dir 1); T upper triangular; z = 0 past w
            T s = T(0);
            if (tid < w) {
                if (dir == 0) {
                    for (int l = 0; l <= tid; ++l) s += sh.tsh[l * TP + tid] * sh.y[l];
                } else {
                    for (int l = tid; l < w; ++l) s += sh.tsh[tid * TP + l] * sh.y[l];
                }
            }
            sh.z[tid] = s;
        }
        __syncthreads();
        for (int r = p0 + tid; r < m; r += nth) {
            const int rr = r - p0;
            const T* vr = Vp + r;
            T v[kNB];
#pragma unroll
            for (int q = 0; q < kNB; ++q) v[q] = vr[(size_t)min(q, wl) * ldv];
            if (rr < kNB) {
#pragma unroll
                for (int q = 0; q < kNB; ++q) v[q] = q < rr ? v[q] : (q == rr ? T(1) : T(0));
            }
            T s = T(0);
#pragma unroll
            for (int q = 0; q < kNB; ++q) s += v[q] * sh.z[q];
            xs[r] -= s;
        }
        __syncthreads();
    }
}

// Upper-triangular solve in shared memory: x <- inv(R) x (trans 0) or
// inv(R^T) x (trans 1), in 32-row blocks. Warp 0 holds the diagonal block in
// registers (lane l: row l for trans 0, column l for trans 1) and solves it
// with shuffles; all threads then update the remaining rows, each issuing its
// 32 loads unconditionally (clamped to the block, weighted by zero past it).
template <class T>
__device__ void tri_solve(T* xs, int k, const T* R, int ldr, int trans, SolveShared<T>& sh) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nth = blockDim.x;
    const int nb = (k + 31) / 32;
    for (int bi = 0; bi < nb; ++bi) {
        const int b = trans == 0 ? nb - 1 - bi : bi;
        const int j0 = b * 32, bw = min(32, k - j0);
        const int bl = bw - 1;
        if (warp == 0) {
            T rd[32];
            const int ll = min(lane, bl);
            if (trans == 0) {
#pragma unroll
                for (int i = 0; i < 32; ++i) rd[i] = R[(j0 + ll) + (size_t)(j0 + min(i, bl)) * ldr];
            } else {
#pragma unroll
                for (int i = 0; i < 32; ++i) rd[i] = R[(j0 + min(i, bl)) + (size_t)(j0 + ll) * ldr];
            }
            T xv = lane < bw ? xs[j0 + lane] : T(0);
            if (trans == 0) {
#pragma unroll
                for (int i = 31; i >= 0; --i) {
                    if (i < bw) {
                        if (lane == i) xv = xv / rd[i];
                        const T xi = __shfl_sync(0xffffffffu, xv, i);
                        if (lane < i) xv -= rd[i] * xi;
                    }
                }
            } else {
#pragma unroll
                for (int i = 0; i < 32; ++i) {
                    if (i < bw) {
                        if (lane == i) xv = xv / rd[i];
                        const T xi = __shfl_sync(0xffffffffu, xv, i);
                        if (lane > i) xv -= rd[i] * xi;
                    }
                }
            }
            if (lane < bw) xs[j0 + lane] = xv;
            sh.y[lane] = lane < bw ? xv : T(0);
        }
        __syncthreads();
        if (trans == 0) {
            for (int i = tid; i < j0; i += nth) {
                T rv[32];
#pragma unroll
                for (int l = 0; l < 32; ++l) rv[l] = R[i + (size_t)(j0 + min(l, bl)) * ldr];
                T s = T(0);
#pragma unroll
                for (int l = 0; l < 32; ++l) s += rv[l] * sh.y[l];
                xs[i] -= s;
            }
        } else {
            for (int i = j0 + bw + tid; i < k; i += nth) {
                T rv[32];
#pragma unroll
                for (int l = 0; l < 32; ++l) rv[l] = R[(j0 + min(l, bl)) + (size_t)i * ldr];
                T s = T(0);
#pragma unroll
                for (int l = 0; l < 32; ++l) s += rv[l] * sh.y[l];
                xs[i] -= s;
            }
        }
        __syncthreads();
    }
}

// xs(0:k) <- Ri xs (trans 0) or Ri^T xs (trans 1) with Ri = R^-1 (k x k,
// column-major, exactly zero below the diagonal), the inverse computed at the
// end of the factorization: the triangular solve as one parallel product
// instead of a chain of diagonal blocks. ys (k elements of shared memory)
// holds the result until every thread is done reading xs.
template <class T>
__device__ void rinv_apply(T* xs, T* ys, int k, const T* Ri, int trans) {
    const int tid = threadIdx.x, nth = blockDim.x, lane = tid & 31, warp = tid >> 5, nw = nth >> 5;
    if (trans == 0) {
        // thread i: row i of Ri; a warp starts at its first row's diagonal (the
        // entries left of it are zero), so the warp's loads stay coalesced
        for (int i0 = 0; i0 < k; i0 += nth) {
            const int i = i0 + tid;
            const int ic = min(i, k - 1);
            const int jb = min(i0 + warp * 32, k - 1);
            T a[4] = {T(0), T(0), T(0), T(0)};
            int j = jb;
            for (; j + 3 < k; j += 4) {
                T r[4], x[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    r[u] = Ri[ic + (size_t)(j + u) * k];
                    x[u] = xs[j + u];
                }
#pragma unroll
                for (int u = 0; u < 4; ++u) a[u] += r[u] * x[u];
            }
            for (; j < k; ++j) a[0] += Ri[ic + (size_t)j * k] * xs[j];
            if (i < k) ys[i] = (a[0] + a[1]) + (a[2] + a[3]);
        }
    } else {
        // warp per row i of Ri^T (column i of Ri, contiguous): lanes stride j <= i
        for (int i = warp; i < k; i += nw) {
            const T* col = Ri + (size_t)i * k;
            T a = T(0);
            for (int j = lane; j <= i; j += 32) a += col[j] * xs[j];
            a = warp_sum(a);
            if (lane == 0) ys[i] = a;
        }
    }
    __syncthreads();
    for (int i = tid; i < k; i += nth) xs[i] = ys[i];
    __syncthreads();
}

// xs(0:k) -= sum_b B_b x_b over the neighbour blocks of a triangular op (B_b:
// k x s_b, ld). Threads form G column groups of RT row threads; each thread
// keeps kGU loads of B in flight (a block's last batch clamped to its last
// column and weighted by zero) and the groups meet in shared memory. The
// block descriptors are staged in shared memory first, so walking the blocks
// costs no dependent global load.
template <class T>
__device__ void gemv_sub(T* xs, int k, const GemvRef<T>* gv, int nb, const T* x, SolveShared<T>& sh) {
    constexpr int kGU = 16;
    const int tid = threadIdx.x, nth = blockDim.x;
    const int RT = min(nth, (k + 31) & ~31);
    const int G = nth / RT;
    const int ri = tid % RT, g = tid / RT;
    const bool staged = nb <= kGemvRefs;
    if (staged)
        for (int b = tid; b < nb; b += nth) sh.gref[b] = gv[b];
    __syncthreads();
    const GemvRef<T>* refs = staged ? sh.gref : gv;
    for (int i0 = 0; i0 < k; i0 += RT) {
        const int i = i0 + ri;
        T a[4] = {T(0), T(0), T(0), T(0)};
        if (g < G && i < k) {
            for (int bb = 0; bb < nb; ++bb) {
                const GemvRef<T> r = refs[bb];
                const T* B = aptr<T>(r.boff) + i;
                const T* xn = x + r.xoff;
                const size_t ld = (size_t)r.ld;
                const int sl = r.s - 1;
                for (int j = g; j < r.s; j += kGU * G) {
                    T bv[kGU], xv[kGU];
#pragma unroll
                    for (int u = 0; u < kGU; ++u) {
                        const int jj = min(j + u * G, sl);
                        bv[u] = B[(size_t)jj * ld];
                        xv[u] = xn[jj];
                    }
#pragma unroll
                    for (int u = 0; u < kGU; ++u)
                        if (j + u * G <= sl) a[u & 3] += bv[u] * xv[u];
                }
            }
        }
        const T part = (a[0] + a[1]) + (a[2] + a[3]);
        if (G == 1) {
            if (i < k) xs[i] -= part;
        } else {
            sh.wred[tid] = part;
            __syncthreads();
            if (g == 0 && i < k) {
                T s = T(0);
                for (int q = 0; q < G; ++q) s += sh.wred[q * RT + ri];
                xs[i] -= s;
            }
            __syncthreads();
        }
    }
}

template <class T>
__global__ void __launch_bounds__(kThreads, sizeof(T) == 4 ? 2 : 1) k_solve_step(const SolveOp* ops, const XSeg* segs,
                                                        const GemvRef<T>* gemv, T* x) {
    pdl_enter();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* xs = reinterpret_cast<T*>(smem_raw);
    __shared__ SolveShared<T> sh;
    const SolveOp op = ops[blockIdx.x];
    const int tid = threadIdx.x;
    switch (op.kind) {
        case SK_APPLYQ: {
            const int m = op.a, kq = op.b, ldv = op.c;
            if (op.nseg > 0) {
                int cur = 0;
                for (int s = 0; s < op.nseg; ++s) {
                    const XSeg sg = segs[op.seg0 + s];
                    for (int i = tid; i < sg.len; i += blockDim.x) xs[cur + i] = x[sg.xoff + i];
                    cur += sg.len;
                }
            } else {
                for (int i = tid; i < m; i += blockDim.x) xs[i] = x[op.x0 + i];
            }
            __syncthreads();
            apply_q(xs, m, kq, aptr<T>(op.p0), ldv, aptr<T>(op.p1), op.dir, sh);
            if (op.nseg > 0) {
                int cur = 0;
                for (int s = 0; s < op.nseg; ++s) {
                    const XSeg sg = segs[op.seg0 + s];
                    for (int i = tid; i < sg.len; i += blockDim.x) x[sg.xoff + i] = xs[cur + i];
                    cur += sg.len;
                }
            } else {
                for (int i = tid; i < m; i += blockDim.x) x[op.x0 + i] = xs[i];
            }
            break;
        }
        case SK_TRI: {
            // p0 == 0: R is the identity (the fine cluster of an order-1.5 sparsification,
            // whose QR op only subtracts the E2 term)
            const int k = op.a, ldr = op.c;
            const T* R = aptr<T>(op.p0);
            const bool has_r = op.p0 != 0;
            for (int i = tid; i < k; i += blockDim.x) xs[i] = x[op.x0 + i];
            __syncthreads();
            const T* Ri = op.p1 != 0 ? aptr<T>(op.p1) : nullptr;  // R^-1 when it was formed
            if (op.dir == 0) {
                gemv_sub(xs, k, gemv + op.seg0, op.nseg, x, sh);
                __syncthreads();
                if (Ri)
                    rinv_apply(xs, xs + k, k, Ri, 0);
                else if (has_r)
                    tri_solve(xs, k, R, ldr, 0, sh);
                for (int i = tid; i < k; i += blockDim.x) x[op.x0 + i] = xs[i];
            } else {
                if (Ri)
                    rinv_apply(xs, xs + k, k, Ri, 1);
                else if (has_r)
                    tri_solve(xs, k, R, ldr, 1, sh);
                for (int i = tid; i < k; i += blockDim.x) x[op.x0 + i] = xs[i];
                // x_n -= B_n^T xs: a warp takes 8 neighbour columns at a time (their
                // loads in flight together; columns past the block re-read its last
                // column and are dropped), lanes stride the rows; each column's sum
                // is the lane-strided partial sums folded by warp_sum
                constexpr int kCG = 8;
                const int lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
                for (int b = 0; b < op.nseg; ++b) {
                    const GemvRef<T> g = gemv[op.seg0 + b];
                    const T* B = aptr<T>(g.boff);
                    const int ngrp = (g.s + kCG - 1) / kCG;
                    for (int grp = warp; grp < ngrp; grp += nw) {
                        const int j0 = grp * kCG;
                        const T* bc[kCG];
#pragma unroll
                        for (int u = 0; u < kCG; ++u) bc[u] = B + (size_t)min(j0 + u, g.s - 1) * g.ld;
                        T sacc[kCG];
#pragma unroll
                        for (int u = 0; u < kCG; ++u) sacc[u] = T(0);
                        for (int i = lane; i < k; i += 32) {
                            const T xi = xs[i];
                            T bv[kCG];
#pragma unroll
                            for (int u = 0; u < kCG; ++u) bv[u] = bc[u][i];
#pragma unroll
                            for (int u = 0; u < kCG; ++u) sacc[u] += bv[u] * xi;
                        }
                        T mine = T(0);
#pragma unroll
                        for (int u = 0; u < kCG; ++u) {
                            const T su = warp_sum(sacc[u]);
                            if (lane == u) mine = su;
                        }
                        if (lane < kCG && j0 + lane < g.s) x[g.xoff + j0 + lane] -= mine;
                    }
                }
            }
            break;
        }
        case SK_SPLIT: {
            const int crows = op.a, ccols = op.b, rank = op.c;
            T* xc = x + op.x0;
            T* xf = x + op.x1;
            for (int i = tid; i < crows; i += blockDim.x) xs[i] = xc[i];
            __syncthreads();
            const int nf = ccols - rank, nr = crows - ccols;
            if (op.dir == 0) {
                for (int q = tid; q < nf; q += blockDim.x) xf[q] = xs[rank + q];
                for (int q = tid; q < nr; q += blockDim.x) xc[rank + q] = xs[ccols + q];
                for (int q = tid; q < nf; q += blockDim.x) xc[crows - nf + q] = xs[rank + q];
            } else {
                for (int q = tid; q < nf; q += blockDim.x) xc[rank + q] = xf[q];
                for (int q = tid; q < nr; q += blockDim.x) xc[ccols + q] = xs[rank + q];
            }
            break;
        }
        case SK_SPLIT0: {
            const int cfull = op.a, chead = op.b, fs = op.c;
            T* xc = x + op.x0;
            T* xf = x + op.x1;
            if (op.dir == 0) {
                for (int q = tid; q < fs; q += blockDim.x) xf[q] = xc[cfull - fs + q];
            } else {
                for (int q = tid; q < fs; q += blockDim.x) xc[chead - fs + q] = xf[q];
            }
            break;
        }
        case SK_SPLIT0_T: {
            const int cfull = op.a, chead = op.b, fs = op.c;
            T* xc = x + op.x0;
            T* xf = x + op.x1;
            if (op.dir == 0) {
                for (int q = tid; q < fs; q += blockDim.x) {
                    xc[cfull - fs + q] += xf[q];
                    xf[q] = T(0);
                }
            } else {
                for (int q = tid; q < fs; q += blockDim.x) {
                    xf[q] += xc[chead - fs + q];
                    xc[chead - fs + q] = T(0);
                }
            }
            break;
        }
        case SK_MERGE: {
            // dir 0: parent <- children rows; dir 1: children cols <- parent
            int cur = 0;
            for (int s = 0; s < op.nseg; ++s) {
                const XSeg sg = segs[op.seg0 + s];
                const int len = op.dir == 0 ? sg.len : sg.pad;
                if (op.dir == 0)
                    for (int i = tid; i < len; i += blockDim.x) x[op.x0 + cur + i] = x[sg.xoff + i];
                else
                    for (int i = tid; i < len; i += blockDim.x) x[sg.xoff + i] = x[op.x0 + cur + i];
                cur += len;
            }
            break;
        }
        case SK_REASSIGN: {
            // Reassign (src/operations.cpp:60-69, src/toperations.cpp:62-70): dir 0
            // moves x(c)[idx[i]] to x(n)[nstart + i]; dir 1 (transposed tape) moves
            // them back. idx holds positions inside c's segment.
            const int nr = op.a;
            const int* idx = reinterpret_cast<const int*>(op.p0);
            T* xc = x + op.x0;
            T* xn = x + op.x1;
            for (int i = tid; i < nr; i += blockDim.x) {
                if (op.dir == 0)
                    xn[i] = xc[idx[i]];
                else
                    xc[idx[i]] = xn[i];
            }
            break;
        }
        case SK_SPLIT_T: {
            // Transposes of the SplitD index maps (adjoint sweeps): dir 0 undoes
            // the forward split (the fine part's adjoint folds back into c and
            // f's adjoint is consumed), dir 1 the backward split.
            const int crows = op.a, ccols = op.b, rank = op.c;
            T* yc = x + op.x0;
            T* yf = x + op.x1;
            for (int i = tid; i < crows; i += blockDim.x) xs[i] = yc[i];
            __syncthreads();
            const int nf = ccols - rank, nr = crows - ccols;
            if (op.dir == 0) {
                for (int q = tid; q < nf; q += blockDim.x) {
                    yc[rank + q] = xs[crows - nf + q] + yf[q];
                    yf[q] = T(0);
                }
                for (int q = tid; q < nr; q += blockDim.x) yc[ccols + q] = xs[rank + q];
            } else {
                for (int q = tid; q < nf; q += blockDim.x) yf[q] += xs[rank + q];
                for (int q = tid; q < nr; q += blockDim.x) yc[rank + q] = xs[ccols + q];
                for (int q = tid; q < nf; q += blockDim.x) yc[rank + nr + q] = T(0);
            }
            break;
        }
        case SK_MERGE_T: {
            // dir 0 (transpose of parent <- children rows): children += parent
            // pieces, parent pieces zeroed; dir 1 (transpose of children cols <-
            // parent): parent pieces += children, children zeroed.
            int cur = 0;
            for (int s = 0; s < op.nseg; ++s) {
                const XSeg sg = segs[op.seg0 + s];
                const int len = op.dir == 0 ? sg.len : sg.pad;
                T* yp = x + op.x0 + cur;
                T* ych = x + sg.xoff;
                if (op.dir == 0) {
                    for (int i = tid; i < len; i += blockDim.x) {
                        ych[i] += yp[i];
                        yp[i] = T(0);
                    }
                } else {
                    for (int i = tid; i < len; i += blockDim.x) {
                        yp[i] += ych[i];
                        ych[i] = T(0);
                    }
                }
                cur += len;
            }
            break;
        }
        default:
            break;
    }
}

template <class T>
__global__ void k_seg_copy(const T* src, T* dst, const int64_t* pos, int n) {
    pdl_enter();
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) dst[pos[i]] = src[pos[i]];
}

// out[t][i] = || row (row0 + i) of block t || (FP64 sums), one warp per row.
template <class T>
__global__ void k_row_norms(const RowNormTask<T>* tasks, int ntasks, double* out) {
    pdl_enter();
    const int lane = threadIdx.x & 31;
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int t = 0; t < ntasks; ++t) {
        const RowNormTask<T> k = tasks[t];
        for (int i = gw; i < k.rows; i += nwarps) {
            const T* row = k.p + k.row0 + i;
            double s = 0.0;
            for (int j = lane; j < k.cols; j += 32) {
                const double v = (double)row[(size_t)j * k.ld];
                s += v * v;
            }
            s = warp_sum(s);
            if (lane == 0) out[k.out + i] = sqrt(s);
        }
    }
}

template <class T>
__global__ void k_gather_in(const double* b, const int* src, const int64_t* xpos, T* x, int n) {
    pdl_enter();
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) x[xpos[i]] = (T)b[src[i]];
}
template <class T>
__global__ void k_scatter_out(const T* x, const int64_t* xpos, const int* dst, double* out, int n) {
    pdl_enter();
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        out[dst[i]] = (double)x[xpos[i]];
}

// ------------------------------------------------------------------ Krylov (FP64)
constexpr int kRedBlocks = 296;

__global__ void k_spmv(int m, const int* rp, const int* ci, const double* v, const double* x, double* y) {
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < m; r += gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int q = rp[r]; q < rp[r + 1]; ++q) s += v[q] * x[ci[q]];
        y[r] = s;
    }
}

// partials[b] = block b's share of sum_{i >= lo} a[i] b[i]; if head is given,
// partials[gridDim.x] = *head (read before any later kernel changes it).
__global__ void k_dot_partials(const double* a, const double* b, int lo, int m, double* partials,
                               const double* head) {
    __shared__ double red[32];
    double s = 0.0;
    for (int i = lo + blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x)
        s += b ? a[i] * b[i] : a[i] * a[i];
    s = block_sum(s, red);
    if (threadIdx.x == 0) partials[blockIdx.x] = s;
    if (head && blockIdx.x == 0 && threadIdx.x == 0) partials[gridDim.x] = *head;
}

__device__ double sum_partials(const double* partials, int nblk, double* red) {
    double s = 0.0;
    for (int i = threadIdx.x; i < nblk; i += blockDim.x) s += partials[i];
    return block_sum(s, red);
}

// v[i:] <- (I - tau h h^T) v[i:], h = [1; ess]; partials hold sum_{r>i} ess[r-i-1] v[r]
// and, at index nblk, v[i] as it was before this kernel (block 0 rewrites v[i],
// so no block may read it here).
__global__ void k_apply_reflector(const double* ess, const double* tau, double* v, int i, int m,
                                  const double* partials, int nblk) {
    __shared__ double red[32];
    const double d = sum_partials(partials, nblk, red) + partials[nblk];
    const double tv = *tau;
    if (tv == 0.0) return;
    __syncthreads();
    const double f = tv * d;
    for (int r = i + 1 + blockIdx.x * blockDim.x + threadIdx.x; r < m; r += gridDim.x * blockDim.x)
        v[r] -= f * ess[r - i - 1];
    if (blockIdx.x == 0 && threadIdx.x == 0) v[i] -= f;
}

// makeHouseholder of v[k:]: partials hold sum_{r>k} v[r]^2.
__global__ void k_make_reflector(const double* v, int k, int m, double* ess, double* tau, double* beta,
                                 const double* partials, int nblk) {
    __shared__ double red[32];
    const double tail = sum_partials(partials, nblk, red);
    const double c0 = v[k];
    double b, tv;
    const bool zero = tail <= DBL_MIN;
    if (zero) {
        tv = 0.0;
        b = c0;
    } else {
        b = sqrt(c0 * c0 + tail);
        if (c0 >= 0.0) b = -b;
        tv = (b - c0) / b;
    }
    for (int r = k + 1 + blockIdx.x * blockDim.x + threadIdx.x; r < m; r += gridDim.x * blockDim.x)
        ess[r - k - 1] = zero ? 0.0 : v[r] / (c0 - b);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        *tau = tv;
        *beta = b;
    }
}

__global__ void k_axpby(int n, double a, const double* x, double b, double* y) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) y[i] = a * x[i] + b * y[i];
}
__global__ void k_sub(int n, const double* a, const double* b, double* y) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) y[i] = a[i] - b[i];
}

inline int grid_for(int64_t n, int threads, int cap = 148 * 16) {
    int64_t g = (n + threads - 1) / threads;
    if (g < 1) g = 1;
    if (g > cap) g = cap;
    return (int)g;
}

template <class T>
size_t trailing_tc_smem() {
    return sizeof(T) * ((size_t)(kNB + kTN) * kTCS + (size_t)kNB * (kTN + 1) + (size_t)kNB * (kNB + 1));
}

}  // namespace

// ------------------------------------------------------------------ launchers
static void pdl_check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw std::runtime_error(std::string(what) + " launch: " + cudaGetErrorString(e));
}

template <class T>
void launch_copy(const CopyDesc<T>* d, int n, int max_cols, cudaStream_t s) {
    if (n <= 0) return;
    const int chunks = std::max(1, std::min(32, (max_cols + 31) / 32));
    pdl_check(launch_pdl(k_copy<T>, dim3(n < 65535 ? n : 65535, chunks), dim3(256), 0, s, 0, d, n), "k_copy");
}

template <class T>
void launch_panel(const QRTask<T>* tasks, const int* ids, int ntasks, int p, int smem_rows, cudaStream_t s) {
    if (ntasks <= 0) return;
    size_t smem = (size_t)smem_rows * kNB * sizeof(T);
    pdl_check(launch_pdl(k_panel<T>, dim3(ntasks), dim3(kThreads), smem, s, 0, tasks, ids, p, smem_rows), "k_panel");
}

template <class T>
void launch_trailing(const QRTask<T>* tasks, const TileRef* tiles, int ntiles, int p, cudaStream_t s) {
    if (ntiles <= 0) return;
    pdl_check(launch_pdl(k_trailing_tc<T>, dim3(ntiles), dim3(kThreads), trailing_tc_smem<T>(), s, 0, tasks, tiles, p),
              "k_trailing_tc");
}

template <class T>
void launch_trsm(const TrsmTask<T>* tasks, const TileRef* tiles, int ntiles, cudaStream_t s) {
    if (ntiles <= 0) return;
    pdl_check(launch_pdl(k_trsm_tc<T>, dim3(ntiles), dim3(128), trsm_tc_smem<T>(), s, 0, tasks, tiles), "k_trsm_tc");
}

template <class T>
void launch_product_norms(const ProdNormTask<T>* tasks, int ntasks, double* out, cudaStream_t s) {
    if (ntasks <= 0) return;
    pdl_check(launch_pdl(k_product_norm<T>, dim3(ntasks), dim3(256), 0, s, 0, tasks, out), "k_product_norm");
}

template <class T>
void launch_sigma_min(const SigmaTask<T>* tasks, int ntasks, cudaStream_t s) {
    if (ntasks <= 0) return;
    pdl_check(launch_pdl(k_sigma_min<T>, dim3(ntasks), dim3(256), 0, s, 0, tasks), "k_sigma_min");
}
template <class T>
void launch_atb_scaled(const AtbTask<T>* tasks, const TileRef* tiles, int ntiles, cudaStream_t s) {
    if (ntiles <= 0) return;
    pdl_check(launch_pdl(k_atb_scaled<T>, dim3(ntiles), dim3(256), 0, s, 0, tasks, tiles), "k_atb_scaled");
}

template <class T>
void launch_unit_diag(const TrsmTask<T>* tasks, int ntasks, cudaStream_t s) {
    if (ntasks <= 0) return;
    pdl_check(launch_pdl(k_unit_diag<T>, dim3(ntasks), dim3(256), 0, s, 0, tasks), "k_unit_diag");
}

template <class T>
void launch_scatter_values(const uint64_t* addr, const double* vals, int64_t n, cudaStream_t s) {
    if (n <= 0) return;
    pdl_check(launch_pdl(k_scatter_values<T>, dim3(grid_for(n, 256)), dim3(256), 0, s, 0, addr, vals, n),
              "k_scatter_values");
}

template <class T>
void launch_solve_step(const SolveOp* ops, int nops, const XSeg* segs, const GemvRef<T>* gemv, const T* arena,
                       T* x, int smem_elems, cudaStream_t s) {
    (void)arena;
    if (nops <= 0) return;
    size_t smem = (size_t)(smem_elems < 32 ? 32 : smem_elems) * sizeof(T);
    pdl_check(launch_pdl(k_solve_step<T>, dim3(nops), dim3(kThreads), smem, s, 0, ops, segs, gemv, x), "k_solve_step");
}

template <class T>
void launch_seg_copy(const T* src, T* dst, const int64_t* pos, int n, cudaStream_t s) {
    if (n <= 0) return;
    pdl_check(launch_pdl(k_seg_copy<T>, dim3(grid_for(n, 256)), dim3(256), 0, s, 0, src, dst, pos, n), "k_seg_copy");
}
template <class T>
void launch_row_norms(const RowNormTask<T>* tasks, int ntasks, int total_rows, double* out, cudaStream_t s) {
    if (ntasks <= 0 || total_rows <= 0) return;
    pdl_check(launch_pdl(k_row_norms<T>, dim3(grid_for((int64_t)total_rows * 32, 256, 148 * 8)), dim3(256), 0, s, 0,
                         tasks, ntasks, out),
              "k_row_norms");
}

template <class T>
void launch_gather_in(const double* b, const int* src, const int64_t* xpos, T* x, int n, cudaStream_t s) {
    pdl_check(launch_pdl(k_gather_in<T>, dim3(grid_for(n, 256)), dim3(256), 0, s, 0, b, src, xpos, x, n), "k_gather_in");
}
template <class T>
void launch_scatter_out(const T* x, const int64_t* xpos, const int* dst, double* out, int n, cudaStream_t s) {
    pdl_check(launch_pdl(k_scatter_out<T>, dim3(grid_for(n, 256)), dim3(256), 0, s, 0, x, xpos, dst, out, n),
              "k_scatter_out");
}

void launch_spmv_csr(int m, const int* rp, const int* ci, const double* v, const double* x, double* y,
                     cudaStream_t s) {
    k_spmv<<<grid_for(m, 256, 148 * 32), 256, 0, s>>>(m, rp, ci, v, x, y);
}
void launch_dot_partials(const double* a, const double* b, int lo, int m, double* partials, int nblk,
                         cudaStream_t s, const double* head) {
    k_dot_partials<<<nblk, 256, 0, s>>>(a, b, lo, m, partials, head);
}
void launch_apply_reflector(const double* ess, const double* tau, double* v, int i, int m, const double* partials,
                            int nblk, cudaStream_t s) {
    k_apply_reflector<<<nblk, 256, 0, s>>>(ess, tau, v, i, m, partials, nblk);
}
void launch_make_reflector(double* v, int k, int m, double* ess_col, double* tau, double* beta,
                           const double* partials, int nblk, cudaStream_t s) {
    k_make_reflector<<<nblk, 256, 0, s>>>(v, k, m, ess_col, tau, beta, partials, nblk);
}
void launch_axpby(int n, double a, const double* x, double b, double* y, cudaStream_t s) {
    k_axpby<<<grid_for(n, 256), 256, 0, s>>>(n, a, x, b, y);
}
void launch_sub(int n, const double* a, const double* b, double* y, cudaStream_t s) {
    k_sub<<<grid_for(n, 256), 256, 0, s>>>(n, a, b, y);
}
int reduce_blocks() { return kRedBlocks; }

void prepare_krylov_kernels() {
    once_per_device(reinterpret_cast<const void*>(&k_spmv), [] {
        const void* fns[] = {reinterpret_cast<const void*>(&k_spmv), reinterpret_cast<const void*>(&k_dot_partials),
                             reinterpret_cast<const void*>(&k_apply_reflector),
                             reinterpret_cast<const void*>(&k_make_reflector), reinterpret_cast<const void*>(&k_axpby),
                             reinterpret_cast<const void*>(&k_sub)};
        for (const void* f : fns) {
            cudaFuncAttributes a;
            cudaFuncGetAttributes(&a, f);
        }
    });
}

void once_per_device(const void* key, void (*setup)()) {
    static std::mutex mu;
    static std::set<std::pair<const void*, int>> seen;
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> g(mu);  // held while setup runs: no launch sees a half-done setup
    if (seen.insert({key, dev}).second) setup();
}

// Function attributes belong to the device's context: set once per device
// (thread-safe; handles on several threads or devices share them).
template <class T>
void prepare_kernels() {
    once_per_device(reinterpret_cast<const void*>(&k_panel<T>), [] {
        cudaFuncSetAttribute(k_panel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024);
        cudaFuncSetAttribute(k_trailing_tc<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)trailing_tc_smem<T>());
        cudaFuncSetAttribute(k_trsm_tc<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)trsm_tc_smem<T>());
        cudaFuncSetAttribute(k_solve_step<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    });
}

#define SPQ_INST(T)                                                                                           \
    template void launch_copy<T>(const CopyDesc<T>*, int, int, cudaStream_t);                                 \
    template void launch_panel<T>(const QRTask<T>*, const int*, int, int, int, cudaStream_t);                 \
    template void launch_trailing<T>(const QRTask<T>*, const TileRef*, int, int, cudaStream_t);               \
    template void launch_trsm<T>(const TrsmTask<T>*, const TileRef*, int, cudaStream_t);                      \
    template void launch_unit_diag<T>(const TrsmTask<T>*, int, cudaStream_t);                                   \
    template void launch_product_norms<T>(const ProdNormTask<T>*, int, double*, cudaStream_t);                  \
    template void launch_sigma_min<T>(const SigmaTask<T>*, int, cudaStream_t);                                  \
    template void launch_atb_scaled<T>(const AtbTask<T>*, const TileRef*, int, cudaStream_t);                   \
    template void launch_scatter_values<T>(const uint64_t*, const double*, int64_t, cudaStream_t);         \
    template void launch_solve_step<T>(const SolveOp*, int, const XSeg*, const GemvRef<T>*, const T*, T*, int, \
                                       cudaStream_t);                                                          \
    template void launch_gather_in<T>(const double*, const int*, const int64_t*, T*, int, cudaStream_t);      \
    template void launch_seg_copy<T>(const T*, T*, const int64_t*, int, cudaStream_t);                         \
    template void launch_row_norms<T>(const RowNormTask<T>*, int, int, double*, cudaStream_t);                \
    template void launch_scatter_out<T>(const T*, const int64_t*, const int*, double*, int, cudaStream_t);    \
    template void prepare_kernels<T>();

SPQ_INST(double)
SPQ_INST(float)

}  // namespace spq
