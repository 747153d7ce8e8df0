// Device kernels of the spaQR factorization and solve, with their batched task
// descriptors. Every launch takes an array of descriptors resident in device
// memory; one CTA (or a few) serves one descriptor. T is double (plain form) or
// float (FP32 factor form).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

namespace spq {

constexpr int kNB = 32;  // Householder panel width (columns per compact-WY block)
constexpr int kTN = 32;  // trailing-update tile width (columns per CTA)

// ---------------------------------------------------------------- copies
// dst(rows x cols, ld dld) = src(rows x cols, ld sld); src == nullptr writes 0;
// mode 1 writes the identity pattern instead of copying; mode 2 writes the
// transpose (dst(j, i) = src(i, j), dst is cols x rows).
template <class T>
struct CopyDesc {
    const T* src;
    T* dst;
    int sld, dld, rows, cols;
    int mode, pad;
};
// Runs setup the first time it is called for this key on the current device
// (thread-safe; callers wait until it has run): per-device one-time setup
// such as function attributes.
void once_per_device(const void* key, void (*setup)());

// Batched copies; max_cols = the widest descriptor (sets the column-chunk grid).
template <class T>
void launch_copy(const CopyDesc<T>* d, int n, int max_cols, cudaStream_t s);

// ---------------------------------------------------------------- Householder QR
// A task factors the first k columns of the m x (k + ntr) matrix [fac | tr]
// (both column-major, ld m) and applies the reflectors to the ntr trailing
// columns. Outputs: R (upper) and V (strictly lower, unit diagonal implied) in
// fac, tau[k], and one NB x NB triangular factor per panel in tp
// (H_panel = I - V T V^T, LAPACK dlarft forward/columnwise convention).
template <class T>
struct QRTask {
    T* fac;
    T* tr;
    T* tau;
    T* tp;
    int m, k, ntr;
    int tr_only;          // 1: the trailing updates touch tr only (fac holds finished reflectors: V of a sparsified interface)
    int* status = nullptr;  // device status word (kStat* bits), or none
};
// Bits of the device status word of a factorization.
constexpr int kStatNonFinite = 1;  // NaN or Inf in a pivot (R_kk) of a QR or RRQR
constexpr int kStatZeroPivot = 2;  // an exactly zero R_kk in an elimination or scaling QR
constexpr int kStatRRQRNaN = 4;    // a sparsification RRQR found no finite column norm left
struct TileRef {
    int task, tile;
};
// Panel p (columns [p, p+NB)) of every listed task.
template <class T>
void launch_panel(const QRTask<T>* tasks, const int* task_ids, int ntasks, int p, int smem_rows,
                  cudaStream_t s);
// Panel p of every listed task on thread-block clusters of `cluster` CTAs
// (row slabs in shared memory, one cluster barrier per column). task_ids
// holds ntasks task indices followed by each task's own cluster size CLt
// (1 <= CLt <= cluster; the task uses its first CLt CTAs): the panel height
// m - p must be at least 32 * CLt when CLt > 1 and at most
// panel_cl_max_rows(CLt); max_slab = the largest ceil((m - p) / CLt).
template <class T>
cudaError_t launch_panel_cl(const QRTask<T>* tasks, const int* task_ids, int ntasks, int cluster, int max_slab, int p,
                            cudaStream_t s);
template <class T>
size_t panel_cl_max_rows(int cluster);
// Panel p of every listed task held in registers: slabs of at most
// kPanelRegRows rows (2 kPanelRegRows in FP32 without clusters), task_ids as
// for launch_panel_cl with CLt = ceil((m - p) / kPanelRegRows) (so
// m - p <= 16 * kPanelRegRows); max_slab = the largest ceil((m - p) / CLt)
// (it picks the rows per lane).
constexpr int kPanelRegRows = 256;
template <class T>
cudaError_t launch_panel_reg(const QRTask<T>* tasks, const int* task_ids, int ntasks, int cluster, int max_slab,
                             int p, cudaStream_t s);
// Trailing update after panel p: tiles of kTN columns of [fac(:, p+NB:k) | tr].
template <class T>
void launch_trailing(const QRTask<T>* tasks, const TileRef* tiles, int ntiles, int p, cudaStream_t s);

// ---------------------------------------------------------------- TRSM
// X(rows x k) <- X * inv(R), R upper k x k (ld ldr). One CTA per 128-row tile.
template <class T>
struct TrsmTask {
    const T* R;
    T* X;
    int ldr, k, ldx, rows;
};
template <class T>
void launch_trsm(const TrsmTask<T>* tasks, const TileRef* tiles, int ntiles, cudaStream_t s);
// ||A1^T A2||_F of fill candidates (the numeric fill test of the ordering
// without coordinates, src/tree.cpp:856-859): A1 rows x c1 and A2 rows x c2,
// column-major, summed in FP64.
template <class T>
struct ProdNormTask {
    const T* a1;
    const T* a2;
    int ld1, ld2, rows, c1, c2, pad;
};
template <class T>
void launch_product_norms(const ProdNormTask<T>* tasks, int ntasks, double* out, cudaStream_t s);
// --scale 0 sparsification (sparsify, src/tree.cpp:887-989):
// sinv = 1 / sigma_min(R) of an upper-triangular n x n R (ld), the smallest
// singular value of the stacked [A_pp; A_mp] after its QR (gesvd_values,
// src/util.cpp:767-782), by one-sided Jacobi on a copy in work (n x n).
template <class T>
struct SigmaTask {
    const T* R;
    T* work;
    double* sinv;
    int ld, n;
};
template <class T>
void launch_sigma_min(const SigmaTask<T>* tasks, int ntasks, cudaStream_t s);
// C(i, off + j) = sinv * sum_r A(r, i) B(r, j) into a row-major C (row stride
// ldc): the A_pp^T A_pm columns of the sparsification matrix. A rows x ni,
// B rows x nj, column-major.
template <class T>
struct AtbTask {
    const T* A;
    const T* B;
    T* C;
    const double* sinv;
    int lda, ldb, ldc, rows, ni, nj, off, pad;
};
template <class T>
void launch_atb_scaled(const AtbTask<T>* tasks, const TileRef* tiles, int ntiles, cudaStream_t s);
// X(i, i) = 1 for i < k of every task (with X zeroed, the identity whose TRSM by
// R is R^-1; the solve's triangular ops of size <= kRinvMax use it).
template <class T>
void launch_unit_diag(const TrsmTask<T>* tasks, int ntasks, cudaStream_t s);
constexpr int kRinvMax = 1024;

// ---------------------------------------------------------------- truncated RRQR
// Write-back after the RRQR (sparsifyD, src/tree.cpp:1082-1110): rebuild the
// interface's column blocks (A(n2, c) <- first rank columns of (Crank P^T)^T)
// and row blocks (top rank rows <- Crank P^T), save V and tau for the solve and
// build the panel T factors of V. Block descriptor:
template <class T>
struct SpBlock {
    T* p;
    int ld, rows, cols, coff, kind;  // kind 0: column block (Amp), 1: row block (Apm)
};
// Cluster-parallel truncated RRQR on a ROW-major C (row stride ldc). Outputs:
// rank, tau[0:rank), pos[c] = pivot position of column c (inverse permutation,
// positions >= rank for the non-pivot columns), colat[q] = column at position
// q (jpvt). One cluster of `cluster` CTAs per task.
template <class T>
struct RRQRTaskRM {
    T* C;
    int* pos;
    int* colat;
    T* tau;
    T* vn1;
    T* vn2;
    int* rank;
    int m, n, ldc, pad;
    double tol;
    int* status = nullptr;  // device status word (kStat* bits), or none
};
template <class T>
cudaError_t launch_rrqr_rm(const RRQRTaskRM<T>* tasks, const int* ids, int ntasks, int cluster, int max_m,
                           int max_n, cudaStream_t s);
// Blocked form of the same factorization (LAPACK dlaqps: the update of the
// rows below a block of pivot steps is deferred to one rank-NB update, NB = 32
// in FP32 and 16 in FP64). Each CTA keeps the F factor of its slab and a copy
// of the block's reflectors in shared memory; rrqr_blk_fits tells whether a
// launch shape fits (else launch_rrqr_blk returns cudaErrorInvalidValue
// without a launch). The result does not depend on the cluster size.
template <class T>
bool rrqr_blk_fits(int max_m, int max_n, int cluster);
template <class T>
cudaError_t launch_rrqr_blk(const RRQRTaskRM<T>* tasks, const int* ids, int ntasks, int cluster, int max_m,
                            int max_n, cudaStream_t s);
// Write-back after the cluster RRQR, with the rank r known on the host.
template <class T>
struct SparsWBRM {
    const T* C;
    const int* pos;
    const int* colat;
    const T* tau_in;
    T* V;    // m x r, ld m (null: rebuild the blocks only)
    T* tau;  // r
    T* tp;   // panel T factors of V
    int m, ldc, r, nblk, blk0, pad;
};
// parts: CTAs per task (blocks, V column groups and T panels are spread over them)
template <class T>
void launch_spars_wb_rm(const SparsWBRM<T>* tasks, const SpBlock<T>* blocks, int ntasks, int parts, cudaStream_t s);

// ---------------------------------------------------------------- assembly
// *(T*)dst_addr[e] = (T) vals[e]
template <class T>
void launch_scatter_values(const uint64_t* dst_addr, const double* vals, int64_t n, cudaStream_t s);

// ---------------------------------------------------------------- solve sweeps
// One CTA per op; all ops of one launch are independent.
enum SolveKind : int {
    SK_APPLYQ = 0,  // x <- Q^T x (dir 0) or Q x (dir 1); gathered or contiguous x
    SK_TRI = 1,     // x <- inv(R) (x - sum_b B_b x_b)  or transposed variant
    SK_SPLIT = 2,   // SplitD fwd/bwd index shuffle
    SK_MERGE = 3,   // Merge fwd/bwd copies
    SK_REASSIGN = 4, // rectangular row reassignment: dir 0 x(n)[nstart + i] = x(c)[idx[i]], dir 1 back
    SK_SPLIT_T = 5, // transpose of SK_SPLIT (same dir)
    SK_MERGE_T = 6, // transpose of SK_MERGE (same dir): add into the source, zero the target
    SK_SPLIT0 = 7,  // Split of --scale 0 (src/operations.cpp:118-119): dir 0 x(f) <- last a.. rows of
                    // x(c)'s full segment (a = its length, c = x(f)'s length); dir 1 the last entries
                    // of x(c)'s head (b = its length) <- x(f)
    SK_SPLIT0_T = 8 // transpose of SK_SPLIT0 (same dir): add into the source, zero the target
};
struct SolveOp {
    int kind, dir;
    int a, b, c, d;       // kind-specific sizes
    int64_t x0, x1;       // x offsets
    int64_t p0, p1, p2;   // offsets into the factor arena (elements) / segment tables
    int seg0, nseg;       // segment / block range
};
struct XSeg {
    int64_t xoff;
    int len, pad;
};
template <class T>
struct GemvRef {
    int64_t boff;  // offset of the block in the arena
    int64_t xoff;  // x segment of the neighbour
    int ld, s;
};
template <class T>
void launch_solve_step(const SolveOp* ops, int nops, const XSeg* segs, const GemvRef<T>* gemv, const T* arena,
                       T* x, int smem_elems, cudaStream_t s);
// SK_APPLYQ ops on thread-block clusters of `cluster` CTAs, each CTA holding
// ceil(m / cluster) <= kApplyqClRows rows of the op's x.
constexpr int kApplyqClRows = 256;
template <class T>
cudaError_t launch_applyq_cl(const SolveOp* ops, int nops, int cluster, const XSeg* segs, T* x, cudaStream_t s);
// SK_TRI ops of dir 0 whose R^-1 was formed (p1) or whose R is the identity
// (p0 == 0), with at most kTriMaxRefs neighbour blocks and k <= kmax <=
// kRinvMax, on thread-block clusters of `cluster` CTAs: the neighbour columns
// and then the rows of R^-1 are split over the cluster (a DSMEM reduction
// between the two).
constexpr int kTriMaxCl = 16;
constexpr int kTriMaxRefs = 64;
template <class T>
cudaError_t launch_tri_cl(const SolveOp* ops, int nops, int cluster, int kmax, const GemvRef<T>* gemv, T* x,
                          cudaStream_t s);
// dst[pos[k]] = src[pos[k]] (one x buffer into the other at the given positions)
template <class T>
void launch_seg_copy(const T* src, T* dst, const int64_t* pos, int n, cudaStream_t s);
// Norms of rows row0 .. row0 + rows - 1 of a column-major block (rectangular
// row reassignment, src/tree.cpp:319-345); results at out[out_off + i].
template <class T>
struct RowNormTask {
    const T* p;
    int ld, row0, rows, cols;
    int64_t out;
};
template <class T>
void launch_row_norms(const RowNormTask<T>* tasks, int ntasks, int total_rows, double* out, cudaStream_t s);
// x[xpos[k]] = (T) b[src[k]]  /  out[dst[k]] = (double) x[xpos[k]]
template <class T>
void launch_gather_in(const double* b, const int* src, const int64_t* xpos, T* x, int n, cudaStream_t s);
template <class T>
void launch_scatter_out(const T* x, const int64_t* xpos, const int* dst, double* out, int n, cudaStream_t s);

// ---------------------------------------------------------------- Krylov helpers (FP64)
void launch_spmv_csr(int m, const int* rp, const int* ci, const double* v, const double* x, double* y,
                     cudaStream_t s);
// partial sums of a[i]*b[i] (or a[i]^2 if b == nullptr) over [lo, m): nblk partials,
// plus partials[nblk] = *head when head is given (the reflector's head element).
void launch_dot_partials(const double* a, const double* b, int lo, int m, double* partials, int nblk,
                         cudaStream_t s, const double* head = nullptr);
// v[i:] <- (I - tau h h^T) v[i:] with h = [1; ess], ess = H[i+1:, col]; dot from partials
// (launch_dot_partials with head = v + i)
void launch_apply_reflector(const double* ess, const double* tau, double* v, int i, int m, const double* partials,
                            int nblk, cudaStream_t s);
// Householder of v[k:] (makeHouseholder): writes ess into H col k (rows k+1..), tau, beta.
void launch_make_reflector(double* v, int k, int m, double* ess_col, double* tau, double* beta,
                           const double* partials, int nblk, cudaStream_t s);
void launch_axpby(int n, double a, const double* x, double b, double* y, cudaStream_t s);  // y = a x + b y
void launch_sub(int n, const double* a, const double* b, double* y, cudaStream_t s);          // y = a - b
int reduce_blocks();
// Loads the Krylov kernels above on the current device (once per device), so
// that a later launch does not load module code lazily.
void prepare_krylov_kernels();

// Sets the shared-memory opt-ins of the kernels (once per process and type);
// called when a handle is created, outside any stream capture.
template <class T>
void prepare_kernels();

}  // namespace spq
