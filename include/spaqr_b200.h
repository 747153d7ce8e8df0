/* spaQR-B200: C ABI of the B200-native hierarchical sparsified QR.
 *
 * The entry points replace the reference's C++ surface one for one:
 *
 *   Tree(int nlevels, int skip)           include/tree.h:113-120  -> spq_create
 *   set_tol / set_scale / set_order /
 *   set_hsl / set_square / set_Xcoo       include/tree.h:124-130  -> spq_set_*
 *   void partition(SpMat& A)              include/tree.h:139      -> spq_partition
 *   void assemble(SpMat& A)               include/tree.h:140      -> spq_assemble
 *   int factorize()                       include/tree.h:143      -> spq_factorize
 *   void solve(VectorXd b, VectorXd& x)   include/tree.h:144      -> spq_solve
 *   void solve_nrml(VectorXd b, ...)      include/tree.h:147      -> spq_solve_nrml
 *   gmres(A, b, x, precond, iters,
 *         restart, tol, verb)             include/is.h:14-15      -> spq_gmres
 *   cgls(A, b, x, precond, iters, tol,..) include/is.h:18-19      -> spq_cgls
 *   ~Tree()                               src/tree.cpp:1520-1546  -> spq_destroy
 *   A = A*D*10 column normalisation       spaQR.cpp:131-147       -> spq_column_normalize
 *   linspace_nd(n, d) coordinates         src/util.cpp:852-881    -> spq_set_coords_grid
 *
 * Matrices are CSC with 0-based int32 indices and sorted row indices inside each
 * column (the layout of Eigen::SparseMatrix<double, ColMajor, int>), m >= n.
 * Every call returns an int status (SPQ_OK = 0); spq_last_error() describes the
 * last failure of the calling thread. A handle owns all of its device memory and
 * one CUDA stream; calls on one handle must not overlap.
 */
#ifndef SPAQR_B200_H
#define SPAQR_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct spq_tree spq_tree;

enum spq_status {
    SPQ_OK = 0,
    SPQ_ERR_ARG = 1,         /* invalid argument or size */
    SPQ_ERR_STATE = 2,       /* call out of order (e.g. solve before factorize) */
    SPQ_ERR_CUDA = 3,        /* CUDA runtime error (no device, launch failure, ...) */
    SPQ_ERR_NUMERIC = 4,     /* NaN/Inf or a zero pivot reported by a kernel */
    SPQ_ERR_ALLOC = 5,       /* device or host allocation failed */
    SPQ_ERR_UNSUPPORTED = 6, /* option outside the built path (e.g. --hsl 1, --scale 0 on a least-squares system) */
    SPQ_ERR_NOCONV = 7       /* Krylov solver did not reach the tolerance */
};

enum spq_precision {
    SPQ_FP64 = 0, /* plain form: factorization and solve sweeps in FP64 */
    SPQ_FP32 = 1  /* FP32 factorization and sweeps; Krylov, SpMV and residuals stay FP64 */
};

const char* spq_last_error(void);
int spq_version(void);
int spq_device_count(int* count);

/* Tree(nlevels, skip) (include/tree.h:113). */
int spq_create(spq_tree** out, int nlevels, int skip);
int spq_destroy(spq_tree* t);

int spq_set_tol(spq_tree* t, double tol);      /* -t   (default 1e-1 in the CLI; 0 in Tree) */
int spq_set_scale(spq_tree* t, int scale);     /* --scale: 1 sparsifyD after diagScale, 0 sparsify
                                                  (src/tree.cpp:887-989; square systems) */
int spq_set_order(spq_tree* t, float order);   /* --order 1 (sparsifyD) or 1.5 (sparsifyD_imp: keeps the E2 term) */
int spq_set_hsl(spq_tree* t, int hsl);         /* --hsl (0 only) */
int spq_set_square(spq_tree* t, int square);
int spq_set_coords(spq_tree* t, int d, int n, const double* X); /* d x n, column-major */
int spq_set_coords_grid(spq_tree* t, int n, int d);             /* -n/-d tensor grid */
/* Without coordinates, spq_partition orders the columns from a leaf part per
 * column (2^(nlevels-1) parts, the first cut in the highest bit), the place of
 * the METIS part vector in MetisPartition (src/partition.cpp:374-426, used by
 * Tree::partition at src/tree.cpp:610-616 when set_Xcoo was not called). The
 * separators, interfaces and permutations then follow the reference's steps.
 * spq_set_parts supplies that vector (for instance METIS's own); without it,
 * spq_partition computes it with spq_graph_parts, this library's recursive
 * bisection of the A^T A graph (host only; needs no GPU and no handle). */
int spq_set_parts(spq_tree* t, int n, const int* parts);
/* Fill rule of the ordering without coordinates. numeric = 1 (default): the
 * reference's test, a fill candidate is kept only if the coupling product
 * ||A(n, c)^T A(n, nin)|| exceeds 1e-14 (src/tree.cpp:856-859), evaluated on
 * the device with one readback per level; 0: every candidate that passes the
 * separator tests is kept (no readback). Ignored with coordinates. */
int spq_set_fill_rule(spq_tree* t, int numeric);
int spq_graph_parts(int m, int n, const int* colptr, const int* rowind, int nlevels, int* parts);
int spq_set_precision(spq_tree* t, int precision);              /* spq_precision */
int spq_set_device(spq_tree* t, int device);
int spq_set_verbose(spq_tree* t, int verbose); /* 1: per-level print lines as src/tree.cpp:1417-1434 */

int spq_partition(spq_tree* t, int m, int n, const int* colptr, const int* rowind, const double* val);
int spq_assemble(spq_tree* t, int m, int n, const int* colptr, const int* rowind, const double* val);
int spq_factorize(spq_tree* t);

/* Batched factorization of n independent handles (each partitioned and
 * assembled, on any devices). Every handle has its own CUDA stream; the
 * handles run on up to nthreads host threads (<= 0: one per handle, at most
 * 32), so the small per-wave launches of different systems share the GPU.
 * Returns the first failure (SPQ_ERR_* with the handle's index in the
 * message); the other handles are factorized regardless. */
int spq_factorize_batch(spq_tree* const* ts, int n, int nthreads);

/* Preconditioner applies on HOST buffers (b of length m for solve, n for
 * solve_nrml; x of length n). spq_solve needs a square factorization
 * (spq_set_square(t, 1)); spq_solve_nrml, M_n ~ (A^T A)^{-1}, a least-squares
 * one (square matching off; include/tree.h:147). */
int spq_solve(spq_tree* t, const double* b, double* x);
int spq_solve_nrml(spq_tree* t, const double* b, double* x);
/* Same on DEVICE buffers (FP64, on the handle's device). The first
 * application of a factorization also captures its solve graph on a host
 * thread; like every call on a handle, it returns only once no capture is in
 * flight, so the caller may synchronize the device right after it. */
int spq_solve_dev(spq_tree* t, const double* d_b, double* d_x);
int spq_solve_nrml_dev(spq_tree* t, const double* d_b, double* d_x);

/* Householder GMRES with the factorization as left preconditioner
 * (src/is.cpp:94-272). A is the matrix that was factorized (host CSC), b and x
 * host vectors (x holds the initial guess on entry). *its = iterations,
 * *res = last preconditioned residual estimate |w(k)|/|r0|. */
int spq_gmres(spq_tree* t, int m, int n, const int* colptr, const int* rowind, const double* val,
              const double* b, double* x, int iters, int restart, double tol, int* its, double* res);
/* Preconditioned CGLS on the normal equations (src/is.cpp:274-345) for a
 * least-squares factorization (square matching off, m >= n): preconditioner
 * spq_solve_nrml. x holds the initial guess; *its = iterations, *res =
 * ||A^T (b - A x)|| / ||A^T b||. */
int spq_cgls(spq_tree* t, int m, int n, const int* colptr, const int* rowind, const double* val,
             const double* b, double* x, int iters, double tol, int* its, double* res);
/* Same with device inputs: A as device CSR (m rows) and A^T as device CSR (n
 * rows; the CSC arrays of A), b (m) and x (n) device vectors. */
int spq_cgls_dev(spq_tree* t, int m, int n, const int* d_rowptr, const int* d_colind, const double* d_val,
                 const int* d_rowptr_t, const int* d_colind_t, const double* d_val_t, const double* d_b, double* d_x,
                 int iters, double tol, int* its, double* res);

/* Time-to-residual driver (the benchmark's metric): iterative refinement on
 * the true residual. Each correction solves A d = b - A x (residual in FP64)
 * with the GMRES above to inner_tol, until ||b - A x|| / ||b|| <= target or
 * max_outer corrections. With the FP64 form one correction with
 * inner_tol = target is the reference's own GMRES call; with the FP32 form the
 * outer loop is the refinement that recovers FP64 accuracy.
 * *its = total GMRES iterations, *true_res = final relative residual. */
int spq_solve_to_residual(spq_tree* t, int m, int n, const int* colptr, const int* rowind, const double* val,
                          const double* b, double* x, double target, double inner_tol, int max_outer, int iters,
                          int* its, double* true_res);
/* Same with device-resident inputs: A as CSR on the device (row pointers,
 * column indices, values; FP64), b and x device vectors. */
int spq_solve_to_residual_dev(spq_tree* t, int m, const int* d_rowptr, const int* d_colind, const double* d_val,
                              const double* d_b, double* d_x, double target, double inner_tol, int max_outer,
                              int iters, int* its, double* true_res);
/* GMRES with device-resident inputs (CSR on the device). */
int spq_gmres_dev(spq_tree* t, int m, const int* d_rowptr, const int* d_colind, const double* d_val,
                  const double* d_b, double* d_x, int iters, int restart, double tol, int* its, double* res);
/* GMRES with device-resident inputs that allocates no device memory. No
 * counterpart in the reference: it exists for callers that cannot allocate
 * once they run (e.g. a service that reserves its GPU memory at start-up, or a
 * real-time loop that must not enter the allocator). Same arguments and result
 * as spq_gmres_dev; its Krylov workspace, gmres workspace = m * (restart + 1)
 * + 5 m + a few hundred doubles, comes from one fixed 32 MiB device array
 * (4 Mi doubles) that every GPU loading this library holds until the process
 * exits; larger requests return SPQ_ERR_ARG with the sizes. Preconditions: the
 * handle is factorized and its preconditioner has been applied at least once
 * (spq_solve, spq_solve_dev or spq_gmres_dev build the solve graph), else
 * SPQ_ERR_STATE. The array's device address is looked up, and the array and
 * the Krylov kernels are loaded onto the device, when a handle binds its
 * device (spq_partition), so the call itself takes no device memory, even
 * under lazy module loading. All calls share
 * the one array: calls that overlap on the GPU (several handles, streams or
 * threads at once) race on it. The workspace is re-initialised by every call. */
int spq_gmres_dev_noalloc(spq_tree* t, int m, const int* d_rowptr, const int* d_colind, const double* d_val,
                          const double* d_b, double* d_x, int iters, int restart, double tol, int* its, double* res);
/* Adjoint (transposed) solves for differentiation: no counterpart in the
 * reference, whose Tree only applies M ~ A^{-1}. For a loss L(x) with A x = b,
 * lambda = A^{-T} dL/dx gives dL/db = lambda and dL/dA_ij = -lambda_i x_j on the
 * pattern of A.
 * spq_solve_adjoint applies y = M^T g with the same factors (R^T solves
 * first, then Q: the solve sweeps transposed and in reverse order); g has
 * length n, y length m. */
int spq_solve_adjoint(spq_tree* t, const double* g, double* y);
int spq_solve_adjoint_dev(spq_tree* t, const double* d_g, double* d_y);
/* GMRES on A^T lambda = g preconditioned by M^T (the GMRES of spq_gmres run on
 * the transpose). A is the factorized matrix as host CSC (which is A^T as CSR);
 * lambda holds the initial guess on entry. */
int spq_gmres_adjoint(spq_tree* t, int m, int n, const int* colptr, const int* rowind, const double* val,
                      const double* g, double* lambda, int iters, int restart, double tol, int* its, double* res);
/* Same on device buffers; d_rowptr_t / d_colind_t / d_val_t are the CSR of A^T
 * (equivalently the CSC of A). */
int spq_gmres_adjoint_dev(spq_tree* t, int n, const int* d_rowptr_t, const int* d_colind_t, const double* d_val_t,
                          const double* d_g, double* d_lambda, int iters, int restart, double tol, int* its,
                          double* res);

/* Time-to-residual driver of the adjoint: iterative refinement on the true
 * residual g - A^T lambda with adjoint GMRES corrections (the transposed
 * spq_solve_to_residual_dev); CSR of A^T on the device. */
int spq_solve_to_residual_adjoint_dev(spq_tree* t, int n, const int* d_rowptr_t, const int* d_colind_t,
                                      const double* d_val_t, const double* d_g, double* d_lambda, double target,
                                      double inner_tol, int max_outer, int iters, int* its, double* true_res);

/* Kernel launches issued by the last spq_factorize and by Krylov calls since
 * the handle was created; solve_graph_kernels = kernels in one preconditioner
 * application (one CUDA graph launch), applications = graph launches so far. */
int spq_get_launches(spq_tree* t, long long* factorize, long long* krylov, long long* solve_graph_kernels,
                     long long* applications);

/* Per-kernel timing (off by default): with profile = 1 every launch of the
 * handle is bracketed by CUDA events on its stream. spq_get_kernel_stats
 * returns, for kernel family f (0 copy, 1 panel QR, 2 trailing update, 3 trsm,
 * 4 truncated RRQR, 5 sparsification write-back, 6 assembly scatter,
 * 7 preconditioner application), out[0..3] = launches, total ms, algorithmic
 * flops, algorithmic bytes. spq_reset_kernel_stats clears the counters.
 * profile = 2 also prints, when the counters are read, one line per launch to
 * stderr: "timeline <family> <start ms> <duration ms> L<level> P<phase>", the
 * start measured from the first launch since the previous read, for locating
 * the stretches where the device waits for the host. */
int spq_set_profile(spq_tree* t, int profile);
int spq_get_kernel_stats(spq_tree* t, int family, double* out4);
int spq_reset_kernel_stats(spq_tree* t);
/* Diagnostic: runs one preconditioner application outside its CUDA graph and
 * times every sweep wave. out (capacity 7 * cap) receives, per wave (forward
 * then backward): [ms, ops, shared vector length, factor words read, kind of
 * the largest op (0 Q apply, 1 triangular), its rows, its columns (Q apply)
 * or neighbour blocks (triangular)]; *nwaves = waves. */
int spq_profile_solve_waves(spq_tree* t, double* out, int cap, int* nwaves);
/* The CUDA stream (cudaStream_t) the handle issues its work on; valid after
 * spq_assemble. */
int spq_get_stream(spq_tree* t, void** stream);

/* Introspection: permutations, event log (records of 8 int64, layout documented
 * in the package's host source), nnz counters, per-level phase times. */
int spq_get_perm(spq_tree* t, int* cperm, int* rperm);
int spq_log_size(spq_tree* t, long long* n);
int spq_get_log(spq_tree* t, long long* out);
int spq_num_bottom(spq_tree* t, int* n);
int spq_get_bottom(spq_tree* t, int* out); /* 10 ints per bottom cluster */
/* times[0..3] = partition, assemble, factorize, last solve (seconds);
 * counters[0..3] = nnzA, nnzR, nnzH, nnzQ; counters[4] = kernel launches of the
 * last factorize; counters[5] = kernel launches of the last solve;
 * counters[6] = device bytes in use; counters[7] = preconditioner applications. */
int spq_get_stats(spq_tree* t, double* times, long long* counters);
/* Per-level factorization phase times in ms (6 per level: fill, elmn, shift,
 * scale, sprsfy, merge), as printed by src/tree.cpp:1417-1426. */
int spq_get_level_times(spq_tree* t, double* out);
/* Host side of the last factorize in seconds: out11 = [wall time, waits for
 * the device readbacks (ranks, row norms), device allocations of the arenas,
 * scratch growth, solve-plan build, then the host time of each level phase
 * summed over the levels: fill, elimination, row shift, scaling,
 * sparsification, merge (waits and allocations included)]. */
int spq_get_host_times(spq_tree* t, double* out11);
/* Device memory of destroyed handles stays cached in a per-device pool for the
 * next handle (no allocation cost on refactorization); this returns the
 * cached, unused part to the device. */
int spq_trim_memory(void);
/* Bytes of the device's memory pool in use by live buffers and held by the
 * pool (in use plus cached), for memory accounting; 0 and 0 before the first
 * handle binds the device. No counterpart in the reference (Eigen allocates on
 * the host heap). */
int spq_pool_memory(int device, unsigned long long* used, unsigned long long* reserved);

/* Autotuner of launch shapes that do not change results (today the cluster
 * size of the blocked RRQR of sparsifyD, src/tree.cpp:1022-1049, whose output
 * is bitwise the same for every size). No counterpart in the reference, which
 * has no launch shapes. Process-wide, shared by all handles.
 *   mode 0: off, the built-in default shape;
 *   mode 1: online (default), each fitting shape is timed twice per size
 *           bucket as factorizations run, then the fastest is used;
 *   mode 2: frozen, only the table (e.g. loaded from a file) is used.
 * save/load write/read a text table (one line per bucket and shape); load
 * merges into the current table. */
int spq_autotune_set_mode(int mode);
int spq_autotune_get(int* mode, int* entries, int* pending); /* pending: timings still to explore */
int spq_autotune_reset(void);
int spq_autotune_save(const char* path);
int spq_autotune_load(const char* path);

/* A <- A * diag(1/||A_j||) * 10, in place on val (spaQR.cpp:131-147). */
int spq_column_normalize(int m, int n, const int* colptr, const int* rowind, double* val);

#ifdef __cplusplus
}
#endif
#endif
