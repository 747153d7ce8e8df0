/* C interface of the CPU oracle. TEST INFRASTRUCTURE ONLY.
 *
 * The oracle is a CPU restatement of the spaQR reference algorithm
 * (Abeynaya/spaQR_public): geometric nested dissection on A^T A, the cluster
 * tree (or, without coordinates, the MetisPartition steps on a given part
 * vector), Householder elimination, block scaling, RRQR sparsification (with
 * block scaling, and without it: --scale 0, square systems), merging,
 * the op-tape solves and the GMRES/CGLS drivers. Its dense kernels are the same
 * LAPACK routines the reference calls (dgeqrf, dlarft, dlarfb, dgeqp3, dormqr,
 * dtrsm, dtrsv), taken from OpenBLAS.
 *
 * PARITY UNPINNED: the reference cannot be compiled here (Eigen, PaToH and METIS
 * are absent) and ships no tests or golden vectors; its only known-answer
 * transcript (README.md:48-84) uses an input matrix that is not distributed.
 * The oracle therefore restates the algorithm from the reference sources, citing
 * file:line, and is itself the parity anchor.
 *
 * Only tests/, the smoke check and the CPU-baseline leg of bench.py use it.
 */
#ifndef SPAQR_ORACLE_H
#define SPAQR_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_tree orc_tree;

/* Tree(nlevels, skip) + set_tol/set_scale/set_order/set_square (include/tree.h:113-130). */
orc_tree* orc_create(int nlevels, int skip, double tol, int scale, float order, int square);
void orc_destroy(orc_tree* t);
const char* orc_last_error(void);
int orc_blas_threads(int nthreads); /* sets OpenBLAS threads; returns the count in use */
/* Host threads for the factorization and the solve (default 1). With n > 1
 * a square, scaled, order-1 factorization runs each level phase as
 * conflict-free waves of tasks on n threads, and the solve runs its op tape in
 * waves: bitwise the sequential results, used to time the CPU baseline. */
int orc_set_threads(orc_tree* t, int n);

/* Coordinates: d x n, column-major (set_Xcoo). */
int orc_set_coords(orc_tree* t, int d, int n, const double* X);

/* Without coordinates: the leaf part of every column (the METIS part vector of
 * MetisPartition, src/partition.cpp:374-426; METIS itself is absent, so the
 * vector is an input). numeric_fill = 1 keeps the reference's numeric fill test
 * (src/tree.cpp:857-860); 0 keeps every candidate that passes the separator
 * tests (the GPU library's rule). */
int orc_set_parts(orc_tree* t, int n, const int* parts, int numeric_fill);

/* A in CSC (sorted row indices), m >= n. */
int orc_partition(orc_tree* t, int m, int n, const int* colptr, const int* rowind, const double* val);
int orc_assemble(orc_tree* t, int m, int n, const int* colptr, const int* rowind, const double* val);
int orc_factorize(orc_tree* t);
int orc_solve(orc_tree* t, const double* b, double* x);      /* square: x ~ A^-1 b */
int orc_solve_nrml(orc_tree* t, const double* b, double* x); /* rect: x ~ (A^T A)^-1 b */

/* Permutations (length n for cperm, m for rperm). */
int orc_get_perm(orc_tree* t, int* cperm, int* rperm);
/* Symbolic/event log (see spaqr_oracle.cpp for the record layout). */
long long orc_log_size(orc_tree* t);
int orc_get_log(orc_tree* t, long long* out);
/* Bottom clusters: 9 ints each (cstart csize rstart rsize self.lvl self.sep l.lvl l.sep r.lvl r.sep) -> 10. */
int orc_num_bottom(orc_tree* t);
int orc_get_bottom(orc_tree* t, int* out);
/* Wall-clock seconds of the last partition / assemble / factorize. */
int orc_get_times(orc_tree* t, double* out3);

/* Householder GMRES (src/is.cpp:94-272) with Tree::solve as left preconditioner. */
int orc_gmres(orc_tree* t, int m, int n, const int* colptr, const int* rowind, const double* val,
              const double* b, double* x, int iters, int restart, double tol, int* its, double* res);
/* Preconditioned CGLS (src/is.cpp:274-345) with Tree::solve_nrml. */
int orc_cgls(orc_tree* t, int m, int n, const int* colptr, const int* rowind, const double* val,
             const double* b, double* x, int iters, double tol, int* its, double* res);

/* Dense LAPACK helpers used as kernel-level references by the tests. */
int orc_dgeqrf(int m, int n, double* a, int lda, double* tau);
int orc_dlarft(int m, int k, const double* v, int ldv, const double* tau, double* t, int ldt);
int orc_dlarfb_lt(int m, int n, int k, const double* v, int ldv, const double* t, int ldt, double* c, int ldc);
int orc_dgeqp3(int m, int n, double* a, int lda, int* jpvt, double* tau);
int orc_choose_rank(const double* rii, int n, double tol);

#ifdef __cplusplus
}
#endif
#endif
