// Device Krylov drivers (src/is.cpp) on top of an engine's preconditioner.
#pragma once
#include "engine.hpp"

namespace spq {

// CSR matrix resident in device memory (FP64).
struct DevCsr {
    int m = 0, n = 0;
    const int* rp = nullptr;
    const int* ci = nullptr;
    const double* v = nullptr;
};

// Householder GMRES, left preconditioned by P (src/is.cpp:94-272). x holds the
// initial guess; returns the iteration count, *res = |w(k)|/|r0|. With
// adjoint set, A is A^T (the caller passes the CSR of A^T) and the
// preconditioner is applied transposed (M^T).
int gmres_device(EngineBase& P, const DevCsr& A, const double* d_b, double* d_x, int iters, int restart, double tol,
                 double* res, long long* launches, bool adjoint = false);

// The same GMRES on a caller-provided device workspace of
// gmres_workspace_elems(m, restart) doubles; allocates no device memory.
size_t gmres_workspace_elems(int m, int restart);
int gmres_device_ws(EngineBase& P, const DevCsr& A, const double* d_b, double* d_x, int iters, int restart,
                    double tol, double* res, long long* launches, double* workspace);

// Device address and size (doubles) of the fixed no-allocation GMRES workspace
// on the current device (noalloc_scratch.cu).
cudaError_t noalloc_scratch(double** ptr, size_t* elems);

// Preconditioned CGLS on the normal equations (src/is.cpp:274-345), with the
// least-squares preconditioner P.solve_nrml_dev. A (m x n) and At (its
// transpose, n x m) as device CSR; x holds the initial guess. Returns the
// iteration count, *res = ||A^T (b - A x)|| / ||A^T b||.
int cgls_device(EngineBase& P, const DevCsr& A, const DevCsr& At, const double* d_b, double* d_x, int iters,
                double tol, double* res, long long* launches);

// ||b - A x|| / ||b|| on the device (FP64).
double residual_norm(cudaStream_t s, const DevCsr& A, const double* d_b, const double* d_x);

// Iterative refinement on the true residual: r = b - A x in FP64, GMRES on
// A d = r preconditioned by P to inner_tol, x += d, until ||b - A x|| / ||b||
// <= target or max_outer corrections. Returns the total GMRES iterations;
// *true_res is the final relative residual, *outer the corrections made.
// With adjoint set, A is A^T and the corrections use the adjoint GMRES.
int refine_device(EngineBase& P, const DevCsr& A, const double* d_b, double* d_x, double target, double inner_tol,
                  int max_outer, int iters, double* true_res, int* outer, long long* launches, bool adjoint = false);

}  // namespace spq
