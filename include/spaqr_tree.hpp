// Header-only C++ facade over the spaQR-B200 C ABI with the reference's names:
// class Tree (include/tree.h:36-152) and the gmres driver (include/is.h:14-15).
// Matrices are passed as compressed-column arrays (what Eigen::SparseMatrix<
// double, ColMajor, int> exposes through outerIndexPtr / innerIndexPtr /
// valuePtr after makeCompressed()), vectors as std::vector<double> or raw
// pointers. Errors throw spq::Error with the library's message.
#pragma once
#include <stdexcept>
#include <string>
#include <vector>

#include "spaqr_b200.h"

namespace spq {

struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

inline void check(int rc) {
    if (rc != SPQ_OK) throw Error(rc, spq_last_error());
}

// Compressed-column view of A (m x n, m >= n, sorted row indices).
struct CscView {
    int m, n;
    const int* colptr;
    const int* rowind;
    const double* val;
};

class Tree {
public:
    Tree(int nlevels, int skip) { check(spq_create(&h_, nlevels, skip)); }
    ~Tree() { spq_destroy(h_); }
    Tree(const Tree&) = delete;
    Tree& operator=(const Tree&) = delete;

    void set_tol(double tol) { check(spq_set_tol(h_, tol)); }
    void set_scale(int s) { check(spq_set_scale(h_, s)); }
    void set_order(float o) { check(spq_set_order(h_, o)); }
    void set_hsl(int h) { check(spq_set_hsl(h_, h)); }
    void set_square(int s) { check(spq_set_square(h_, s)); }
    // set_Xcoo: X is d x ncols, column-major (column j = coordinates of unknown j)
    void set_Xcoo(const double* X, int d, int ncols) { check(spq_set_coords(h_, d, ncols, X)); }
    void set_grid(int n, int d) { check(spq_set_coords_grid(h_, n, d)); }  // -n / -d
    // Without coordinates: the leaf part of every column (e.g. METIS's part
    // vector); when neither is set, partition() bisects the A^T A graph itself.
    void set_parts(const int* parts, int ncols) { check(spq_set_parts(h_, ncols, parts)); }
    void set_precision(int p) { check(spq_set_precision(h_, p)); }

    void partition(const CscView& A) {
        m_ = A.m;
        n_ = A.n;
        check(spq_partition(h_, A.m, A.n, A.colptr, A.rowind, A.val));
    }
    void assemble(const CscView& A) { check(spq_assemble(h_, A.m, A.n, A.colptr, A.rowind, A.val)); }
    int factorize() {
        check(spq_factorize(h_));
        return 0;
    }
    void solve(const std::vector<double>& b, std::vector<double>& x) const {
        x.resize(n_);
        check(spq_solve(h_, b.data(), x.data()));
    }
    void solve_nrml(const std::vector<double>& b, std::vector<double>& x) const {
        x.resize(n_);
        check(spq_solve_nrml(h_, b.data(), x.data()));
    }
    int rows() const { return m_; }
    int cols() const { return n_; }
    spq_tree* handle() const { return h_; }

private:
    spq_tree* h_ = nullptr;
    int m_ = 0, n_ = 0;
};

// gmres(A, b, x, precond, iters, restart, tol, verb) -> iterations
// (src/is.cpp:94-272). x holds the initial guess; tol is updated to the final
// preconditioned residual estimate.
inline int gmres(const CscView& A, const std::vector<double>& b, std::vector<double>& x, const Tree& precond,
                 int iters, int restart, double& tol) {
    x.resize(A.n, 0.0);
    int its = 0;
    double res = 0;
    check(spq_gmres(precond.handle(), A.m, A.n, A.colptr, A.rowind, A.val, b.data(), x.data(), iters, restart, tol,
                    &its, &res));
    tol = res;
    return its;
}

// cgls(A, b, x, precond, iters, tol, verb) -> iterations (src/is.cpp:274-345) for a
// least-squares Tree (square matching off). x holds the initial guess; tol is
// updated to ||A^T (b - A x)|| / ||A^T b||.
inline int cgls(const CscView& A, const std::vector<double>& b, std::vector<double>& x, const Tree& precond,
                int iters, double& tol) {
    x.resize(A.n, 0.0);
    int its = 0;
    double res = 0;
    check(spq_cgls(precond.handle(), A.m, A.n, A.colptr, A.rowind, A.val, b.data(), x.data(), iters, tol, &its, &res));
    tol = res;
    return its;
}

// Adjoint solve for differentiation: lambda = A^{-T} g by GMRES on A^T with the
// factors applied transposed. With x = A^{-1} b and a loss L(x): g = dL/dx,
// dL/db = lambda, dL/dA_ij = -lambda_i x_j.
inline int gmres_adjoint(const CscView& A, const std::vector<double>& g, std::vector<double>& lambda,
                         const Tree& precond, int iters, int restart, double& tol) {
    lambda.resize(A.m, 0.0);
    int its = 0;
    double res = 0;
    check(spq_gmres_adjoint(precond.handle(), A.m, A.n, A.colptr, A.rowind, A.val, g.data(), lambda.data(), iters,
                            restart, tol, &its, &res));
    tol = res;
    return its;
}

}  // namespace spq
