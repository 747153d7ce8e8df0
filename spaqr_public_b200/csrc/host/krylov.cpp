// Householder GMRES with the spaQR factorization as left preconditioner
// (src/is.cpp:94-272), on device vectors in FP64.
//
// The Arnoldi basis is kept as Householder reflectors in the columns of H
// (m x (restart+1), column-major, device). Reflector applications, SpMV and
// the preconditioner run on the GPU; the (k+1)-long head of the rotated
// vector, the Givens rotations and the small triangular solve run on the host,
// which also reads the residual estimate to decide convergence each iteration.
#include "krylov.hpp"

#include <cfloat>
#include <cmath>
#include <vector>

#include "../kernels/kernels.hpp"

namespace spq {
namespace {

// Device vector from the device's retained memory pool, allocated and freed
// in the order of the handle's stream.
struct DevVec {
    double* p = nullptr;
    bool owned = false;
    cudaStream_t s = nullptr;
    ~DevVec() {
        if (p && owned) cudaFreeAsync(p, s);
    }
    void alloc(size_t n, cudaStream_t st) {
        if (p && owned) cudaFreeAsync(p, s);
        s = st;
        int dev = 0;
        cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
        p = static_cast<double*>(
            pool_alloc(device_pool(dev), std::max<size_t>(n, 1) * sizeof(double), st, "krylov allocation"));
        owned = true;
    }
    // Points at caller-provided device memory (never freed here).
    void borrow(double* q) {
        p = q;
        owned = false;
    }
};

// Givens rotation (c, s) with [c -s; s c] [p; q] = [r; 0].
void make_givens(double p, double q, double& c, double& s) {
    if (q == 0) {
        c = p < 0 ? -1 : 1;
        s = 0;
    } else if (p == 0) {
        c = 0;
        s = q < 0 ? 1 : -1;
    } else if (std::abs(p) > std::abs(q)) {
        double t = q / p, u = std::sqrt(1 + t * t);
        if (p < 0) u = -u;
        c = 1 / u;
        s = -t * c;
    } else {
        double t = p / q, u = std::sqrt(1 + t * t);
        if (q < 0) u = -u;
        s = -1 / u;
        c = -t * s;
    }
}
inline void rot(double& a, double& b, double c, double s) {
    double x = a, y = b;
    a = c * x - s * y;
    b = s * x + c * y;
}

class Gmres {
public:
    Gmres(EngineBase& P, const DevCsr& A, int restart) : P_(P), A_(A), m_(A.m), restart_(restart) {
        s_ = P.stream();
        nblk_ = reduce_blocks();
        p0_.alloc(m_, s_);
        r0_.alloc(m_, s_);
        t_.alloc(m_, s_);
        v_.alloc(m_, s_);
        xnew_.alloc(m_, s_);
        part_.alloc(nblk_ + 1, s_);
        scal_.alloc(2 * (size_t(restart) + 1) + 4, s_);
        H_.alloc(size_t(m_) * (size_t(restart) + 1), s_);
        hpart_.resize(nblk_);
    }
    // Same driver on a caller-provided workspace of workspace_elems(m, restart)
    // doubles; nothing is allocated on the device.
    Gmres(EngineBase& P, const DevCsr& A, int restart, double* ws) : P_(P), A_(A), m_(A.m), restart_(restart) {
        s_ = P.stream();
        nblk_ = reduce_blocks();
        double* q = ws;
        auto take = [&q](DevVec& v, size_t n) {
            v.borrow(q);
            q += (std::max<size_t>(n, 1) + 31) & ~size_t(31);  // 256-byte steps
        };
        take(p0_, m_);
        take(r0_, m_);
        take(t_, m_);
        take(v_, m_);
        take(xnew_, m_);
        take(part_, nblk_ + 1);
        take(scal_, 2 * (size_t(restart) + 1) + 4);
        take(H_, size_t(m_) * (size_t(restart) + 1));
        hpart_.resize(nblk_);
    }
    static size_t workspace_elems(int m, int restart) {
        auto r = [](size_t n) { return (std::max<size_t>(n, 1) + 31) & ~size_t(31); };
        // sizes in size_t: restart near INT_MAX must not overflow before the
        // caller compares the result with its workspace
        const size_t rs = size_t(restart) + 1;
        return 5 * r(size_t(m)) + r(size_t(reduce_blocks()) + 1) + r(2 * rs + 4) + r(size_t(m) * rs);
    }

    // Sum of a reduction's partials on the host, in fixed order.
    double host_sum() {
        cuda_check(cudaMemcpyAsync(hpart_.data(), part_.p, nblk_ * sizeof(double), cudaMemcpyDeviceToHost, s_),
                   "partials");
        cuda_check(cudaStreamSynchronize(s_), "partials sync");
        double s = 0;
        for (double v : hpart_) s += v;
        return s;
    }
    double* col(int j) { return H_.p + (size_t)j * m_; }
    double* tau(int j) { return scal_.p + j; }
    double* beta() { return scal_.p + 2 * (restart_ + 1); }

    // v[i:] <- H_i v[i:]
    void reflect(int i, double* v) {
        launch_dot_partials(col(i), v, i + 1, m_, part_.p, nblk_, s_, v + i);
        launch_apply_reflector(col(i) + i + 1, tau(i), v, i, m_, part_.p, nblk_, s_);
        launches_ += 2;
    }
    // Builds H_k from v[k:] (ess into column k), returns beta.
    double make(int k, double* v) {
        launch_dot_partials(v, nullptr, k + 1, m_, part_.p, nblk_, s_);
        launch_make_reflector(v, k, m_, col(k) + k + 1, tau(k), beta(), part_.p, nblk_, s_);
        launches_ += 2;
        double b;
        cuda_check(cudaMemcpyAsync(&b, beta(), sizeof(double), cudaMemcpyDeviceToHost, s_), "beta");
        cuda_check(cudaStreamSynchronize(s_), "beta sync");
        return b;
    }
    void residual(const double* b, const double* x, double* out) {  // out = b - A x
        launch_spmv_csr(m_, A_.rp, A_.ci, A_.v, x, t_.p, s_);
        launch_sub(m_, b, t_.p, out, s_);
        launches_ += 2;
    }

    int run(const double* b, double* x, int iters, double tol, double* res) {
        const int m = m_, restart = restart_;
        launch_dot_partials(b, nullptr, 0, m, part_.p, nblk_, s_);
        ++launches_;
        if (std::sqrt(host_sum()) <= DBL_MIN) {
            cuda_check(cudaMemsetAsync(x, 0, sizeof(double) * m, s_), "x zero");
            *res = 0;
            return 0;
        }
        const int maxIters = iters;
        int it = 0;
        residual(b, x, p0_.p);
        precond(p0_.p, r0_.p);
        launch_dot_partials(r0_.p, nullptr, 0, m, part_.p, nblk_, s_);
        ++launches_;
        const double r0Norm = std::sqrt(host_sum());
        if (r0Norm == 0) {
            *res = 0;
            return 0;
        }
        cuda_check(cudaMemsetAsync(H_.p, 0, sizeof(double) * (size_t)m * (restart + 1), s_), "H zero");
        cuda_check(cudaMemsetAsync(scal_.p, 0, sizeof(double) * (2 * (restart + 1) + 4), s_), "tau zero");
        std::vector<double> w(restart + 1, 0.0), Hs((size_t)(restart + 1) * (restart + 1), 0.0);
        std::vector<double> Gc(restart, 0.0), Gs(restart, 0.0), vh(restart + 2, 0.0);
        auto hs = [&](int i, int j) -> double& { return Hs[(size_t)j * (restart + 1) + i]; };
        w[0] = make(0, r0_.p);
        double tol_error = 0;
        const double one = 1.0;
        for (int k = 1; k <= restart; ++k) {
            ++it;
            cuda_check(cudaMemsetAsync(v_.p, 0, sizeof(double) * m, s_), "v zero");
            cuda_check(cudaMemcpyAsync(v_.p + (k - 1), &one, sizeof(double), cudaMemcpyHostToDevice, s_), "v unit");
            for (int i = k - 1; i >= 0; --i) reflect(i, v_.p);
            launch_spmv_csr(m, A_.rp, A_.ci, A_.v, v_.p, t_.p, s_);
            ++launches_;
            precond(t_.p, v_.p);
            for (int i = 0; i < k; ++i) reflect(i, v_.p);
            if (k < m) {
                launch_dot_partials(v_.p, nullptr, k, m, part_.p, nblk_, s_);
                ++launches_;
                if (std::sqrt(host_sum()) != 0.0) {
                    make(k, v_.p);
                    reflect(k, v_.p);
                }
            }
            const int nh = std::min(k + 1, m);
            cuda_check(cudaMemcpyAsync(vh.data(), v_.p, sizeof(double) * nh, cudaMemcpyDeviceToHost, s_), "v head");
            cuda_check(cudaStreamSynchronize(s_), "v head sync");
            for (int i = 0; i < k - 1; ++i) rot(vh[i], vh[i + 1], Gc[i], Gs[i]);
            if (k < m && vh[k] != 0) {
                make_givens(vh[k - 1], vh[k], Gc[k - 1], Gs[k - 1]);
                rot(vh[k - 1], vh[k], Gc[k - 1], Gs[k - 1]);
                rot(w[k - 1], w[k], Gc[k - 1], Gs[k - 1]);
            }
            for (int i = 0; i < k; ++i) hs(i, k - 1) = vh[i];
            tol_error = std::abs(w[k]) / r0Norm;
            const bool stop = (k == m || tol_error < tol || it == maxIters);
            if (stop || k == restart) {
                std::vector<double> y(w.begin(), w.begin() + k);
                for (int i = k - 1; i >= 0; --i) {
                    double s = y[i];
                    for (int j = i + 1; j < k; ++j) s -= hs(i, j) * y[j];
                    y[i] = s / hs(i, i);
                }
                cuda_check(cudaMemsetAsync(xnew_.p, 0, sizeof(double) * m, s_), "xnew zero");
                cuda_check(cudaMemcpyAsync(t_.p, y.data(), sizeof(double) * k, cudaMemcpyHostToDevice, s_), "y");
                for (int i = k - 1; i >= 0; --i) {
                    launch_axpby(1, 1.0, t_.p + i, 1.0, xnew_.p + i, s_);
                    ++launches_;
                    reflect(i, xnew_.p);
                }
                launch_axpby(m, 1.0, xnew_.p, 1.0, x, s_);
                ++launches_;
                if (stop) {
                    *res = tol_error;
                    cuda_check(cudaStreamSynchronize(s_), "gmres end");
                    return it;
                }
                k = 0;
                residual(b, x, p0_.p);
                precond(p0_.p, r0_.p);
                cuda_check(cudaMemsetAsync(H_.p, 0, sizeof(double) * (size_t)m * (restart + 1), s_), "H zero");
                cuda_check(cudaMemsetAsync(scal_.p, 0, sizeof(double) * (2 * (restart + 1) + 4), s_), "tau");
                std::fill(w.begin(), w.end(), 0.0);
                std::fill(Hs.begin(), Hs.end(), 0.0);
                w[0] = make(0, r0_.p);
            }
        }
        *res = tol_error;
        return it;
    }
    long long launches_ = 0;
    bool adjoint_ = false;  // A is A^T and the preconditioner is applied transposed

private:
    // M r, or M^T r in an adjoint solve
    void precond(const double* in, double* out) {
        if (adjoint_)
            P_.solve_adjoint_dev(in, out);
        else
            P_.solve_dev(in, out);
    }

    EngineBase& P_;
    DevCsr A_;
    int m_, restart_, nblk_;
    cudaStream_t s_;
    DevVec p0_, r0_, t_, v_, xnew_, part_, scal_, H_;
    std::vector<double> hpart_;
};

}  // namespace

int gmres_device(EngineBase& P, const DevCsr& A, const double* d_b, double* d_x, int iters, int restart, double tol,
                 double* res, long long* launches, bool adjoint) {
    if (restart < 1) restart = 1;
    // the workspace (m x (restart + 1) Krylov basis) is the handle's scratch
    // buffer, which persists across solves and handles: no allocation per call
    Gmres g(P, A, restart, P.krylov_workspace(Gmres::workspace_elems(A.m, restart)));
    g.adjoint_ = adjoint;
    int it = g.run(d_b, d_x, iters, tol, res);
    if (launches) *launches = g.launches_;
    return it;
}

size_t gmres_workspace_elems(int m, int restart) { return Gmres::workspace_elems(m, restart < 1 ? 1 : restart); }

int gmres_device_ws(EngineBase& P, const DevCsr& A, const double* d_b, double* d_x, int iters, int restart,
                    double tol, double* res, long long* launches, double* workspace) {
    if (restart < 1) restart = 1;
    Gmres g(P, A, restart, workspace);
    int it = g.run(d_b, d_x, iters, tol, res);
    if (launches) *launches = g.launches_;
    return it;
}

int refine_device(EngineBase& P, const DevCsr& A, const double* d_b, double* d_x, double target, double inner_tol,
                  int max_outer, int iters, double* true_res, int* outer, long long* launches, bool adjoint) {
    cudaStream_t s = P.stream();
    DevVec r, d;
    r.alloc(A.m, s);
    d.alloc(A.n, s);
    int total = 0, k = 0;
    long long l = 0;
    double rel = residual_norm(s, A, d_b, d_x);
    l += 6;
    while (rel > target && k < max_outer) {
        launch_spmv_csr(A.m, A.rp, A.ci, A.v, d_x, r.p, s);
        launch_sub(A.m, d_b, r.p, r.p, s);
        cuda_check(cudaMemsetAsync(d.p, 0, sizeof(double) * A.n, s), "refine zero");
        double res = 0;
        long long gl = 0;
        total += gmres_device(P, A, r.p, d.p, iters, iters, inner_tol, &res, &gl, adjoint);
        launch_axpby(A.n, 1.0, d.p, 1.0, d_x, s);
        l += gl + 3;
        ++k;
        rel = residual_norm(s, A, d_b, d_x);
        l += 6;
    }
    if (true_res) *true_res = rel;
    if (outer) *outer = k;
    if (launches) *launches = l;
    return total;
}

int cgls_device(EngineBase& P, const DevCsr& A, const DevCsr& At, const double* d_b, double* d_x, int iters,
                double tol, double* res, long long* launches) {
    cudaStream_t s = P.stream();
    const int m = A.m, n = A.n;
    const int nblk = reduce_blocks();
    DevVec residual, nr, tmp, p, z, atb, part;
    residual.alloc(m, s);
    nr.alloc(n, s);
    tmp.alloc(m, s);
    p.alloc(n, s);
    z.alloc(n, s);
    atb.alloc(n, s);
    part.alloc(nblk, s);
    std::vector<double> h(nblk);
    long long l = 0;
    // deterministic inner product: fixed block partials summed in order on the host
    auto dot = [&](const double* a, const double* b, int len) {
        launch_dot_partials(a, b, 0, len, part.p, nblk, s, nullptr);
        ++l;
        cuda_check(cudaMemcpyAsync(h.data(), part.p, nblk * sizeof(double), cudaMemcpyDeviceToHost, s), "cgls dot");
        cuda_check(cudaStreamSynchronize(s), "cgls dot");
        double acc = 0;
        for (double v : h) acc += v;
        return acc;
    };
    auto spmv = [&](const DevCsr& M, const double* x, double* y) {
        launch_spmv_csr(M.m, M.rp, M.ci, M.v, x, y, s);
        ++l;
    };
    spmv(A, d_x, tmp.p);
    launch_sub(m, d_b, tmp.p, residual.p, s);
    spmv(At, residual.p, nr.p);
    spmv(At, d_b, atb.p);
    l += 1;
    const double rhs2 = dot(atb.p, atb.p, n);
    if (rhs2 == 0) {
        cuda_check(cudaMemsetAsync(d_x, 0, sizeof(double) * n, s), "cgls zero");
        *res = 0;
        if (launches) *launches = l;
        return 0;
    }
    const double threshold = tol * tol * rhs2;
    double rn2 = dot(nr.p, nr.p, n);
    if (rn2 < threshold) {
        *res = std::sqrt(rn2 / rhs2);
        if (launches) *launches = l;
        return 0;
    }
    P.solve_nrml_dev(nr.p, p.p);
    double abs_new = dot(nr.p, p.p, n);
    int i = 0;
    while (i < iters) {
        spmv(A, p.p, tmp.p);
        const double alpha = abs_new / dot(tmp.p, tmp.p, m);
        launch_axpby(n, alpha, p.p, 1.0, d_x, s);
        launch_axpby(m, -alpha, tmp.p, 1.0, residual.p, s);
        l += 2;
        spmv(At, residual.p, nr.p);
        rn2 = dot(nr.p, nr.p, n);
        if (rn2 < threshold) break;
        P.solve_nrml_dev(nr.p, z.p);
        const double abs_old = abs_new;
        abs_new = dot(nr.p, z.p, n);
        const double beta = abs_new / abs_old;
        launch_axpby(n, 1.0, z.p, beta, p.p, s);
        ++l;
        ++i;
    }
    *res = std::sqrt(rn2 / rhs2);
    if (launches) *launches = l;
    return i;
}

double residual_norm(cudaStream_t s, const DevCsr& A, const double* d_b, const double* d_x) {
    DevVec t, part;
    t.alloc(A.m, s);
    const int nblk = reduce_blocks();
    part.alloc(nblk, s);
    std::vector<double> h(nblk);
    auto sum = [&]() {
        cuda_check(cudaMemcpyAsync(h.data(), part.p, nblk * sizeof(double), cudaMemcpyDeviceToHost, s), "res");
        cuda_check(cudaStreamSynchronize(s), "res sync");
        double a = 0;
        for (double v : h) a += v;
        return a;
    };
    launch_spmv_csr(A.m, A.rp, A.ci, A.v, d_x, t.p, s);
    launch_sub(A.m, d_b, t.p, t.p, s);
    launch_dot_partials(t.p, nullptr, 0, A.m, part.p, nblk, s);
    const double rn = std::sqrt(sum());
    launch_dot_partials(d_b, nullptr, 0, A.m, part.p, nblk, s);
    const double bn = std::sqrt(sum());
    return bn > 0 ? rn / bn : rn;
}

}  // namespace spq
