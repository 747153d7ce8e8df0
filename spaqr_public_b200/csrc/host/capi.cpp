// C ABI of spaQR-B200 (declared in include/spaqr_b200.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <thread>
#include <memory>
#include <new>
#include <string>
#include <vector>

#include "../../../include/spaqr_b200.h"
#include "autotune.hpp"
#include "engine.hpp"
#include "krylov.hpp"

using namespace spq;

struct spq_tree {
    Config cfg;
    int precision = SPQ_FP64;
    std::unique_ptr<EngineBase> eng;
    int state = 0;  // 0 created, 1 partitioned, 2 assembled, 3 factorized
    long long launches_krylov = 0;
};

namespace {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
    g_err = msg;
    return code;
}

template <class F>
int guard(F&& f) {
    try {
        return f();
    } catch (const CudaError& e) {
        return fail(SPQ_ERR_CUDA, e.what());
    } catch (const std::bad_alloc&) {
        return fail(SPQ_ERR_ALLOC, "host allocation failed");
    } catch (const std::invalid_argument& e) {
        return fail(SPQ_ERR_UNSUPPORTED, e.what());
    } catch (const std::logic_error& e) {
        return fail(SPQ_ERR_STATE, e.what());
    } catch (const std::exception& e) {
        return fail(SPQ_ERR_NUMERIC, e.what());
    }
}

// guard() for calls on a handle whose device is open: the calling thread's
// current device becomes the handle's, so a handle may be used from any
// thread (batches run one handle per thread).
template <class F>
int guard_on(spq_tree* t, F&& f) {
    if (t && t->eng && t->state >= 2) {
        cudaError_t e = cudaSetDevice(t->cfg.device);
        if (e != cudaSuccess) return fail(SPQ_ERR_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
    }
    const int rc = guard(std::forward<F>(f));
    // The first preconditioner application leaves a host thread capturing the
    // solve graph (it overlaps the applications that follow inside the call).
    // The capture ends before control returns: while a stream is capturing, a
    // caller's cudaDeviceSynchronize (torch.cuda.synchronize) fails with
    // cudaErrorStreamCaptureUnsupported. An error of the call is kept.
    if (t && t->eng) {
        const std::string err = g_err;
        const int rs = guard([&] {
            t->eng->solve_ready();
            return SPQ_OK;
        });
        if (rc != SPQ_OK) {
            g_err = err;
            return rc;
        }
        return rs;
    }
    return rc;
}

int check_csc(int m, int n, const int* cp, const int* ri, const double* va, bool need_values = true) {
    if (m <= 0 || n <= 0 || !cp || (!ri && cp[n] > 0) || (need_values && !va && cp[n] > 0))
        return fail(SPQ_ERR_ARG, "invalid CSC matrix");
    if (cp[0] != 0) return fail(SPQ_ERR_ARG, "colptr[0] must be 0");
    for (int j = 0; j < n; ++j) {
        if (cp[j + 1] < cp[j]) return fail(SPQ_ERR_ARG, "colptr must be non-decreasing");
        for (int q = cp[j]; q < cp[j + 1]; ++q) {
            if (ri[q] < 0 || ri[q] >= m) return fail(SPQ_ERR_ARG, "row index out of range");
            if (q > cp[j] && ri[q] <= ri[q - 1]) return fail(SPQ_ERR_ARG, "row indices must be strictly increasing");
        }
    }
    return SPQ_OK;
}

// Device buffers of one host-API call, from the device's retained memory pool
// in the order of the handle's stream (no cudaMalloc / cudaFree, which map
// pages and synchronise the device, on every solve).
struct DevBuf {
    void* p = nullptr;
    cudaStream_t s = nullptr;
    template <class U>
    U* get(size_t n, cudaStream_t st) {
        int dev = 0;
        cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
        s = st;
        p = pool_alloc(device_pool(dev), std::max<size_t>(n, 1) * sizeof(U), st, "host-API buffer");
        return static_cast<U*>(p);
    }
    ~DevBuf() {
        if (p) cudaFreeAsync(p, s);
    }
};
struct DevCsrOwned {
    DevBuf rp, ci, v;
};

// Host CSC -> device CSR (rows of A with sorted column indices).
void upload_csr(const Csc& A, DevCsrOwned& o, DevCsr& d, cudaStream_t s) {
    Csc T = csc_transpose(A);  // column r of T = row r of A
    int* rp = o.rp.get<int>(T.p.size(), s);
    int* ci = o.ci.get<int>(T.i.size(), s);
    double* va = o.v.get<double>(T.v.size(), s);
    cuda_check(cudaMemcpyAsync(rp, T.p.data(), sizeof(int) * T.p.size(), cudaMemcpyHostToDevice, s), "csr up");
    cuda_check(cudaMemcpyAsync(ci, T.i.data(), sizeof(int) * T.i.size(), cudaMemcpyHostToDevice, s), "csr up");
    cuda_check(cudaMemcpyAsync(va, T.v.data(), sizeof(double) * T.v.size(), cudaMemcpyHostToDevice, s), "csr up");
    // the host arrays are released when this returns: the copies must have read them
    cuda_check(cudaStreamSynchronize(s), "csr up");
    d.m = A.m;
    d.n = A.n;
    d.rp = rp;
    d.ci = ci;
    d.v = va;
}

}  // namespace

extern "C" {

const char* spq_last_error(void) { return g_err.c_str(); }
int spq_version(void) { return 1; }

int spq_device_count(int* count) {
    if (!count) return fail(SPQ_ERR_ARG, "null count");
    cudaError_t e = cudaGetDeviceCount(count);
    if (e != cudaSuccess) {
        *count = 0;
        return fail(SPQ_ERR_CUDA, cudaGetErrorString(e));
    }
    return SPQ_OK;
}

int spq_create(spq_tree** out, int nlevels, int skip) {
    if (!out) return fail(SPQ_ERR_ARG, "null handle pointer");
    if (nlevels < 1) return fail(SPQ_ERR_ARG, "nlevels must be >= 1");
    if (skip < 0) return fail(SPQ_ERR_ARG, "skip must be >= 0");
    spq_tree* t = new (std::nothrow) spq_tree;
    if (!t) return fail(SPQ_ERR_ALLOC, "handle allocation failed");
    t->cfg.nlevels = nlevels;
    t->cfg.skip = skip;
    *out = t;
    return SPQ_OK;
}

int spq_destroy(spq_tree* t) {
    delete t;
    return SPQ_OK;
}

#define SPQ_SETTER_GUARD                                                          \
    if (!t) return fail(SPQ_ERR_ARG, "null handle");                             \
    if (t->state != 0) return fail(SPQ_ERR_STATE, "options must be set before partition");

int spq_set_tol(spq_tree* t, double tol) {
    SPQ_SETTER_GUARD
    if (!(tol >= 0)) return fail(SPQ_ERR_ARG, "tol must be >= 0");
    t->cfg.tol = tol;
    return SPQ_OK;
}
int spq_set_scale(spq_tree* t, int scale) {
    SPQ_SETTER_GUARD
    t->cfg.scale = scale;
    return SPQ_OK;
}
int spq_set_order(spq_tree* t, float order) {
    SPQ_SETTER_GUARD
    if (order != 1.0f && order != 1.5f) return fail(SPQ_ERR_ARG, "order must be 1 or 1.5");
    t->cfg.order = order;
    return SPQ_OK;
}
int spq_set_hsl(spq_tree* t, int hsl) {
    SPQ_SETTER_GUARD
    if (hsl) return fail(SPQ_ERR_UNSUPPORTED, "HSL bipartite matching is not available");
    t->cfg.hsl = hsl;
    return SPQ_OK;
}
int spq_set_square(spq_tree* t, int square) {
    SPQ_SETTER_GUARD
    t->cfg.square = square;
    return SPQ_OK;
}
int spq_set_coords(spq_tree* t, int d, int n, const double* X) {
    SPQ_SETTER_GUARD
    if (d < 1 || n < 1 || !X) return fail(SPQ_ERR_ARG, "invalid coordinates");
    t->cfg.d = d;
    t->cfg.X.assign(X, X + (size_t)d * n);
    return SPQ_OK;
}
int spq_set_coords_grid(spq_tree* t, int n, int d) {
    SPQ_SETTER_GUARD
    if (n < 1 || d < 1 || d > 3) return fail(SPQ_ERR_ARG, "grid coordinates need n >= 1 and 1 <= d <= 3");
    // linspace_nd (src/util.cpp:852-881): lexicographic, first coordinate slowest
    const size_t N = (size_t)std::llround(std::pow((double)n, d));
    t->cfg.d = d;
    t->cfg.X.assign(N * d, 0.0);
    for (size_t id = 0; id < N; ++id) {
        size_t r = id;
        for (int a = d - 1; a >= 0; --a) {
            t->cfg.X[id * d + a] = (double)(r % n);
            r /= n;
        }
    }
    return SPQ_OK;
}
int spq_set_parts(spq_tree* t, int n, const int* parts) {
    SPQ_SETTER_GUARD
    if (n < 1 || !parts) return fail(SPQ_ERR_ARG, "invalid part vector");
    const int nleaves = t->cfg.nlevels >= 2 ? 1 << (t->cfg.nlevels - 1) : 1;
    for (int i = 0; i < n; ++i)
        if (parts[i] < 0 || parts[i] >= nleaves) return fail(SPQ_ERR_ARG, "part index out of range for nlevels");
    t->cfg.parts.assign(parts, parts + n);
    return SPQ_OK;
}
int spq_set_fill_rule(spq_tree* t, int numeric) {
    SPQ_SETTER_GUARD
    if (numeric != 0 && numeric != 1) return fail(SPQ_ERR_ARG, "fill rule must be 0 or 1");
    t->cfg.numeric_fill = numeric;
    return SPQ_OK;
}
int spq_graph_parts(int m, int n, const int* cp, const int* ri, int nlevels, int* parts) {
    int rc = check_csc(m, n, cp, ri, nullptr, false);
    if (rc) return rc;
    if (nlevels < 1 || nlevels > 30 || !parts) return fail(SPQ_ERR_ARG, "need 1 <= nlevels <= 30 and an output");
    return guard([&] {
        Csc A;
        A.m = m;
        A.n = n;
        A.p.assign(cp, cp + n + 1);
        A.i.assign(ri, ri + cp[n]);
        A.v.assign((size_t)cp[n], 0.0);  // pattern only; the values are not read
        const std::vector<int> p = graph_bisection(A, nlevels);
        std::copy(p.begin(), p.end(), parts);
        return SPQ_OK;
    });
}
int spq_set_precision(spq_tree* t, int precision) {
    SPQ_SETTER_GUARD
    if (precision != SPQ_FP64 && precision != SPQ_FP32) return fail(SPQ_ERR_ARG, "unknown precision");
    t->precision = precision;
    return SPQ_OK;
}
int spq_set_device(spq_tree* t, int device) {
    SPQ_SETTER_GUARD
    t->cfg.device = device;
    return SPQ_OK;
}
int spq_set_verbose(spq_tree* t, int verbose) {
    if (!t) return fail(SPQ_ERR_ARG, "null handle");
    t->cfg.verbose = verbose;
    return SPQ_OK;
}

int spq_partition(spq_tree* t, int m, int n, const int* cp, const int* ri, const double* va) {
    if (!t) return fail(SPQ_ERR_ARG, "null handle");
    if (t->state != 0) return fail(SPQ_ERR_STATE, "partition called twice");
    int rc = check_csc(m, n, cp, ri, va);
    if (rc) return rc;
    if (m < n) return fail(SPQ_ERR_ARG, "need rows >= cols (factor the transpose instead)");
    if (!t->cfg.X.empty() && (int64_t)t->cfg.X.size() != (int64_t)t->cfg.d * n)
        return fail(SPQ_ERR_ARG, "coordinates must be d x ncols");
    if (t->cfg.X.empty() && !t->cfg.parts.empty() && (int64_t)t->cfg.parts.size() != n)
        return fail(SPQ_ERR_ARG, "parts must have one entry per column");
    return guard([&] {
        if (!t->eng) t->eng = make_engine(t->cfg, t->precision);
        t->eng->partition(csc_from(m, n, cp, ri, va));
        t->state = 1;
        return SPQ_OK;
    });
}

int spq_assemble(spq_tree* t, int m, int n, const int* cp, const int* ri, const double* va) {
    if (!t) return fail(SPQ_ERR_ARG, "null handle");
    if (t->state != 1) return fail(SPQ_ERR_STATE, "assemble must follow partition");
    int rc = check_csc(m, n, cp, ri, va);
    if (rc) return rc;
    if (m != t->eng->nrows() || n != t->eng->ncols()) return fail(SPQ_ERR_ARG, "matrix size differs from partition");
    return guard_on(t, [&] {
        t->eng->assemble(csc_from(m, n, cp, ri, va));
        t->state = 2;
        return SPQ_OK;
    });
}

int spq_factorize(spq_tree* t) {
    if (!t) return fail(SPQ_ERR_ARG, "null handle");
    if (t->state != 2) return fail(SPQ_ERR_STATE, "factorize must follow assemble");
    return guard_on(t, [&] {
        t->eng->factorize();
        t->state = 3;
        return SPQ_OK;
    });
}

int spq_solve_dev(spq_tree* t, const double* d_b, double* d_x) {
    if (!t) return fail(SPQ_ERR_ARG, "null handle");
    if (t->state != 3) return fail(SPQ_ERR_STATE, "solve before factorize");
    if (!d_b || !d_x) return fail(SPQ_ERR_ARG, "null vector");
    return guard_on(t, [&] {
        t->eng->solve_dev(d_b, d_x);
        cuda_check(cudaStreamSynchronize(t->eng->stream()), "solve");
        return SPQ_OK;
    });
}

int spq_solve(spq_tree* t, const double* b, double* x) {
    if (!t) return fail(SPQ_ERR_ARG, "null handle");
    if (t->state != 3) return fail(SPQ_ERR_STATE, "solve before factorize");
    if (!b || !x) return fail(SPQ_ERR_ARG, "null vector");
    return guard_on(t, [&] {
        const int m = t->eng->nrows(), n = t->eng->ncols();
        cudaStream_t s = t->eng->stream();
        DevBuf buf_db, buf_dx;
        double* db = buf_db.get<double>(m, s);
        double* dx = buf_dx.get<double>(n, s);
        cuda_check(cudaMemcpyAsync(db, b, sizeof(double) * m, cudaMemcpyHostToDevice, s), "solve h2d");
        t->eng->solve_dev(db, dx);
        cuda_check(cudaMemcpyAsync(x, dx, sizeof(double) * n, cudaMemcpyDeviceToHost, s), "solve d2h");
        cuda_check(cudaStreamSynchronize(s), "solve");
        return SPQ_OK;
    });
}

int spq_solve_adjoint_dev(spq_tree* t, const double* d_g, double* d_y) {
    if (!t) return fail(SPQ_ERR_ARG, "null handle");
    if (t->state != 3) return fail(SPQ_ERR_STATE, "adjoint solve before factorize");
    if (!d_g || !d_y) return fail(SPQ_ERR_ARG, "null vector");
    return guard_on(t, [&] {
        t->eng->solve_adjoint_dev(d_g, d_y);
        cuda_check(cudaStreamSynchronize(t->eng->stream()), "adjoint solve");
        return SPQ_OK;
    });
}

int spq_solve_adjoint(spq_tree* t, const double* g, double* y) {
    if (!t) return fail(SPQ_ERR_ARG, "null handle");
    if (t->state != 3) return fail(SPQ_ERR_STATE, "adjoint solve before factorize");
    if (!g || !y) return fail(SPQ_ERR_ARG, "null vector");
    return guard_on(t, [&] {
        const int m = t->eng->nrows(), n = t->eng->ncols();
        cudaStream_t s = t->eng->stream();
        DevBuf buf_dg, buf_dy;
        double* dg = buf_dg.get<double>(n, s);
        double* dy = buf_dy.get<double>(m, s);
        cuda_check(cudaMemcpyAsync(dg, g, sizeof(double) * n, cudaMemcpyHostToDevice, s), "adjoint h2d");
        t->eng->solve_adjoint_dev(dg, dy);
        cuda_check(cudaMemcpyAsync(y, dy, sizeof(double) * m, cudaMemcpyDeviceToHost, s), "adjoint d2h");
        cuda_check(cudaStreamSynchronize(s), "adjoint solve");
        return SPQ_OK;
    });
}

int spq_gmres_adjoint_dev(spq_tree* t, int n, const int* rp, const int* ci, const double* va, const double* d_g,
                          double* d_l, int iters, int restart, double tol, int* its, double* res) {
    if (!t) return fail(SPQ_ERR_ARG, "null handle");
    if (t->state != 3) return fail(SPQ_ERR_STATE, "adjoint gmres before factorize");
    if (n != t->eng->nrows() || n != t->eng->ncols()) return fail(SPQ_ERR_ARG, "needs the square factorized matrix");
    if (!rp || !ci || !va || !d_g || !d_l || !its || !res || iters < 1) return fail(SPQ_ERR_ARG, "invalid arguments");
    return guard_on(t, [&] {
        DevCsr At;
        At.m = At.n = n;
        At.rp = rp;
        At.ci = ci;
        At.v = va;
        long long l = 0;
        *its = gmres_device(*t->eng, At, d_g, d_l, iters, restart, tol, res, &l, true);
        t->launches_krylov += l;
        cuda_check(cudaStreamSynchronize(t->eng->stream()), "adjoint gmres");
        return SPQ_OK;
    });
}

int spq_solve_to_residual_adjoint_dev(spq_tree* t, int n, const int* rp, const int* ci, const double* va,
                                      const double* d_g, double* d_l, double target, double inner_tol, int max_outer,
                                      int iters, int* its, double* true_res) {
    if (!t) return fail(SPQ_ERR_ARG, "null handle");
    if (t->state != 3) return fail(SPQ_ERR_STATE, "adjoint solve before factorize");
    if (n != t->eng->nrows() || n != t->eng->ncols()) return fail(SPQ_ERR_ARG, "needs the square factorized matrix");
    if (!rp || !ci || !va || !d_g || !d_l || !its || !true_res || iters < 1 || max_outer < 1 || !(target > 0))
        return fail(SPQ_ERR_ARG, "invalid arguments");
    return guard_on(t, [&] {
        DevCsr At;
        At.m = At.n = n;
        At.rp = rp;
        At.ci = ci;
        At.v = va;
        int outer = 0;
        long long l = 0;
        *its = refine_device(*t->eng, At, d_g, d_l, target, inner_tol, max_outer, iters, true_res, &outer, &l, true);
        t->launches_krylov += l;
        cuda_check(cudaStreamSynchronize(t->eng->stream()), "adjoint solve_to_residual");
        return *true_res <= target ? SPQ_OK : fail(SPQ_ERR_NOCONV, "target residual not reached");
    });
}

int spq_gmres_adjoint(spq_tree* t, int m, int n, const int* cp, const int* ri, const double* va, const double* g,
                      double* lam, int iters, int restart, double tol, int* its, double* res) {
    if (!t) return fail(SPQ_ERR_ARG, "null handle");
    if (t->state != 3) return fail(SPQ_ERR_STATE, "adjoint gmres before factorize");
    if (m != n || m != t->eng->nrows()) return fail(SPQ_ERR_ARG, "adjoint gmres needs the square factorized matrix");
    int rc = check_csc(m, n, cp, ri, va);
    if (rc) return rc;
    if (!g || !lam || !its || !res || iters < 1) return fail(SPQ_ERR_ARG, "invalid adjoint gmres arguments");
    return guard_on(t, [&] {
        cudaStream_t s = t->eng->stream();
        // the CSC arrays of A are the CSR arrays of A^T
        DevCsrOwned o;
        const size_t nnz = (size_t)cp[n];
        int* o_rp = o.rp.get<int>((size_t)n + 1, s);
        int* o_ci = o.ci.get<int>(nnz, s);
        double* o_v = o.v.get<double>(nnz, s);
        cuda_check(cudaMemcpyAsync(o_rp, cp, sizeof(int) * (n + 1), cudaMemcpyHostToDevice, s), "csr up");
        cuda_check(cudaMemcpyAsync(o_ci, ri, sizeof(int) * nnz, cudaMemcpyHostToDevice, s), "csr up");
        cuda_check(cudaMemcpyAsync(o_v, va, sizeof(double) * nnz, cudaMemcpyHostToDevice, s), "csr up");
        DevCsr At;
        At.m = n;
        At.n = m;
        At.rp = o_rp;
        At.ci = o_ci;
        At.v = o_v;
        DevBuf buf_dg, buf_dl;
        double* dg = buf_dg.get<double>(n, s);
        double* dl = buf_dl.get<double>(m, s);
        cuda_check(cudaMemcpyAsync(dg, g, sizeof(double) * n, cudaMemcpyHostToDevice, s), "adjoint h2d");
        cuda_check(cudaMemcpyAsync(dl, lam, sizeof(double) * m, cudaMemcpyHostToDevice, s), "adjoint h2d");
        long long l = 0;
        *its = gmres_device(*t->eng, At, dg, dl, iters, restart, tol, res, &l, true);
        t->launches_krylov += l;
        cuda_check(cudaMemcpyAsync(lam, dl, sizeof(double) * m, cudaMemcpyDeviceToHost, s), "adjoint d2h");
        cuda_check(cudaStreamSynchronize(s), "adjoint gmres");
        return SPQ_OK;
    });
}

int spq_solve_nrml_dev(spq_tree* t, const double* d_b, double* d_x) {
    if (!t) return fail(SPQ_ERR_ARG, "null handle");
    if (t->state != 3) return fail(SPQ_ERR_STATE, "solve_nrml before factorize");
    if (!d_b || !d_x) return fail(SPQ_ERR_ARG, "null vector");
    return guard_on(t, [&] {
        t->eng->solve_nrml_dev(d_b, d_x);
        cuda_check(cudaStreamSynchronize(t->eng->stream()), "solve_nrml");
        return SPQ_OK;
    });
}
int spq_solve_nrml(spq_tree* t, const double* b, double* x) {
    if (!t) return fail(SPQ_ERR_ARG, "null handle");
    if (t->state != 3) return fail(SPQ_ERR_STATE, "solve_nrml before factorize");
    if (!b || !x) return fail(SPQ_ERR_ARG, "null vector");
    return guard_on(t, [&] {
        const int n = t->eng->ncols();
        cudaStream_t s = t->eng->stream();
        DevBuf buf_db, buf_dx;
        double* db = buf_db.get<double>(n, s);
        double* dx = buf_dx.get<double>(n, s);
        cuda_check(cudaMemcpyAsync(db, b, sizeof(double) * n, cudaMemcpyHostToDevice, s), "solve_nrml h2d");
        t->eng->solve_nrml_dev(db, dx);
        cuda_check(cudaMemcpyAsync(x, dx, sizeof(double) * n, cudaMemcpyDeviceToHost, s), "solve_nrml d2h");
        cuda_check(cudaStreamSynchronize(s), "solve_nrml");
        return SPQ_OK;
    });
}

int spq_gmres(spq_tree* t, int m, int n, const int* cp, const int* ri, const double* va, const double* b, double* x,
              int iters, int restart, double tol, int* its, double* res) {
    if (!t) return fail(SPQ_ERR_ARG, "null handle");
    if (t->state != 3) return fail(SPQ_ERR_STATE, "gmres before factorize");
    if (m != n || m != t->eng->nrows()) return fail(SPQ_ERR_ARG, "gmres needs the square factorized matrix");
    int rc = check_csc(m, n, cp, ri, va);
    if (rc) return rc;
    if (!b || !x || !its || !res || iters < 1) return fail(SPQ_ERR_ARG, "invalid gmres arguments");
    return guard_on(t, [&] {
        cudaStream_t s = t->eng->stream();
        DevCsrOwned o;
        DevCsr A;
        upload_csr(csc_from(m, n, cp, ri, va), o, A, s);
        DevBuf buf_db, buf_dx;
        double* db = buf_db.get<double>(m, s);
        double* dx = buf_dx.get<double>(n, s);
        cuda_check(cudaMemcpyAsync(db, b, sizeof(double) * m, cudaMemcpyHostToDevice, s), "gmres h2d");
        cuda_check(cudaMemcpyAsync(dx, x, sizeof(double) * n, cudaMemcpyHostToDevice, s), "gmres h2d");
        long long l = 0;
        *its = gmres_device(*t->eng, A, db, dx, iters, restart, tol, res, &l);
        t->launches_krylov += l;
        cuda_check(cudaMemcpyAsync(x, dx, sizeof(double) * n, cudaMemcpyDeviceToHost, s), "gmres d2h");
        cuda_check(cudaStreamSynchronize(s), "gmres");
        return SPQ_OK;
    });
}

int spq_solve_to_residual(spq_tree* t, int m, int n, const int* cp, const int* ri, const double* va, const double* b,
                          double* x, double target, double inner_tol, int max_outer, int iters, int* its,
                          double* true_res) {
    if (!t) return fail(SPQ_ERR_ARG, "null handle");
    if (t->state != 3) return fail(SPQ_ERR_STATE, "solve_to_residual before factorize");
    if (m != n || m != t->eng->nrows()) return fail(SPQ_ERR_ARG, "needs the square factorized matrix");
    int rc = check_csc(m, n, cp, ri, va);
    if (rc) return rc;
    if (!b || !x || !its || !true_res || iters < 1 || max_outer < 1 || !(target > 0))
        return fail(SPQ_ERR_ARG, "invalid arguments");
    return guard_on(t, [&] {
        cudaStream_t s = t->eng->stream();
        DevCsrOwned o;
        DevCsr A;
        upload_csr(csc_from(m, n, cp, ri, va), o, A, s);
        DevBuf buf_db, buf_dx;
        double* db = buf_db.get<double>(m, s);
        double* dx = buf_dx.get<double>(n, s);
        cuda_check(cudaMemcpyAsync(db, b, sizeof(double) * m, cudaMemcpyHostToDevice, s), "h2d");
        cuda_check(cudaMemcpyAsync(dx, x, sizeof(double) * n, cudaMemcpyHostToDevice, s), "h2d");
        int outer = 0;
        long long l = 0;
        *its = refine_device(*t->eng, A, db, dx, target, inner_tol, max_outer, iters, true_res, &outer, &l);
        t->launches_krylov += l;
        cuda_check(cudaMemcpyAsync(x, dx, sizeof(double) * n, cudaMemcpyDeviceToHost, s), "d2h");
        cuda_check(cudaStreamSynchronize(s), "solve_to_residual");
        return *true_res <= target ? SPQ_OK : fail(SPQ_ERR_NOCONV, "target residual not reached");
    });
}

int spq_solve_to_residual_dev(spq_tree* t, int m, const int* rp, const int* ci, const double* va, const double* d_b,
                              double* d_x, double target, double inner_tol, int max_outer, int iters, int* its,
                              double* true_res) {
    if (!t) return fail(SPQ_ERR_ARG, "null handle");
    if (t->state != 3) return fail(SPQ_ERR_STATE, "solve_to_residual before factorize");
    if (m != t->eng->nrows() || m != t->eng->ncols()) return fail(SPQ_ERR_ARG, "needs the square factorized matrix");
    if (!rp || !ci || !va || !d_b || !d_x || !its || !true_res || iters < 1 || max_outer < 1 || !(target > 0))
        return fail(SPQ_ERR_ARG, "invalid arguments");
    return guard_on(t, [&] {
        DevCsr A;
        A.m = A.n = m;
        A.rp = rp;
        A.ci = ci;
        A.v = va;
        int outer = 0;
        long long l = 0;
        *its = refine_device(*t->eng, A, d_b, d_x, target, inner_tol, max_outer, iters, true_res, &outer, &l);
        t->launches_krylov += l;
        cuda_check(cudaStreamSynchronize(t->eng->stream()), "solve_to_residual");
        return *true_res <= target ? SPQ_OK : fail(SPQ_ERR_NOCONV, "target residual not reached");
    });
}

int spq_gmres_dev(spq_tree* t, int m, const int* rp, const int* ci, const double* va, const double* d_b, double* d_x,
                  int iters, int restart, double tol, int* its, double* res) {
    if (!t) return fail(SPQ_ERR_ARG, "null handle");
    if (t->state != 3) return fail(SPQ_ERR_STATE, "gmres before factorize");
    if (m != t->eng->nrows() || m != t->eng->ncols()) return fail(SPQ_ERR_ARG, "needs the square factorized matrix");
    if (!rp || !ci || !va || !d_b || !d_x || !its || !res || iters < 1) return fail(SPQ_ERR_ARG, "invalid arguments");
    return guard_on(t, [&] {
        DevCsr A;
        A.m = A.n = m;
        A.rp = rp;
        A.ci = ci;
        A.v = va;
        long long l = 0;
        *its = gmres_device(*t->eng, A, d_b, d_x, iters, restart, tol, res, &l);
        t->launches_krylov += l;
        cuda_check(cudaStreamSynchronize(t->eng->stream()), "gmres");
        return SPQ_OK;
    });
}

int spq_gmres_dev_noalloc(spq_tree* t, int m, const int* rp, const int* ci, const double* va, const double* d_b,
                          double* d_x, int iters, int restart, double tol, int* its, double* res) {
    if (!t) return fail(SPQ_ERR_ARG, "null handle");
    if (t->state != 3) return fail(SPQ_ERR_STATE, "gmres before factorize");
    if (m != t->eng->nrows() || m != t->eng->ncols()) return fail(SPQ_ERR_ARG, "needs the square factorized matrix");
    if (!rp || !ci || !va || !d_b || !d_x || !its || !res || iters < 1) return fail(SPQ_ERR_ARG, "invalid arguments");
    if (!t->eng->solve_ready())
        return fail(SPQ_ERR_STATE,
                    "apply the preconditioner once (spq_solve, spq_solve_dev or spq_gmres_dev) before the "
                    "no-allocation GMRES: the first application builds its solve graph");
    return guard_on(t, [&]() -> int {
        cuda_check(cudaSetDevice(t->cfg.device), "cudaSetDevice");
        double* ws = nullptr;
        size_t cap = 0;
        cuda_check(noalloc_scratch(&ws, &cap), "no-allocation workspace address");
        const size_t need = gmres_workspace_elems(m, restart);
        if (need > cap)
            return fail(SPQ_ERR_ARG, "no-allocation GMRES needs " + std::to_string(need) +
                                         " doubles of workspace (m * (restart + 1) + 5 m + ...) but the fixed "
                                         "workspace holds " + std::to_string(cap) + "; lower restart or use spq_gmres_dev");
        DevCsr A;
        A.m = A.n = m;
        A.rp = rp;
        A.ci = ci;
        A.v = va;
        long long l = 0;
        *its = gmres_device_ws(*t->eng, A, d_b, d_x, iters, restart, tol, res, &l, ws);
        t->launches_krylov += l;
        cuda_check(cudaStreamSynchronize(t->eng->stream()), "gmres");
        return SPQ_OK;
    });
}

int spq_get_launches(spq_tree* t, long long* factorize, long long* krylov, long long* solve_graph_kernels,
                     long long* applications) {
    if (!t) return fail(SPQ_ERR_ARG, "null handle");
    double times[4];
    long long c[8] = {0};
    if (t->eng) t->eng->stats(times, c);
    if (factorize) *factorize = c[4];
    if (krylov) *krylov = t->launches_krylov;
    if (solve_graph_kernels) *solve_graph_kernels = c[5];
    if (applications) *applications = c[7];
    return SPQ_OK;
}

int spq_set_profile(spq_tree* t, int profile) {
    if (!t) return fail(SPQ_ERR_ARG, "null handle");
    if (!t->eng) return fail(SPQ_ERR_STATE, "profile before partition");
    t->eng->set_profile(profile);
    return SPQ_OK;
}
int spq_get_kernel_stats(spq_tree* t, int family, double* out4) {
    if (!t || !out4) return fail(SPQ_ERR_ARG, "null argument");
    if (!t->eng) return fail(SPQ_ERR_STATE, "no engine");
    if (family < 0 || family >= kNumFamilies) return fail(SPQ_ERR_ARG, "unknown kernel family");
    return guard_on(t, [&] {
        KernelStat s = t->eng->kernel_stat(family);
        out4[0] = (double)s.launches;
        out4[1] = s.ms;
        out4[2] = s.flops;
        out4[3] = s.bytes;
        return SPQ_OK;
    });
}
int spq_reset_kernel_stats(spq_tree* t) {
    if (!t) return fail(SPQ_ERR_ARG, "null handle");
    if (!t->eng) return SPQ_OK;
    return guard_on(t, [&] {
        t->eng->reset_kernel_stats();
        return SPQ_OK;
    });
}
int spq_profile_solve_waves(spq_tree* t, double* out, int cap, int* nwaves) {
    if (!t || !out || !nwaves) return fail(SPQ_ERR_ARG, "null argument");
    if (t->state != 3) return fail(SPQ_ERR_STATE, "profile before factorize");
    return guard_on(t, [&] {
        auto v = t->eng->profile_solve_waves();
        *nwaves = (int)(v.size() / 7);
        std::memcpy(out, v.data(), sizeof(double) * std::min<size_t>(v.size(), (size_t)cap * 7));
        return SPQ_OK;
    });
}

int spq_get_stream(spq_tree* t, void** stream) {
    if (!t || !stream) return fail(SPQ_ERR_ARG, "null argument");
    if (!t->eng || t->state < 2) return fail(SPQ_ERR_STATE, "no stream before assemble");
    *stream = (void*)t->eng->stream();
    return SPQ_OK;
}

int spq_cgls_dev(spq_tree* t, int m, int n, const int* rp, const int* ci, const double* va, const int* rp_t,
                 const int* ci_t, const double* va_t, const double* d_b, double* d_x, int iters, double tol, int* its,
                 double* res) {
    if (!t) return fail(SPQ_ERR_ARG, "null handle");
    if (t->state != 3) return fail(SPQ_ERR_STATE, "cgls before factorize");
    if (!t->eng->least_squares())
        return fail(SPQ_ERR_STATE, "cgls needs a least-squares factorization (square matching off)");
    if (m != t->eng->nrows() || n != t->eng->ncols()) return fail(SPQ_ERR_ARG, "cgls needs the factorized matrix");
    if (!rp || !ci || !va || !rp_t || !ci_t || !va_t || !d_b || !d_x || !its || !res || iters < 0)
        return fail(SPQ_ERR_ARG, "invalid cgls arguments");
    return guard_on(t, [&] {
        DevCsr A, At;
        A.m = m;
        A.n = n;
        A.rp = rp;
        A.ci = ci;
        A.v = va;
        At.m = n;
        At.n = m;
        At.rp = rp_t;
        At.ci = ci_t;
        At.v = va_t;
        long long l = 0;
        *its = cgls_device(*t->eng, A, At, d_b, d_x, iters, tol, res, &l);
        t->launches_krylov += l;
        cuda_check(cudaStreamSynchronize(t->eng->stream()), "cgls");
        return SPQ_OK;
    });
}

int spq_cgls(spq_tree* t, int m, int n, const int* cp, const int* ri, const double* va, const double* b, double* x,
             int iters, double tol, int* its, double* res) {
    if (!t) return fail(SPQ_ERR_ARG, "null handle");
    if (t->state != 3) return fail(SPQ_ERR_STATE, "cgls before factorize");
    if (m != t->eng->nrows() || n != t->eng->ncols()) return fail(SPQ_ERR_ARG, "cgls needs the factorized matrix");
    int rc = check_csc(m, n, cp, ri, va);
    if (rc) return rc;
    if (!b || !x || !its || !res || iters < 0) return fail(SPQ_ERR_ARG, "invalid cgls arguments");
    if (!t->eng->least_squares())
        return fail(SPQ_ERR_STATE, "cgls needs a least-squares factorization (square matching off)");
    return guard_on(t, [&]() -> int {
        cudaStream_t s = t->eng->stream();
        DevCsrOwned o, ot;
        DevCsr A;
        upload_csr(csc_from(m, n, cp, ri, va), o, A, s);
        // the CSC arrays of A are the CSR arrays of A^T
        const size_t nnz = (size_t)cp[n];
        int* ot_rp = ot.rp.get<int>((size_t)n + 1, s);
        int* ot_ci = ot.ci.get<int>(nnz, s);
        double* ot_v = ot.v.get<double>(nnz, s);
        cuda_check(cudaMemcpyAsync(ot_rp, cp, sizeof(int) * (n + 1), cudaMemcpyHostToDevice, s), "csr up");
        cuda_check(cudaMemcpyAsync(ot_ci, ri, sizeof(int) * nnz, cudaMemcpyHostToDevice, s), "csr up");
        cuda_check(cudaMemcpyAsync(ot_v, va, sizeof(double) * nnz, cudaMemcpyHostToDevice, s), "csr up");
        DevBuf buf_db, buf_dx;
        double* db = buf_db.get<double>(m, s);
        double* dx = buf_dx.get<double>(n, s);
        cuda_check(cudaMemcpyAsync(db, b, sizeof(double) * m, cudaMemcpyHostToDevice, s), "cgls h2d");
        cuda_check(cudaMemcpyAsync(dx, x, sizeof(double) * n, cudaMemcpyHostToDevice, s), "cgls h2d");
        const int r2 = spq_cgls_dev(t, m, n, A.rp, A.ci, A.v, ot_rp, ot_ci, ot_v, db, dx, iters, tol, its, res);
        if (r2 == SPQ_OK) {
            cuda_check(cudaMemcpyAsync(x, dx, sizeof(double) * n, cudaMemcpyDeviceToHost, s), "cgls d2h");
            cuda_check(cudaStreamSynchronize(s), "cgls");
        }
        return r2;
    });
}

int spq_get_perm(spq_tree* t, int* cperm, int* rperm) {
    if (!t || !t->eng || t->state < 1) return fail(SPQ_ERR_STATE, "no partition");
    if (cperm) std::memcpy(cperm, t->eng->cperm().data(), sizeof(int) * t->eng->cperm().size());
    if (rperm) std::memcpy(rperm, t->eng->rperm().data(), sizeof(int) * t->eng->rperm().size());
    return SPQ_OK;
}
int spq_log_size(spq_tree* t, long long* n) {
    if (!t || !n) return fail(SPQ_ERR_ARG, "null argument");
    *n = t->eng ? (long long)t->eng->log().size() : 0;
    return SPQ_OK;
}
int spq_get_log(spq_tree* t, long long* out) {
    if (!t || !out) return fail(SPQ_ERR_ARG, "null argument");
    if (t->eng) std::memcpy(out, t->eng->log().data(), sizeof(long long) * t->eng->log().size());
    return SPQ_OK;
}
int spq_num_bottom(spq_tree* t, int* n) {
    if (!t || !n) return fail(SPQ_ERR_ARG, "null argument");
    *n = t->eng ? (int)(t->eng->bottom_info().size() / 10) : 0;
    return SPQ_OK;
}
int spq_get_bottom(spq_tree* t, int* out) {
    if (!t || !out) return fail(SPQ_ERR_ARG, "null argument");
    if (t->eng) {
        auto v = t->eng->bottom_info();
        std::memcpy(out, v.data(), sizeof(int) * v.size());
    }
    return SPQ_OK;
}
int spq_get_stats(spq_tree* t, double* times, long long* counters) {
    if (!t || !times || !counters) return fail(SPQ_ERR_ARG, "null argument");
    if (!t->eng) return fail(SPQ_ERR_STATE, "no engine");
    t->eng->stats(times, counters);
    return SPQ_OK;
}
int spq_factorize_batch(spq_tree* const* ts, int n, int nthreads) {
    if (n < 0 || (n > 0 && !ts)) return fail(SPQ_ERR_ARG, "invalid batch");
    for (int i = 0; i < n; ++i) {
        if (!ts[i]) return fail(SPQ_ERR_ARG, "null handle in batch at " + std::to_string(i));
        if (ts[i]->state != 2) return fail(SPQ_ERR_STATE, "batch handle " + std::to_string(i) + " is not assembled");
        for (int j = 0; j < i; ++j)
            if (ts[j] == ts[i]) return fail(SPQ_ERR_ARG, "a handle appears twice in the batch");
    }
    if (n == 0) return SPQ_OK;
    const int hw = (int)std::max(1u, std::thread::hardware_concurrency());
    const int nt = std::max(1, std::min(n, nthreads > 0 ? nthreads : std::min(hw, 32)));
    std::atomic<int> next{0};
    std::vector<int> rc(n, SPQ_OK);
    std::vector<std::string> err(n);
    auto work = [&] {
        for (int i = next++; i < n; i = next++) {
            rc[i] = spq_factorize(ts[i]);
            if (rc[i] != SPQ_OK) err[i] = g_err;
        }
    };
    std::vector<std::thread> pool;
    for (int q = 1; q < nt; ++q) pool.emplace_back(work);
    work();
    for (auto& th : pool) th.join();
    for (int i = 0; i < n; ++i)
        if (rc[i] != SPQ_OK) return fail(rc[i], "batch handle " + std::to_string(i) + ": " + err[i]);
    return SPQ_OK;
}

int spq_trim_memory(void) {
    return guard([&] {
        trim_device_pools();
        return SPQ_OK;
    });
}
int spq_pool_memory(int device, unsigned long long* used, unsigned long long* reserved) {
    if (!used || !reserved || device < 0) return fail(SPQ_ERR_ARG, "invalid arguments");
    return guard([&] {
        *used = *reserved = 0;
        cudaMemPool_t pool = nullptr;
        {
            std::lock_guard<std::mutex> g(pool_mutex());
            auto it = pool_table().find(device);
            if (it != pool_table().end()) pool = it->second;
        }
        if (!pool) return SPQ_OK;
        uint64_t u = 0, r = 0;
        cuda_check(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &u), "pool used memory");
        cuda_check(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &r), "pool reserved memory");
        *used = u;
        *reserved = r;
        return SPQ_OK;
    });
}
int spq_autotune_set_mode(int mode) {
    if (mode < 0 || mode > 2) return fail(SPQ_ERR_ARG, "autotune mode must be 0 (off), 1 (online) or 2 (frozen)");
    spq::Autotuner::get().set_mode(mode);
    return SPQ_OK;
}
int spq_autotune_get(int* mode, int* entries, int* pending) {
    if (!mode && !entries && !pending) return fail(SPQ_ERR_ARG, "null arguments");
    if (mode) *mode = spq::Autotuner::get().mode();
    if (entries) *entries = spq::Autotuner::get().entries();
    if (pending) *pending = spq::Autotuner::get().pending();
    return SPQ_OK;
}
int spq_autotune_reset(void) {
    spq::Autotuner::get().reset();
    return SPQ_OK;
}
int spq_autotune_save(const char* path) {
    if (!path) return fail(SPQ_ERR_ARG, "null path");
    return spq::Autotuner::get().save(path) ? SPQ_OK : fail(SPQ_ERR_ARG, std::string("cannot write ") + path);
}
int spq_autotune_load(const char* path) {
    if (!path) return fail(SPQ_ERR_ARG, "null path");
    return spq::Autotuner::get().load(path) ? SPQ_OK
                                            : fail(SPQ_ERR_ARG, std::string("cannot read a tuning table from ") + path);
}
int spq_get_host_times(spq_tree* t, double* out11) {
    if (!t || !out11) return fail(SPQ_ERR_ARG, "null argument");
    if (!t->eng || t->state < 3) return fail(SPQ_ERR_STATE, "not factorized");
    auto v = t->eng->host_times();
    std::memcpy(out11, v.data(), sizeof(double) * 11);
    return SPQ_OK;
}
int spq_get_level_times(spq_tree* t, double* out) {
    if (!t || !out) return fail(SPQ_ERR_ARG, "null argument");
    if (!t->eng || t->state < 3) return fail(SPQ_ERR_STATE, "not factorized");
    auto v = t->eng->level_times();
    std::memcpy(out, v.data(), sizeof(double) * v.size());
    return SPQ_OK;
}

int spq_column_normalize(int m, int n, const int* cp, const int* ri, double* va) {
    int rc = check_csc(m, n, cp, ri, va);
    if (rc) return rc;
    for (int j = 0; j < n; ++j) {
        double s = 0;
        for (int q = cp[j]; q < cp[j + 1]; ++q) s += va[q] * va[q];
        const double d = 1.0 / std::sqrt(s);
        for (int q = cp[j]; q < cp[j + 1]; ++q) va[q] = (va[q] * d) * 10.0;
    }
    return SPQ_OK;
}

}  // extern "C"
