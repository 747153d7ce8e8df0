"""Python mirror of the reference's ``Tree`` and Krylov drivers over the C ABI.

Reference surface (include/tree.h:113-147, include/is.h:14-19):

    Tree t(nlevels, skip); t.set_tol(tol); t.set_scale(1); t.set_square(1);
    t.set_Xcoo(&X); t.partition(A); t.assemble(A); t.factorize();
    t.solve(b, x);  gmres(A, b, x, t, iters, restart, tol, verb);

Here::

    t = Tree(nlevels, skip); t.set_tol(tol); t.set_scale(1); t.set_square(1)
    t.set_coords_grid(n, d)            # -n/-d, i.e. set_Xcoo(linspace_nd(n, d))
    t.partition(A); t.assemble(A); t.factorize()
    x = t.solve(b)
    x, its, res = gmres(A, b, t, iters, restart, tol)

Matrices are CSC tuples ``(m, n, colptr, rowind, val)`` (as produced by
``spaqr_public_b200.matgen``) with sorted row indices.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi
from ._abi import check, dptr, iptr, lib

FP64 = _abi.SPQ_FP64
FP32 = _abi.SPQ_FP32


def _csc(A):
    m, n, cp, ri, va = A
    return (int(m), int(n), np.ascontiguousarray(cp, dtype=np.int32), np.ascontiguousarray(ri, dtype=np.int32),
            np.ascontiguousarray(va, dtype=np.float64))


class Tree:
    """spaQR hierarchical sparsified QR on one B200 (include/tree.h:36-152)."""

    def __init__(self, nlevels, skip=0, precision=FP64, device=0):
        h = C.c_void_p()
        check(lib().spq_create(C.byref(h), int(nlevels), int(skip)))
        self._h = h
        self.nlevels = nlevels
        self.m = self.n = 0
        if precision != FP64:
            self.set_precision(precision)
        if device:
            check(lib().spq_set_device(h, int(device)))

    def close(self):
        if getattr(self, "_h", None):
            lib().spq_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # setters (include/tree.h:124-130)
    def set_tol(self, tol):
        check(lib().spq_set_tol(self._h, float(tol)))

    def set_scale(self, s):
        check(lib().spq_set_scale(self._h, int(s)))

    def set_order(self, o):
        check(lib().spq_set_order(self._h, float(o)))

    def set_hsl(self, h):
        check(lib().spq_set_hsl(self._h, int(h)))

    def set_square(self, s):
        check(lib().spq_set_square(self._h, int(s)))

    def set_precision(self, p):
        check(lib().spq_set_precision(self._h, int(p)))

    def set_verbose(self, v):
        check(lib().spq_set_verbose(self._h, int(v)))

    def set_coords(self, X):
        """X: d x n coordinates (set_Xcoo)."""
        X = np.asarray(X, dtype=np.float64)
        d, n = X.shape
        Xc = np.ascontiguousarray(X.T.reshape(-1))
        check(lib().spq_set_coords(self._h, d, n, dptr(Xc)))

    def set_coords_grid(self, n, d):
        check(lib().spq_set_coords_grid(self._h, int(n), int(d)))

    def set_parts(self, parts):
        """Leaf part of every column for the ordering without coordinates
        (the METIS part vector of src/partition.cpp:374-426)."""
        p = np.ascontiguousarray(parts, dtype=np.int32)
        check(lib().spq_set_parts(self._h, int(p.size), iptr(p)))

    def set_fill_rule(self, numeric):
        """Ordering without coordinates: 1 (default) keeps a fill candidate only
        if ||A1^T A2|| > 1e-14 (the reference, src/tree.cpp:856-859); 0 keeps
        every candidate that passes the separator tests."""
        check(lib().spq_set_fill_rule(self._h, int(numeric)))

    # main steps (include/tree.h:139-147)
    def partition(self, A):
        m, n, cp, ri, va = _csc(A)
        self.m, self.n = m, n
        check(lib().spq_partition(self._h, m, n, iptr(cp), iptr(ri), dptr(va)))

    def assemble(self, A):
        m, n, cp, ri, va = _csc(A)
        check(lib().spq_assemble(self._h, m, n, iptr(cp), iptr(ri), dptr(va)))

    def factorize(self):
        check(lib().spq_factorize(self._h))
        return 0

    def solve(self, b):
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.zeros(self.n)
        check(lib().spq_solve(self._h, dptr(b), dptr(x)))
        return x

    def solve_dev(self, d_b, d_x):
        """Device pointers (e.g. torch tensors' data_ptr()) of FP64 vectors."""
        check(lib().spq_solve_dev(self._h, C.c_void_p(d_b), C.c_void_p(d_x)))

    def solve_adjoint(self, g):
        """y = M^T g: the preconditioner's transpose (factors applied transposed)."""
        g = np.ascontiguousarray(g, dtype=np.float64)
        y = np.zeros(self.m)
        check(lib().spq_solve_adjoint(self._h, dptr(g), dptr(y)))
        return y

    def solve_adjoint_dev(self, d_g, d_y):
        check(lib().spq_solve_adjoint_dev(self._h, C.c_void_p(d_g), C.c_void_p(d_y)))

    def solve_nrml(self, b):
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.zeros(self.n)
        check(lib().spq_solve_nrml(self._h, dptr(b), dptr(x)))
        return x

    # introspection
    def perms(self):
        cp = np.zeros(self.n, dtype=np.int32)
        rp = np.zeros(self.m, dtype=np.int32)
        check(lib().spq_get_perm(self._h, iptr(cp), iptr(rp)))
        return cp, rp

    def log(self):
        n = C.c_longlong(0)
        check(lib().spq_log_size(self._h, C.byref(n)))
        out = np.zeros(n.value, dtype=np.int64)
        if n.value:
            check(lib().spq_get_log(self._h, out.ctypes.data_as(C.POINTER(C.c_longlong))))
        return out.reshape(-1, 8)

    def bottom(self):
        k = C.c_int(0)
        check(lib().spq_num_bottom(self._h, C.byref(k)))
        out = np.zeros(10 * k.value, dtype=np.int32)
        if k.value:
            check(lib().spq_get_bottom(self._h, iptr(out)))
        return out.reshape(-1, 10)

    def stats(self):
        t = np.zeros(4)
        c = np.zeros(8, dtype=np.int64)
        check(lib().spq_get_stats(self._h, dptr(t), c.ctypes.data_as(C.POINTER(C.c_longlong))))
        return dict(partition=t[0], assemble=t[1], factorize=t[2], solve=t[3], nnzA=int(c[0]), nnzR=int(c[1]),
                    nnzH=int(c[2]), nnzQ=int(c[3]), launches_factorize=int(c[4]), launches_solve=int(c[5]),
                    device_bytes=int(c[6]))

    def level_times(self):
        out = np.zeros(6 * self.nlevels)
        check(lib().spq_get_level_times(self._h, dptr(out)))
        return out.reshape(self.nlevels, 6)


def gmres(A, b, precond, iters=300, restart=None, tol=1e-12, x0=None):
    """Householder GMRES left-preconditioned by ``precond`` (src/is.cpp:94-272).
    Returns (x, iterations, preconditioned residual estimate)."""
    m, n, cp, ri, va = _csc(A)
    b = np.ascontiguousarray(b, dtype=np.float64)
    x = np.zeros(n) if x0 is None else np.array(x0, dtype=np.float64)
    its = C.c_int(0)
    res = C.c_double(0)
    check(lib().spq_gmres(precond._h, m, n, iptr(cp), iptr(ri), dptr(va), dptr(b), dptr(x), int(iters),
                          int(iters if restart is None else restart), float(tol), C.byref(its), C.byref(res)))
    return x, its.value, res.value


def factorize_batch(trees, nthreads=0):
    """Factorizes independent assembled trees together (spq_factorize_batch):
    one host thread and CUDA stream per tree, so their launches share the GPU."""
    arr = (C.c_void_p * len(trees))(*[t._h.value for t in trees])
    check(lib().spq_factorize_batch(arr, len(trees), int(nthreads)))


def gmres_adjoint(A, g, precond, iters=300, restart=None, tol=1e-12, lam0=None):
    """GMRES on A^T lambda = g preconditioned by M^T (the adjoint of ``gmres``).
    A is the factorized matrix (CSC). Returns (lambda, iterations, residual estimate)."""
    m, n, cp, ri, va = _csc(A)
    g = np.ascontiguousarray(g, dtype=np.float64)
    lam = np.zeros(m) if lam0 is None else np.array(lam0, dtype=np.float64)
    its = C.c_int(0)
    res = C.c_double(0)
    check(lib().spq_gmres_adjoint(precond._h, m, n, iptr(cp), iptr(ri), dptr(va), dptr(g), dptr(lam), int(iters),
                                  int(iters if restart is None else restart), float(tol), C.byref(its),
                                  C.byref(res)))
    return lam, its.value, res.value


def solve_to_residual(A, b, precond, target=1e-10, inner_tol=None, max_outer=8, iters=300, x0=None):
    """Iterative refinement on the true FP64 residual with preconditioned GMRES
    corrections (the time-to-residual driver). Returns (x, gmres iterations,
    final ||b - A x|| / ||b||). Raises SpqError(SPQ_ERR_NOCONV) if the target is
    not reached."""
    m, n, cp, ri, va = _csc(A)
    if inner_tol is None:
        inner_tol = target
    b = np.ascontiguousarray(b, dtype=np.float64)
    x = np.zeros(n) if x0 is None else np.array(x0, dtype=np.float64)
    its = C.c_int(0)
    res = C.c_double(0)
    rc = lib().spq_solve_to_residual(precond._h, m, n, iptr(cp), iptr(ri), dptr(va), dptr(b), dptr(x),
                                     float(target), float(inner_tol), int(max_outer), int(iters), C.byref(its),
                                     C.byref(res))
    check(rc)
    return x, its.value, res.value


def launches(precond):
    """Kernel launches: factorize, Krylov vector kernels, kernels per preconditioner
    application (one CUDA graph) and applications so far."""
    f, k, s, a = C.c_longlong(0), C.c_longlong(0), C.c_longlong(0), C.c_longlong(0)
    check(lib().spq_get_launches(precond._h, C.byref(f), C.byref(k), C.byref(s), C.byref(a)))
    return dict(factorize=f.value, krylov=k.value, solve_graph_kernels=s.value, applications=a.value,
                total=f.value + k.value + s.value * a.value)


def cgls(A, b, precond, iters=300, tol=1e-12):
    """Preconditioned CGLS (src/is.cpp:274-345)."""
    m, n, cp, ri, va = _csc(A)
    b = np.ascontiguousarray(b, dtype=np.float64)
    x = np.zeros(n)
    its = C.c_int(0)
    res = C.c_double(0)
    check(lib().spq_cgls(precond._h, m, n, iptr(cp), iptr(ri), dptr(va), dptr(b), dptr(x), int(iters), float(tol),
                         C.byref(its), C.byref(res)))
    return x, its.value, res.value


def column_normalize(A):
    """A <- A diag(1/||A_j||) 10 (spaQR.cpp:131-147), computed by the library."""
    m, n, cp, ri, va = _csc(A)
    out = va.copy()
    check(lib().spq_column_normalize(m, n, iptr(cp), iptr(ri), dptr(out)))
    return (m, n, cp, ri, out)


def graph_parts(A, nlevels):
    """Leaf parts (2^(nlevels-1), first cut in the highest bit) of this library's
    recursive bisection of the A^T A graph: the ordering used when no
    coordinates are set. Host only."""
    m, n, cp, ri, _ = _csc(A)
    parts = np.zeros(n, dtype=np.int32)
    check(lib().spq_graph_parts(m, n, iptr(cp), iptr(ri), int(nlevels), iptr(parts)))
    return parts


def autotune(mode=None, reset=False, save=None, load=None):
    """The library's launch-shape autotuner (process-wide; shapes it picks never
    change results). ``mode``: 0 off, 1 online (default), 2 frozen table;
    ``reset`` clears the table; ``save`` / ``load`` a text table file.
    Returns (mode, number of table entries, timed launches still to explore)."""
    if reset:
        check(lib().spq_autotune_reset())
    if load is not None:
        check(lib().spq_autotune_load(str(load).encode()))
    if mode is not None:
        check(lib().spq_autotune_set_mode(int(mode)))
    if save is not None:
        check(lib().spq_autotune_save(str(save).encode()))
    md, ne, pe = C.c_int(0), C.c_int(0), C.c_int(0)
    check(lib().spq_autotune_get(C.byref(md), C.byref(ne), C.byref(pe)))
    return md.value, ne.value, pe.value
