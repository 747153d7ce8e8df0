"""ctypes binding of the CPU oracle (oracle/_build/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, the smoke check and the CPU
baseline leg of bench.py. PARITY UNPINNED (see spaqr_oracle.h).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None

_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        L.orc_create.restype = C.c_void_p
        L.orc_create.argtypes = [C.c_int, C.c_int, C.c_double, C.c_int, C.c_float, C.c_int]
        L.orc_destroy.argtypes = [C.c_void_p]
        L.orc_last_error.restype = C.c_char_p
        L.orc_blas_threads.argtypes = [C.c_int]
        L.orc_set_threads.argtypes = [C.c_void_p, C.c_int]
        L.orc_set_coords.argtypes = [C.c_void_p, C.c_int, C.c_int, _f64p]
        L.orc_set_parts.argtypes = [C.c_void_p, C.c_int, _i32p, C.c_int]
        for f in (L.orc_partition, L.orc_assemble):
            f.argtypes = [C.c_void_p, C.c_int, C.c_int, _i32p, _i32p, _f64p]
        L.orc_factorize.argtypes = [C.c_void_p]
        L.orc_solve.argtypes = [C.c_void_p, _f64p, _f64p]
        L.orc_solve_nrml.argtypes = [C.c_void_p, _f64p, _f64p]
        L.orc_get_perm.argtypes = [C.c_void_p, _i32p, _i32p]
        L.orc_log_size.restype = C.c_longlong
        L.orc_log_size.argtypes = [C.c_void_p]
        L.orc_get_log.argtypes = [C.c_void_p, _i64p]
        L.orc_num_bottom.argtypes = [C.c_void_p]
        L.orc_get_bottom.argtypes = [C.c_void_p, _i32p]
        L.orc_get_times.argtypes = [C.c_void_p, _f64p]
        L.orc_gmres.argtypes = [C.c_void_p, C.c_int, C.c_int, _i32p, _i32p, _f64p, _f64p, _f64p,
                                C.c_int, C.c_int, C.c_double, C.POINTER(C.c_int), C.POINTER(C.c_double)]
        L.orc_cgls.argtypes = [C.c_void_p, C.c_int, C.c_int, _i32p, _i32p, _f64p, _f64p, _f64p,
                               C.c_int, C.c_double, C.POINTER(C.c_int), C.POINTER(C.c_double)]
        L.orc_dgeqrf.argtypes = [C.c_int, C.c_int, _f64p, C.c_int, _f64p]
        L.orc_dlarft.argtypes = [C.c_int, C.c_int, _f64p, C.c_int, _f64p, _f64p, C.c_int]
        L.orc_dlarfb_lt.argtypes = [C.c_int, C.c_int, C.c_int, _f64p, C.c_int, _f64p, C.c_int, _f64p, C.c_int]
        L.orc_dgeqp3.argtypes = [C.c_int, C.c_int, _f64p, C.c_int, _i32p, _f64p]
        L.orc_choose_rank.argtypes = [_f64p, C.c_int, C.c_double]
        _lib = L
    return _lib


def _check(rc):
    if rc != 0:
        raise RuntimeError("oracle: " + lib().orc_last_error().decode())


def linspace_nd(n, d):
    """Grid coordinates, d x n^d column-major, first coordinate slowest
    (src/util.cpp:852-881)."""
    g = np.indices((n,) * d).reshape(d, -1).astype(np.float64)
    return np.ascontiguousarray(g.T.reshape(-1))  # column j = (x0_j, x1_j, ...)


def _csc(A):
    m, n, cp, ri, va = A
    return (int(m), int(n), np.ascontiguousarray(cp, dtype=np.int32), np.ascontiguousarray(ri, dtype=np.int32),
            np.ascontiguousarray(va, dtype=np.float64))


class OracleTree:
    """CPU restatement of Tree (include/tree.h:36-152)."""

    def __init__(self, nlevels, skip=0, tol=1e-1, scale=1, order=1.0, square=1):
        self.h = lib().orc_create(nlevels, skip, tol, scale, order, square)
        if not self.h:
            raise RuntimeError(lib().orc_last_error().decode())
        self.m = self.n = 0

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_destroy(self.h)
            self.h = None

    def set_threads(self, n):
        """Host threads for the wave-parallel factorization and solve (CPU
        baseline timing; bitwise the sequential results)."""
        _check(lib().orc_set_threads(self.h, int(n)))

    def set_coords_grid(self, n, d):
        X = linspace_nd(n, d)
        _check(lib().orc_set_coords(self.h, d, n ** d, X))

    def set_parts(self, parts, numeric_fill=True):
        """Leaf parts for the partition without coordinates (the METIS part
        vector); numeric_fill keeps the reference's numeric fill test."""
        p = np.ascontiguousarray(parts, dtype=np.int32)
        _check(lib().orc_set_parts(self.h, int(p.size), p, int(bool(numeric_fill))))

    def partition(self, A):
        m, n, cp, ri, va = _csc(A)
        self.m, self.n = m, n
        _check(lib().orc_partition(self.h, m, n, cp, ri, va))

    def assemble(self, A):
        _check(lib().orc_assemble(self.h, *_csc(A)))

    def factorize(self):
        _check(lib().orc_factorize(self.h))

    def solve(self, b):
        x = np.zeros(self.n)
        _check(lib().orc_solve(self.h, np.ascontiguousarray(b, dtype=np.float64), x))
        return x

    def solve_nrml(self, b):
        x = np.zeros(self.n)
        _check(lib().orc_solve_nrml(self.h, np.ascontiguousarray(b, dtype=np.float64), x))
        return x

    def perms(self):
        cp = np.zeros(self.n, dtype=np.int32)
        rp = np.zeros(self.m, dtype=np.int32)
        _check(lib().orc_get_perm(self.h, cp, rp))
        return cp, rp

    def log(self):
        n = lib().orc_log_size(self.h)
        out = np.zeros(n, dtype=np.int64)
        _check(lib().orc_get_log(self.h, out))
        return out.reshape(-1, 8)

    def bottom(self):
        k = lib().orc_num_bottom(self.h)
        out = np.zeros(10 * k, dtype=np.int32)
        _check(lib().orc_get_bottom(self.h, out))
        return out.reshape(-1, 10)

    def times(self):
        out = np.zeros(3)
        _check(lib().orc_get_times(self.h, out))
        return dict(partition=out[0], assemble=out[1], factorize=out[2])

    def gmres(self, A, b, iters=300, restart=None, tol=1e-12, x0=None):
        m, n, cp, ri, va = _csc(A)
        x = np.zeros(n) if x0 is None else np.array(x0, dtype=np.float64)
        its = C.c_int(0)
        res = C.c_double(0)
        _check(lib().orc_gmres(self.h, m, n, cp, ri, va, np.ascontiguousarray(b, dtype=np.float64), x, iters,
                               iters if restart is None else restart, tol, C.byref(its), C.byref(res)))
        return x, its.value, res.value

    def cgls(self, A, b, iters=300, tol=1e-12):
        m, n, cp, ri, va = _csc(A)
        x = np.zeros(n)
        its = C.c_int(0)
        res = C.c_double(0)
        _check(lib().orc_cgls(self.h, m, n, cp, ri, va, np.ascontiguousarray(b, dtype=np.float64), x, iters, tol,
                              C.byref(its), C.byref(res)))
        return x, its.value, res.value


def blas_threads(n=0):
    return lib().orc_blas_threads(n)


def run(A, b, grid_n, d, nlevels, tol, skip=0, scale=1, iters=300, res=1e-12, threads=0):
    """partition -> assemble -> factorize -> Krylov, as spaQR.cpp:249-319."""
    if threads:
        blas_threads(threads)
    square = int(A[0] == A[1])
    t = OracleTree(nlevels, skip if tol != 0 else nlevels - 1, tol, scale, 1.0, square)
    t.set_coords_grid(grid_n, d)
    t.partition(A)
    t.assemble(A)
    t.factorize()
    if square:
        x, its, r = t.gmres(A, b, iters=iters, tol=res)
    else:
        x, its, r = t.cgls(A, b, iters=iters, tol=res)
    return t, x, its, r
