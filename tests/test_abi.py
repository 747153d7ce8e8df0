"""C ABI: the library loads, exports every symbol include/spaqr_b200.h declares,
and validates arguments and call order without touching a GPU."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from spaqr_public_b200 import Tree, _abi, matgen

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = []
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if not fn.endswith(".h"):
            continue
        src = open(os.path.join(ROOT, "include", fn)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names += re.findall(r"\b(spq_[a-z0-9_]+)\s*\(", src)
    return sorted(set(names))


def test_header_symbols_exported():
    lib = C.CDLL(_abi.LIB_PATH)
    names = declared_symbols()
    assert len(names) >= 30
    for name in names:
        assert hasattr(lib, name), name
    # the Python binding covers every declared entry point
    assert set(names) <= set(_abi.SIGNATURES)


def test_version_and_errors():
    L = _abi.lib()
    assert L.spq_version() >= 1
    h = C.c_void_p()
    assert L.spq_create(C.byref(h), 0, 0) == 1  # SPQ_ERR_ARG
    assert b"nlevels" in L.spq_last_error()
    assert L.spq_create(None, 4, 0) == 1
    assert L.spq_create(C.byref(h), 4, 0) == 0
    assert L.spq_factorize(h) == 2  # SPQ_ERR_STATE: before assemble
    assert L.spq_set_tol(h, -1.0) == 1
    assert L.spq_set_hsl(h, 1) == 6  # SPQ_ERR_UNSUPPORTED
    assert L.spq_destroy(h) == 0
    assert L.spq_factorize(None) == 1


def test_partition_without_coordinates_uses_graph_ordering():
    A = matgen.advdiff2d(8)
    t = Tree(3, 0)
    t.partition(A)  # graph bisection of A^T A (host only)
    assert t.bottom()[:, 1].sum() == 64
    t = Tree(3, 0)
    t.set_coords(np.zeros((2, 10)))  # coordinates for 10 columns, matrix has 64
    with pytest.raises(_abi.SpqError) as e:
        t.partition(A)
    assert e.value.code == 1


def test_invalid_csc_rejected():
    t = Tree(3, 0)
    t.set_coords_grid(4, 2)
    m, n, cp, ri, va = matgen.advdiff2d(4)
    bad = ri.copy()
    bad[1], bad[0] = bad[0], bad[1]  # unsorted rows in column 0
    with pytest.raises(_abi.SpqError) as e:
        t.partition((m, n, cp, bad, va))
    assert e.value.code == 1
    bad = ri.copy()
    bad[0] = m + 3
    with pytest.raises(_abi.SpqError):
        t.partition((m, n, cp, bad, va))


def test_rectangular_needs_square_matching_off():
    A, b, _ = matgen.lsq2d(16, seed=1)
    t = Tree(4, 0)
    t.set_square(1)
    t.set_coords_grid(16, 2)
    with pytest.raises(_abi.SpqError) as e:  # identity matching of a 300 x 256 matrix
        t.partition(A)
    assert e.value.code == 6
    t = Tree(4, 0)
    t.set_coords_grid(16, 2)
    t.partition(A)  # least squares: partitions on the host
    with pytest.raises(_abi.SpqError) as e:
        t.solve_nrml(np.zeros(A[1]))
    assert e.value.code == 2


def test_setters_after_partition_rejected():
    A = matgen.column_normalize(matgen.advdiff2d(16))
    t = Tree(4, 0)
    t.set_coords_grid(16, 2)
    t.set_tol(1e-2)
    t.partition(A)
    with pytest.raises(_abi.SpqError) as e:
        t.set_tol(1e-3)
    assert e.value.code == 2
    with pytest.raises(_abi.SpqError) as e:
        t.solve(np.zeros(256))
    assert e.value.code == 2


def test_coords_grid_is_linspace_nd():
    # linspace_nd (src/util.cpp:852-881): first coordinate slowest
    from oracle.oracle_py import linspace_nd
    X = linspace_nd(3, 2).reshape(-1, 2)
    assert X[:4].tolist() == [[0, 0], [0, 1], [0, 2], [1, 0]]


def test_factorize_batch_argument_checks():
    L = _abi.lib()
    h = C.c_void_p()
    assert L.spq_create(C.byref(h), 4, 0) == 0
    arr = (C.c_void_p * 2)(h.value, h.value)
    assert L.spq_factorize_batch(arr, 2, 0) == 2  # not assembled
    assert b"not assembled" in L.spq_last_error()
    assert L.spq_factorize_batch(None, 1, 0) == 1
    assert L.spq_factorize_batch(arr, 0, 0) == 0
    assert L.spq_destroy(h) == 0
