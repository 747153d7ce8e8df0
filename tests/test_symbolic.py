"""Host symbolic layer of the product vs the oracle (CPU only, bit-exact):
nested-dissection permutations and the bottom clusters (ids, sizes, offsets).
The product's partition runs on the host and does not open the GPU."""
import numpy as np
import pytest

from oracle import oracle_py as O
from spaqr_public_b200 import Tree, matgen


def _compare(A, n, d, levels, square=1):
    t = Tree(levels, 0)
    t.set_tol(1e-2)
    t.set_scale(1)
    t.set_square(square)
    t.set_coords_grid(n, d)
    t.partition(A)
    o = O.OracleTree(levels, 0, 1e-2, 1, 1.0, square)
    o.set_coords_grid(n, d)
    o.partition(A)
    cp, rp = t.perms()
    ocp, orp = o.perms()
    assert np.array_equal(cp, ocp)
    assert np.array_equal(rp, orp)
    assert np.array_equal(t.bottom(), o.bottom())
    return t


@pytest.mark.parametrize("n,levels", [(32, 4), (37, 5), (64, 6), (128, 8), (20, 1), (20, 2)])
def test_partition_2d(n, levels):
    A = matgen.column_normalize(matgen.advdiff2d(n, seed=7 + n))
    _compare(A, n, 2, levels)


@pytest.mark.parametrize("n,levels", [(12, 5), (16, 6), (24, 8), (32, 9)])
def test_partition_3d(n, levels):
    A = matgen.column_normalize(matgen.advdiff3d(n, seed=11 + n))
    _compare(A, n, 3, levels)


def test_partition_high_contrast():
    A = matgen.column_normalize(matgen.contrast2d(64, patches=8, seed=3))
    _compare(A, 64, 2, 6)


def test_partition_too_many_levels():
    # more bisections than unknowns: empty parts must not break the ordering
    A = matgen.column_normalize(matgen.advdiff2d(6, seed=1))
    _compare(A, 6, 2, 7)


def test_bottom_clusters_cover_all_columns():
    A = matgen.column_normalize(matgen.advdiff2d(32, seed=9))
    t = _compare(A, 32, 2, 5)
    b = t.bottom()
    assert b[:, 1].sum() == 32 * 32
    assert np.all(np.diff(b[:, 0]) == b[:-1, 1])  # contiguous column ranges
    assert np.all(b[:, 1] == b[:, 3])  # square input: rows == cols per cluster


def test_column_normalize_matches_reference_formula():
    from spaqr_public_b200 import column_normalize
    A = matgen.advdiff2d(16, seed=2)
    B = column_normalize(A)
    C = matgen.column_normalize(A)
    assert np.array_equal(B[4], C[4])
    m, n, cp, ri, va = B
    for j in range(n):
        assert abs(np.linalg.norm(va[cp[j]:cp[j + 1]]) - 10.0) < 1e-12


@pytest.mark.parametrize("n,levels", [(16, 4), (24, 5), (32, 5)])
def test_partition_least_squares(n, levels):
    # rectangular [L; 10 S]: rows join the first column of their largest-norm cluster run
    A, _, _ = matgen.lsq2d(n, seed=5 + n)
    t = _compare(A, n, 2, levels, square=0)
    b = t.bottom()
    assert b[:, 3].sum() == A[0] and b[:, 1].sum() == A[1]
