"""The oracle's restatement of --scale 0 (CPU only).

Without block scaling the reference sparsifies with `sparsify`
(src/tree.cpp:887-989): C = [A_mp^T | (1/s) A_pp^T A_pm] with s the smallest
singular value of [A_pp; A_mp] (gesvd_values), A_pp <- A_pp Q
(ormqr_notrans_right), an `Orthogonal` op (backward only), a `Split` op and the
fine cluster eliminated at once through split_edges. The reference has no tests
or golden vectors for this path, so the restatement is checked for internal
consistency: at a tolerance near zero the preconditioner is an exact solve, the
one-shot error follows the tolerance, and GMRES converges. It is the checker
of the library's device path for --scale 0 (tests/test_gpu_scale0.py).
"""
import numpy as np
import pytest

from oracle import oracle_py as O
from spaqr_public_b200 import matgen

CASES = [("2d", 32, 5, 0), ("2d", 64, 6, 0), ("3d", 16, 6, 1)]


def _matrix(kind, n):
    return matgen.column_normalize(matgen.advdiff2d(n, seed=5) if kind == "2d" else matgen.advdiff3d(n, seed=5))


def _oracle(A, kind, n, levels, skip, tol, scale=0):
    o = O.OracleTree(levels, skip, tol, scale, 1.0, 1)
    o.set_coords_grid(n, 2 if kind == "2d" else 3)
    o.partition(A)
    o.assemble(A)
    o.factorize()
    return o


def _one_shot(o, A, b):
    x = o.solve(b)
    return np.linalg.norm(matgen.spmv(A, x) - b) / np.linalg.norm(b)


@pytest.mark.parametrize("case", CASES)
def test_scale0_near_exact_at_tiny_tolerance(case):
    kind, n, levels, skip = case
    A = _matrix(kind, n)
    b = np.random.default_rng(n).standard_normal(A[0])
    o = _oracle(A, kind, n, levels, skip, 1e-12)
    lg = o.log().reshape(-1, 8)
    assert (lg[:, 0] == 3).any()  # sparsifications ran
    assert _one_shot(o, A, b) <= 1e-11


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("tol", [1e-6, 1e-3])
def test_scale0_error_follows_tolerance(case, tol):
    kind, n, levels, skip = case
    A = _matrix(kind, n)
    b = np.random.default_rng(n).standard_normal(A[0])
    o = _oracle(A, kind, n, levels, skip, tol)
    lg = o.log().reshape(-1, 8)
    spars = lg[lg[:, 0] == 3]
    assert (spars[:, 4] < spars[:, 3]).any()  # some interface compressed
    assert _one_shot(o, A, b) <= 20 * tol


@pytest.mark.parametrize("case", CASES)
def test_scale0_gmres_converges(case):
    kind, n, levels, skip = case
    A = _matrix(kind, n)
    b = np.random.default_rng(n).standard_normal(A[0])
    o = _oracle(A, kind, n, levels, skip, 1e-2)
    x, its, res = o.gmres(A, b, tol=1e-12)
    assert its <= 20
    assert np.linalg.norm(matgen.spmv(A, x) - b) <= 1e-10 * np.linalg.norm(b)


def test_scale0_fine_clusters_are_eliminated_in_place():
    # records [type, level, order, a, b, ...]: every compressed interface
    # (sparsification, a = cols before, b = rank) is preceded by the
    # elimination of its fine cluster (a = stacked rows, b = cols before - rank)
    A = _matrix("2d", 32)
    o = _oracle(A, "2d", 32, 5, 0, 1e-3)
    lg = o.log().reshape(-1, 8)
    k = np.where((lg[:, 0] == 3) & (lg[:, 4] < lg[:, 3]))[0]
    assert len(k) > 0
    assert np.all(lg[k - 1, 0] == 1)
    assert np.array_equal(lg[k - 1, 4], lg[k, 3] - lg[k, 4])
    assert np.all(lg[k - 1, 1] == lg[k, 1])
