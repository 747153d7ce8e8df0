"""--scale 0 on the GPU (sparsify, src/tree.cpp:887-989, square systems)
against the oracle's restatement: sinv = 1 / sigma_min([A_pp; A_mp]) (QR of
the stacked column, one-sided Jacobi on its R; the oracle: LAPACK gesvd),
the RRQR of C = [A_mp^T | sinv A_pp^T A_pm], A_pp <- A_pp Q, the split of the
interface's row and diagonal block (split_edges) and the immediate
elimination of the fine cluster.

Bar (FP64): event log identical (every fine elimination, every RRQR rank,
merges, nnz counters), one-shot solve within 1e-10 relative, GMRES iteration
count identical; the FP32 factor reaches a true residual of 1e-10 through the
refinement; the transposed application is the transpose (adjoint solves).
"""
import numpy as np
import pytest

from oracle import oracle_py as O
from spaqr_public_b200 import FP32, FP64, Tree, gmres, matgen, solve_to_residual

pytestmark = pytest.mark.gpu

CASES = [("2d", 32, 5, 0, 1e-3), ("2d", 64, 6, 0, 1e-3), ("3d", 16, 6, 1, 1e-2), ("2d", 64, 6, 0, 1e-1)]


def _matrix(kind, n):
    return matgen.column_normalize(matgen.advdiff2d(n, seed=5) if kind == "2d" else matgen.advdiff3d(n, seed=5))


def _pair(kind, n, levels, skip, tol, prec=FP64):
    A = _matrix(kind, n)
    d = 2 if kind == "2d" else 3
    t = Tree(levels, skip, precision=prec)
    t.set_tol(tol)
    t.set_scale(0)
    t.set_square(1)
    t.set_coords_grid(n, d)
    t.partition(A)
    t.assemble(A)
    t.factorize()
    o = O.OracleTree(levels, skip, tol, 0, 1.0, 1)
    o.set_coords_grid(n, d)
    o.partition(A)
    o.assemble(A)
    o.factorize()
    return A, t, o


@pytest.mark.parametrize("case", CASES)
def test_scale0_log_solve_gmres_match_oracle(gpu, case):
    A, t, o = _pair(*case)
    lg, lo = t.log(), o.log()
    assert lg.shape == lo.shape
    bad = np.where((lg != lo).any(axis=1))[0]
    assert bad.size == 0, f"{bad.size} records differ, first: device {lg[bad[:3]].tolist()} oracle {lo[bad[:3]].tolist()}"
    b = np.random.default_rng(case[1]).standard_normal(A[0])
    x = t.solve(b)
    xo = o.solve(b)
    assert np.linalg.norm(x - xo) <= 1e-10 * np.linalg.norm(xo)
    x, its, res = gmres(A, b, t, iters=300, tol=1e-12)
    xo, itso, reso = o.gmres(A, b, tol=1e-12)
    assert its == itso
    assert np.linalg.norm(matgen.spmv(A, x) - b) <= 1e-11 * np.linalg.norm(b)


def test_scale0_fp32_refinement(gpu):
    A, t, _ = _pair("2d", 64, 6, 0, 1e-3, prec=FP32)
    b = np.random.default_rng(9).standard_normal(A[0])
    x, its, res = solve_to_residual(A, b, t, target=1e-10, inner_tol=1e-6)
    assert np.linalg.norm(matgen.spmv(A, x) - b) <= 1e-10 * np.linalg.norm(b)


def test_scale0_adjoint_is_the_transpose(gpu):
    A, t, _ = _pair("2d", 32, 5, 0, 1e-3)
    rng = np.random.default_rng(4)
    for _ in range(3):
        u = rng.standard_normal(A[1])
        v = rng.standard_normal(A[0])
        Mv = t.solve(v)
        Mtu = t.solve_adjoint(u)
        assert abs(u @ Mv - Mtu @ v) <= 1e-12 * np.linalg.norm(u) * np.linalg.norm(Mv)
