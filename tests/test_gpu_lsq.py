"""Least squares on the GPU (rectangular A = [L; 10 S], square matching off)
against the oracle: the per-level event log (elimination shapes, row shifts
of reassign_rows, extra-row compressions of sparsify_extra, scaling and RRQR
ranks, merges, nnz counters), the preconditioner M_n ~ (A^T A)^{-1}
(solve_nrml) and the CGLS iterations and solution."""
import numpy as np
import pytest

from oracle import oracle_py as O
from spaqr_public_b200 import FP32, FP64, Tree, cgls, matgen

pytestmark = pytest.mark.gpu


def _setup(n, levels, tol=1e-2, skip=0, prec=FP64):
    A, b, _ = matgen.lsq2d(n, seed=5 + n)
    A = matgen.column_normalize(A)
    t = Tree(levels, skip, precision=prec)
    t.set_tol(tol)
    t.set_scale(1)
    t.set_coords_grid(n, 2)
    t.partition(A)
    t.assemble(A)
    t.factorize()
    o = O.OracleTree(levels, skip, tol, 1, 1.0, 0)
    o.set_coords_grid(n, 2)
    o.partition(A)
    o.assemble(A)
    o.factorize()
    return A, b, t, o


@pytest.mark.parametrize("n,levels,tol", [(16, 4, 1e-2), (24, 5, 1e-2), (32, 5, 1e-1), (32, 6, 1e-3)])
def test_lsq_log_and_solve_nrml_match_oracle(gpu, n, levels, tol):
    A, b, t, o = _setup(n, levels, tol)
    lg, lo = t.log(), o.log()
    assert lg.shape == lo.shape
    assert np.array_equal(lg, lo)
    kinds = set(lo[:, 0].tolist())
    assert 7 in kinds  # rows moved by reassign_rows
    g = np.random.default_rng(n).standard_normal(A[1])
    x = t.solve_nrml(g)
    xo = o.solve_nrml(g)
    assert np.linalg.norm(x - xo) <= 1e-10 * np.linalg.norm(xo)


@pytest.mark.parametrize("n,levels", [(24, 5), (32, 6)])
def test_lsq_cgls_matches_oracle(gpu, n, levels):
    A, b, t, o = _setup(n, levels)
    x, its, res = cgls(A, b, t, iters=200, tol=1e-10)
    xo, ito, reso = o.cgls(A, b, iters=200, tol=1e-10)
    assert its == ito
    assert res <= 1e-10
    assert np.linalg.norm(x - xo) <= 1e-8 * np.linalg.norm(xo)


def test_lsq_fp32_factor_cgls_converges(gpu):
    A, b, t, o = _setup(32, 6, prec=FP32)
    x, its, res = cgls(A, b, t, iters=300, tol=1e-10)
    xo, ito, _ = o.cgls(A, b, iters=300, tol=1e-10)
    assert res <= 1e-10
    assert its <= 3 * ito + 5
    assert np.linalg.norm(x - xo) <= 1e-7 * np.linalg.norm(xo)
