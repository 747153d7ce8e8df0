"""GPU factorization on the ordering without coordinates, against the oracle.

No coordinates are set: the library orders the matrix from its own bisection of
the A^T A graph through the reference's MetisPartition / getInterfacesUsingATA
steps, and applies the reference's numeric fill test (a candidate is kept only
if ||A1^T A2|| > 1e-14, src/tree.cpp:856-859) on the device. The oracle gets
the same part vector and the same fill rule; the second rule (keep every
candidate, spq_set_fill_rule 0) is checked against the oracle with the test off.

Bar (FP64): event log identical, one-shot solve within 1e-10 relative, GMRES
(square) or CGLS (least squares) iteration counts identical. FP32 factor: the
refinement driver reaches 1e-10.
"""
import os
import re
import subprocess

import numpy as np
import pytest

from oracle import oracle_py as O
from spaqr_public_b200 import FP32, FP64, Tree, cgls, gmres, graph_parts, matgen, solve_to_residual

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "spaqr_public_b200", "_build", "spaqr")


def _pair(A, levels, tol, skip, square=1, prec=FP64, numeric=True):
    t = Tree(levels, skip, precision=prec)
    t.set_tol(tol)
    t.set_scale(1)
    t.set_square(square)
    if not numeric:
        t.set_fill_rule(0)
    t.partition(A)
    t.assemble(A)
    t.factorize()
    o = O.OracleTree(levels, skip, tol, 1, 1.0, square)
    o.set_parts(graph_parts(A, levels), numeric_fill=numeric)
    o.partition(A)
    o.assemble(A)
    o.factorize()
    return t, o


@pytest.mark.parametrize("numeric", [True, False])
@pytest.mark.parametrize("kind,n,levels,tol,skip", [("2d", 64, 6, 1e-3, 0), ("3d", 16, 6, 1e-2, 1)])
def test_graph_ordering_log_solve_gmres_match_oracle(gpu, kind, n, levels, tol, skip, numeric):
    A = matgen.column_normalize(matgen.advdiff2d(n, seed=5) if kind == "2d" else matgen.advdiff3d(n, seed=5))
    t, o = _pair(A, levels, tol, skip, numeric=numeric)
    assert np.array_equal(t.log(), o.log())
    b = np.random.default_rng(n).standard_normal(A[0])
    x = t.solve(b)
    xo = o.solve(b)
    assert np.linalg.norm(x - xo) <= 1e-10 * np.linalg.norm(xo)
    x, its, res = gmres(A, b, t, iters=300, tol=1e-12)
    xo, itso, reso = o.gmres(A, b, tol=1e-12)
    assert its == itso
    assert np.linalg.norm(matgen.spmv(A, x) - b) <= 1e-11 * np.linalg.norm(b)


def test_graph_ordering_least_squares_matches_oracle(gpu):
    A, b, _ = matgen.lsq2d(24, seed=29)
    A = matgen.column_normalize(A)
    t, o = _pair(A, 5, 1e-2, 0, square=0)
    assert np.array_equal(t.log(), o.log())
    x, its, res = cgls(A, b, t, iters=200, tol=1e-10)
    xo, ito, _ = o.cgls(A, b, iters=200, tol=1e-10)
    assert its == ito
    assert res <= 1e-10
    assert np.linalg.norm(x - xo) <= 1e-8 * np.linalg.norm(xo)


def test_graph_ordering_fp32_refinement(gpu):
    A = matgen.column_normalize(matgen.advdiff2d(64, seed=5))
    t = Tree(6, 0, precision=FP32)
    t.set_tol(1e-3)
    t.set_scale(1)
    t.set_square(1)
    t.partition(A)
    t.assemble(A)
    t.factorize()
    b = np.random.default_rng(3).standard_normal(A[0])
    x, _, res = solve_to_residual(A, b, t, target=1e-10)
    assert np.linalg.norm(matgen.spmv(A, x) - b) <= 1e-10 * np.linalg.norm(b)


def test_cli_without_coordinates(gpu, tmp_path):
    w = matgen.workload("advdiff2d_64")
    mtx = tmp_path / "A.mtx"
    matgen.write_mm(mtx, w["A"])
    p = subprocess.run([CLI, "-m", str(mtx), "-l", "6", "-t", "1e-3", "--res", "1e-12"], capture_output=True,
                       text=True, timeout=600)
    assert p.returncode == 0, p.stderr
    assert "Using graph bisection partition" in p.stdout
    m = re.search(r"<<<<GMRES=(\d+)", p.stdout)
    assert m and int(m.group(1)) <= 20
    res = float(re.search(r"residual \|Ax-b\|/\|b\|: ([0-9.eE+-]+)", p.stdout).group(1))
    assert res <= 1e-11
