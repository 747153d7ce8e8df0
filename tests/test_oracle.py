"""CPU oracle checks: its LAPACK kernels, its rank rule, its end-to-end solve,
and its event log against the committed fixtures.

The reference ships no tests or golden vectors and cannot be built here (no
Eigen), so the fixtures under tests/golden are produced by the oracle itself
(tests/golden/make_golden.py) and pin it against regressions: parity with the
reference is unpinned.
"""
import json
import os

import numpy as np
import pytest

from oracle import oracle_py as O
from spaqr_public_b200 import matgen

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def rng(seed=0):
    return np.random.default_rng(seed)


def test_dgeqrf_larft_larfb_reconstruct():
    m, n = 37, 11
    A = rng(1).normal(size=(m, n))
    a = np.asfortranarray(A).copy().ravel(order="F")
    tau = np.zeros(n)
    assert O.lib().orc_dgeqrf(m, n, a, m, tau) == 0
    F = a.reshape((m, n), order="F")
    R = np.triu(F[:n, :])
    V = np.tril(F, -1)
    V[np.arange(n), np.arange(n)] = 1.0
    T = np.zeros(n * n)
    assert O.lib().orc_dlarft(m, n, np.ascontiguousarray(V.ravel(order="F")), m, tau, T, n) == 0
    T = T.reshape((n, n), order="F")
    H = np.eye(m) - V @ T @ V.T
    assert np.allclose(H @ np.vstack([R, np.zeros((m - n, n))]), A, atol=1e-12)
    # larfb applies H^T
    C = rng(2).normal(size=(m, 5))
    c = C.ravel(order="F").copy()
    assert O.lib().orc_dlarfb_lt(m, 5, n, np.ascontiguousarray(V.ravel(order="F")), m,
                                 np.ascontiguousarray(T.ravel(order="F")), n, c, m) == 0
    assert np.allclose(c.reshape((m, 5), order="F"), H.T @ C, atol=1e-12)


def test_dgeqp3_pivots_and_rank():
    m, n = 12, 30
    U = rng(3).normal(size=(m, 4))
    W = rng(4).normal(size=(4, n))
    A = U @ W + 1e-9 * rng(5).normal(size=(m, n))
    a = A.ravel(order="F").copy()
    jp = np.zeros(n, dtype=np.int32)
    tau = np.zeros(m)
    assert O.lib().orc_dgeqp3(m, n, a, m, jp, tau) == 0
    assert sorted(jp.tolist()) == list(range(n))
    R = np.triu(a.reshape((m, n), order="F")[:m, :])
    d = np.abs(np.diag(R))
    assert np.all(d[:-1] >= d[1:] * (1 - 1e-12))  # non-increasing |R_kk|
    assert O.lib().orc_choose_rank(np.ascontiguousarray(np.diag(R)), m, 1e-6) == 4


@pytest.mark.parametrize("tol,expect", [(0.0, 5), (1.0, 0), (0.5, 2), (1e-3, 4)])
def test_choose_rank_rule(tol, expect):
    # src/util.cpp:795-816
    s = np.array([-2.0, 1.5, 0.9, 0.01, 1e-4])
    assert O.lib().orc_choose_rank(s, 5, tol) == expect


def test_choose_rank_single():
    assert O.lib().orc_choose_rank(np.array([0.0]), 1, 1e-3) == 1


def _run_small(name):
    w = matgen.workload(name)
    A = matgen.column_normalize(w["A"])
    t, x, its, r = O.run(A, w["b"], w["n"], w["d"], w["levels"], w["tol"], w["skip"], res=w["res"])
    return w, A, t, x, its, r


def test_oracle_gmres_converges_2d():
    w, A, t, x, its, r = _run_small("advdiff2d_32")
    res = np.linalg.norm(matgen.spmv(A, x) - w["b"]) / np.linalg.norm(w["b"])
    assert res < 1e-11
    assert its <= 10


@pytest.mark.parametrize("name", ["advdiff2d_32", "advdiff3d_16"])
def test_oracle_log_matches_fixture(name):
    with open(os.path.join(GOLD, f"{name}.json")) as f:
        g = json.load(f)
    w, A, t, x, its, r = _run_small(name)
    log = t.log()
    assert np.array_equal(log, np.array(g["log"], dtype=np.int64).reshape(-1, 8))
    cp, rp = t.perms()
    assert cp.tolist() == g["cperm"]
    assert its == g["gmres_its"]
    assert abs(r - g["gmres_res"]) <= 1e-3 * g["gmres_res"] + 1e-16


def test_oracle_tol_zero_is_exact_qr():
    """tol = 0: no sparsification (skip = nlevels-1), the preconditioner is an exact QR."""
    w = matgen.workload("advdiff2d_32")
    A = matgen.column_normalize(w["A"])
    t = O.OracleTree(w["levels"], w["levels"] - 1, 0.0, 1, 1.0, 1)
    t.set_coords_grid(w["n"], w["d"])
    t.partition(A)
    t.assemble(A)
    t.factorize()
    x = t.solve(w["b"])
    assert np.linalg.norm(matgen.spmv(A, x) - w["b"]) / np.linalg.norm(w["b"]) < 1e-12
    log = t.log()
    assert not np.any(log[:, 0] == 3)  # no sparsification records


def test_default_levels_matches_reference_transcript():
    # README.md:51-52: 16384 columns -> "Levels set to ceil(log2(ncols/64)) = 8"
    assert matgen.default_levels(16384) == 8
    A = matgen.advdiff2d(128)
    assert len(A[4]) == 81408  # nnzA of a 128^2 5-point matrix (README.md:74)
