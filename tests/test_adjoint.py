"""Adjoint solves for differentiation.

* M^T (spq_solve_adjoint: the factors applied transposed, sweeps reversed) is
  the transpose of M (spq_solve): u . (M v) == (M^T u) . v.
* The adjoint GMRES on A^T (spq_gmres_adjoint) reaches the FP64 CPU solution
  of A^T lambda = g (scipy's sparse LU).
* The torch.autograd wrapper's gradients of L = 1/2 ||x - x*||^2 match central
  finite differences (step 1e-6, FP64) on 64 seeded entries of b and of A's
  values, and the FP64 CPU reference gradient (lambda = A^{-T} (x - x*),
  dL/db = lambda, dL/dA_ij = -lambda_i x_j).
"""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from spaqr_public_b200 import FP32, FP64, Tree, gmres_adjoint, matgen

pytestmark = pytest.mark.gpu


def _tree(name, prec=FP64):
    w = matgen.workload(name)
    A = matgen.column_normalize(w["A"])
    t = Tree(w["levels"], w["skip"], precision=prec)
    t.set_tol(w["tol"])
    t.set_scale(1)
    t.set_square(1)
    t.set_coords_grid(w["n"], w["d"])
    t.partition(A)
    t.assemble(A)
    t.factorize()
    return w, A, t


def _csc(A):
    m, n, cp, ri, va = A
    return sp.csc_matrix((va, ri, cp), shape=(m, n))


@pytest.mark.parametrize("name,prec,tol", [("advdiff2d_32", FP64, 1e-12), ("advdiff2d_37", FP64, 1e-12),
                                           ("advdiff3d_16", FP64, 1e-12), ("advdiff2d_32", FP32, 2e-5)])
def test_adjoint_apply_is_the_transpose(gpu, name, prec, tol):
    w, A, t = _tree(name, prec)
    rng = np.random.default_rng(7)
    for _ in range(3):
        u = rng.standard_normal(A[1])
        v = rng.standard_normal(A[0])
        Mv = t.solve(v)
        Mtu = t.solve_adjoint(u)
        lhs, rhs = float(u @ Mv), float(Mtu @ v)
        scale = np.linalg.norm(u) * np.linalg.norm(Mv)
        assert abs(lhs - rhs) <= tol * scale, (lhs, rhs)
    # M^T is a good preconditioner for A^T exactly as M is for A
    As = _csc(A)
    g = rng.standard_normal(A[1])
    y = t.solve_adjoint(g)
    assert np.linalg.norm(As.T @ y - g) <= 0.5 * np.linalg.norm(g)


@pytest.mark.parametrize("name", ["advdiff2d_32", "advdiff3d_16"])
def test_adjoint_gmres_matches_cpu_solve(gpu, name):
    w, A, t = _tree(name)
    As = _csc(A)
    g = np.random.default_rng(3).standard_normal(A[1])
    lam, its, res = gmres_adjoint(A, g, t, iters=100, tol=1e-13)
    ref = spla.spsolve(As.T.tocsc(), g)
    assert its <= 100
    assert np.linalg.norm(As.T @ lam - g) <= 1e-11 * np.linalg.norm(g)
    assert np.linalg.norm(lam - ref) <= 1e-9 * np.linalg.norm(ref)


@pytest.mark.parametrize("prec", [FP64, FP32])
def test_autograd_gradients(gpu, prec):
    import torch

    from spaqr_public_b200.autograd import SparsePattern, spaqr_solve
    w, A, t = _tree("advdiff2d_32", prec)
    m, n, cp, ri, va = A
    pat = SparsePattern(A)
    rng = np.random.default_rng(2024)
    xstar_np = rng.standard_normal(n)
    inner = 1e-12 if prec == FP64 else 1e-6
    vals = torch.tensor(va, dtype=torch.float64, device="cuda", requires_grad=True)
    b = torch.tensor(w["b"], dtype=torch.float64, device="cuda", requires_grad=True)
    xstar = torch.tensor(xstar_np, dtype=torch.float64, device="cuda")
    x = spaqr_solve(vals, b, t, pat, target=1e-13, inner_tol=inner)
    L = 0.5 * ((x - xstar) ** 2).sum()
    L.backward()
    gb = b.grad.cpu().numpy()
    gA = vals.grad.cpu().numpy()

    # FP64 CPU reference gradient
    As = _csc(A)
    x_ref = spla.spsolve(As, w["b"])
    lam_ref = spla.spsolve(As.T.tocsc(), x_ref - xstar_np)
    cols = np.repeat(np.arange(n), np.diff(cp))
    gA_ref = -lam_ref[ri] * x_ref[cols]
    assert np.linalg.norm(gb - lam_ref) <= 1e-9 * np.linalg.norm(lam_ref)
    assert np.linalg.norm(gA - gA_ref) <= 1e-9 * np.linalg.norm(gA_ref)

    # central finite differences on 64 seeded entries of b and of A's values
    def loss(vv, bb):
        with torch.no_grad():
            xx = spaqr_solve(vv, bb, t, pat, target=1e-13, inner_tol=inner)
            return 0.5 * float(((xx - xstar) ** 2).sum())

    h = 1e-6
    vd = vals.detach()
    bd = b.detach()
    kb = rng.choice(m, 64, replace=False)
    ka = rng.choice(len(va), 64, replace=False)
    fd_b, fd_a = [], []
    for k in kb:
        e = torch.zeros_like(bd)
        e[k] = h
        fd_b.append((loss(vd, bd + e) - loss(vd, bd - e)) / (2 * h))
    for k in ka:
        e = torch.zeros_like(vd)
        e[k] = h
        fd_a.append((loss(vd + e, bd) - loss(vd - e, bd)) / (2 * h))
    fd_b, fd_a = np.array(fd_b), np.array(fd_a)
    assert np.max(np.abs(fd_b - gb[kb])) <= 1e-4 * max(np.max(np.abs(gb[kb])), 1.0)
    assert np.max(np.abs(fd_a - gA[ka])) <= 1e-4 * max(np.max(np.abs(gA[ka])), 1.0)
