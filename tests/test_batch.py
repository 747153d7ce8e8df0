"""Batched factorization and differentiation (independent systems on one GPU).

spq_factorize_batch runs each handle on its own host thread and CUDA stream;
the result of every handle must equal its own sequential factorization
(identical ranks and sizes, identical preconditioner output), and the batched
autograd solve must give the gradients of the single-system solve.
"""
import numpy as np
import pytest

from spaqr_public_b200 import FP32, FP64, Tree, factorize_batch, matgen

pytestmark = pytest.mark.gpu


def _assembled(w, prec):
    A = matgen.column_normalize(w["A"])
    t = Tree(w["levels"], w["skip"], precision=prec)
    t.set_tol(w["tol"])
    t.set_scale(1)
    t.set_square(1)
    t.set_coords_grid(w["n"], w["d"])
    t.partition(A)
    t.assemble(A)
    return A, t


@pytest.mark.parametrize("prec", [FP64, FP32])
def test_factorize_batch_equals_sequential(gpu, prec):
    ws = matgen.diff_batch(6, 24, 56, seed=77)
    seq, bat = [], []
    for w in ws:
        A, t = _assembled(w, prec)
        t.factorize()
        seq.append((A, t))
        bat.append(_assembled(w, prec))
    factorize_batch([t for _, t in bat], nthreads=6)
    for (A, ts), (_, tb), w in zip(seq, bat, ws):
        assert np.array_equal(ts.log(), tb.log())
        xs = ts.solve(w["b"])
        xb = tb.solve(w["b"])
        assert np.array_equal(xs, xb)


def test_batched_autograd_matches_single(gpu):
    import torch

    from spaqr_public_b200.autograd import SparsePattern, spaqr_solve, spaqr_solve_batch
    ws = matgen.diff_batch(4, 24, 48, seed=5)
    trees, pats, As = [], [], []
    for w in ws:
        A, t = _assembled(w, FP32)
        trees.append(t)
        pats.append(SparsePattern(A))
        As.append(A)
    factorize_batch(trees)
    vals = [torch.tensor(A[4], dtype=torch.float64, device="cuda", requires_grad=True) for A in As]
    bs = [torch.tensor(w["b"], dtype=torch.float64, device="cuda", requires_grad=True) for w in ws]
    xst = [torch.tensor(w["xstar"], dtype=torch.float64, device="cuda") for w in ws]
    xs = spaqr_solve_batch(vals, bs, trees, pats, target=1e-13, inner_tol=1e-6)
    L = sum(0.5 * ((x - s) ** 2).sum() for x, s in zip(xs, xst))
    L.backward()
    for i in range(len(ws)):
        v1 = vals[i].detach().clone().requires_grad_(True)
        b1 = bs[i].detach().clone().requires_grad_(True)
        x1 = spaqr_solve(v1, b1, trees[i], pats[i], target=1e-13, inner_tol=1e-6)
        (0.5 * ((x1 - xst[i]) ** 2).sum()).backward()
        assert torch.allclose(xs[i].detach(), x1.detach(), rtol=0, atol=1e-11 * float(x1.detach().abs().max()))
        assert torch.allclose(bs[i].grad, b1.grad, rtol=0, atol=1e-10 * float(b1.grad.abs().max()))
        assert torch.allclose(vals[i].grad, v1.grad, rtol=0, atol=1e-10 * float(v1.grad.abs().max()))
