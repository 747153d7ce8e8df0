"""Differentiable sparse solve x = A^{-1} b on the spaQR factorization.

The forward pass solves A x = b to a true FP64 residual target with GMRES
corrections preconditioned by the factorization (M ~ A^{-1}). The backward
pass is the hand-written adjoint: lambda = A^{-T} dL/dx, solved with GMRES on
A^T preconditioned by M^T (the same factors applied transposed: R^T solves,
then Q), again to a true residual target. Then

    dL/db    = lambda
    dL/dA_ij = -lambda_i x_j     for every (i, j) on the pattern of A.

This module is the package's only use of PyTorch: tensors carry the device
vectors and values, the arithmetic runs in the CUDA library behind the C ABI
(spq_solve_to_residual_dev / spq_solve_to_residual_adjoint_dev).

The factorization is a preconditioner only: it is built once from the values
the Tree was assembled with and is not differentiated. Solves with other
values on the same pattern (finite differences, optimisation steps) stay exact
to the residual target, only their iteration count depends on how far the
values moved.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._abi import SpqError, check, lib


class SparsePattern:
    """Index arrays of one sparse matrix on the device.

    Values are ordered as the CSC arrays of A (the layout the Tree was built
    from). The CSR of A (for A x) takes them through ``perm``; the CSR of A^T
    is the CSC of A itself (for A^T lambda), so it takes them as they are.
    """

    def __init__(self, A, device="cuda"):
        import torch
        m, n, cp, ri, _ = A
        cp = np.asarray(cp, dtype=np.int64)
        ri = np.asarray(ri, dtype=np.int64)
        cols = np.repeat(np.arange(n, dtype=np.int64), np.diff(cp))
        perm = np.lexsort((cols, ri))  # CSR position k <- CSC position perm[k]
        rp = np.zeros(m + 1, dtype=np.int64)
        np.add.at(rp, ri + 1, 1)
        rp = np.cumsum(rp)
        self.m, self.n = int(m), int(n)
        self.nnz = int(cp[-1])
        dev = torch.device(device)
        self.rows = torch.tensor(ri, device=dev)            # row of each CSC value
        self.cols = torch.tensor(cols, device=dev)          # column of each CSC value
        self.perm = torch.tensor(perm, device=dev)
        self.rp = torch.tensor(rp, dtype=torch.int32, device=dev)
        self.ci = torch.tensor(cols[perm], dtype=torch.int32, device=dev)
        self.rp_t = torch.tensor(cp, dtype=torch.int32, device=dev)   # CSR of A^T = CSC of A
        self.ci_t = torch.tensor(ri, dtype=torch.int32, device=dev)


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def _prepare(pat, values, rhs, adjoint):
    """Device buffers of one solve (torch's stream): values in the CSR order the
    solve needs and a zero initial guess."""
    import torch
    out = torch.zeros(pat.n if not adjoint else pat.m, dtype=torch.float64, device=rhs.device)
    vals = values.contiguous() if adjoint else values[pat.perm].contiguous()
    return vals, rhs.contiguous(), out


def _call(tree, pat, vals, rhs, out, target, inner_tol, adjoint):
    """The library solve on the handle's own stream (returns when it is done)."""
    its = C.c_int(0)
    res = C.c_double(0)
    if adjoint:
        rc = lib().spq_solve_to_residual_adjoint_dev(tree._h, pat.n, _ptr(pat.rp_t), _ptr(pat.ci_t), _ptr(vals),
                                                     _ptr(rhs), _ptr(out), float(target), float(inner_tol), 8, 300,
                                                     C.byref(its), C.byref(res))
    else:
        rc = lib().spq_solve_to_residual_dev(tree._h, pat.m, _ptr(pat.rp), _ptr(pat.ci), _ptr(vals), _ptr(rhs),
                                             _ptr(out), float(target), float(inner_tol), 8, 300, C.byref(its),
                                             C.byref(res))
    check(rc)
    return its.value, res.value


def _solve(tree, pat, values, rhs, target, inner_tol, adjoint):
    import torch
    vals, rhs, out = _prepare(pat, values, rhs, adjoint)
    torch.cuda.current_stream().synchronize()  # the library runs on the handle's own stream
    its, res = _call(tree, pat, vals, rhs, out, target, inner_tol, adjoint)
    return out, its, res


def _solve_many(trees, pats, values, rhss, target, inner_tol, adjoint, nthreads):
    """Independent solves of a batch, one host thread per handle (each handle
    has its own CUDA stream, so the solves share the GPU)."""
    import concurrent.futures as cf

    import torch
    bufs = [_prepare(p, v, r, adjoint) for p, v, r in zip(pats, values, rhss)]
    torch.cuda.current_stream().synchronize()
    with cf.ThreadPoolExecutor(max_workers=max(1, min(nthreads, len(trees)))) as ex:
        futs = [ex.submit(_call, t, p, b[0], b[1], b[2], target, inner_tol, adjoint)
                for t, p, b in zip(trees, pats, bufs)]
        for f in futs:
            f.result()
    return [b[2] for b in bufs]


def _make_function():
    import torch

    class SpaqrSolve(torch.autograd.Function):
        """x = A(values)^{-1} b with the adjoint backward described above."""

        @staticmethod
        def forward(ctx, values, b, tree, pattern, target, inner_tol):
            values = values.detach().to(torch.float64).contiguous()
            b = b.detach().to(torch.float64).contiguous()
            x, its, res = _solve(tree, pattern, values, b, target, inner_tol, adjoint=False)
            ctx.save_for_backward(values, x)
            ctx.tree, ctx.pattern, ctx.target, ctx.inner_tol = tree, pattern, target, inner_tol
            ctx.stats = {"its": its, "res": res}
            return x

        @staticmethod
        def backward(ctx, gx):
            values, x = ctx.saved_tensors
            gx = gx.detach().to(torch.float64).contiguous()
            if not bool(torch.any(gx != 0)):
                return torch.zeros_like(values), torch.zeros_like(gx), None, None, None, None
            lam, _, _ = _solve(ctx.tree, ctx.pattern, values, gx, ctx.target, ctx.inner_tol, adjoint=True)
            p = ctx.pattern
            grad_values = -lam[p.rows] * x[p.cols]
            return grad_values, lam, None, None, None, None

    return SpaqrSolve


def _make_batch_function():
    import torch

    class SpaqrSolveBatch(torch.autograd.Function):
        """x_i = A_i^{-1} b_i for a batch of independent systems; forward and
        adjoint solves of the batch run concurrently (one stream each)."""

        @staticmethod
        def forward(ctx, trees, patterns, target, inner_tol, nthreads, *tensors):
            n = len(trees)
            values = [v.detach().to(torch.float64).contiguous() for v in tensors[:n]]
            bs = [b.detach().to(torch.float64).contiguous() for b in tensors[n:]]
            xs = _solve_many(trees, patterns, values, bs, target, inner_tol, False, nthreads)
            ctx.save_for_backward(*values, *xs)
            ctx.trees, ctx.patterns, ctx.target, ctx.inner_tol, ctx.nthreads = trees, patterns, target, inner_tol, \
                nthreads
            return tuple(xs)

        @staticmethod
        def backward(ctx, *gxs):
            n = len(ctx.trees)
            saved = ctx.saved_tensors
            values, xs = saved[:n], saved[n:]
            gxs = [g.detach().to(torch.float64).contiguous() for g in gxs]
            lams = _solve_many(ctx.trees, ctx.patterns, values, gxs, ctx.target, ctx.inner_tol, True, ctx.nthreads)
            gvals = [-lam[p.rows] * x[p.cols] for lam, x, p in zip(lams, xs, ctx.patterns)]
            return (None, None, None, None, None, *gvals, *lams)

    return SpaqrSolveBatch


_FN = None
_FNB = None


def spaqr_solve_batch(values, bs, trees, patterns, target=1e-12, inner_tol=None, nthreads=32):
    """Batched :func:`spaqr_solve`: lists of values, right-hand sides, factorized
    trees and patterns of independent systems; returns the list of solutions.
    Forward and backward solves of the batch run concurrently."""
    global _FNB
    if _FNB is None:
        _FNB = _make_batch_function()
    if inner_tol is None:
        inner_tol = target
    return list(_FNB.apply(list(trees), list(patterns), target, inner_tol, nthreads, *values, *bs))



def spaqr_solve(values, b, tree, pattern, target=1e-12, inner_tol=None):
    """Differentiable x = A^{-1} b. ``values``: the nonzeros of A in CSC order of
    the pattern (FP64 CUDA tensor, requires_grad as needed); ``b``: FP64 CUDA
    vector; ``tree``: a factorized :class:`Tree` of A on the same pattern;
    ``pattern``: its :class:`SparsePattern`. ``target`` is the true relative
    residual both solves reach (forward on A, adjoint on A^T); ``inner_tol`` the
    GMRES tolerance of each correction (default: target for FP64 factors,
    1e-6 otherwise is a good choice for FP32 factors)."""
    global _FN
    if _FN is None:
        _FN = _make_function()
    if inner_tol is None:
        inner_tol = target
    return _FN.apply(values, b, tree, pattern, target, inner_tol)


__all__ = ["SparsePattern", "spaqr_solve", "spaqr_solve_batch", "SpqError"]
