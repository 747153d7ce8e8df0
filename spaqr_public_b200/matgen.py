"""Seeded synthetic sparse systems with the shapes of the spaQR benchmark workloads.

The reference reads MatrixMarket files (``spaQR.cpp:86``) produced by an external
generator that is not part of the reference repository. These generators stand in
for those files: every system is defined here by its PDE, its stencil and a seeded
random field, with unknowns numbered lexicographically with the FIRST grid
coordinate slowest (``id = i*n + j`` in 2D, ``(i*n + j)*n + k`` in 3D), which is the
numbering ``linspace_nd`` (``src/util.cpp:852-881``) assumes for ``-n/-d``.

All matrices are returned as CSC triplets ``(m, n, colptr, rowind, val)`` with
sorted row indices and no duplicates (int32 indices, float64 values).

Workloads (seed = 1000 + workload index unless given):

* ``advdiff2d(n, vmag=1000)``: -lap(u) + v.grad(u) on the unit square, Dirichlet,
  n x n interior grid, h = 1/(n+1), 5-point diffusion, first-order upwind
  advection, v = vmag*(cos t, sin t) where t(x, y) is a sum of 8 Fourier modes
  with integer frequencies <= 4.
* ``advdiff3d(n, vmag=100)``: the 3D analogue with the 7-point stencil and a unit
  direction field built from two seeded Fourier angle fields.
* ``contrast2d(n, patches=16)``: -div(a grad u) with a piecewise-constant
  coefficient on a patches x patches checkerboard, log-uniform in [1e-3, 1e3],
  harmonic-mean face coefficients.
* ``lsq2d(n, frac=0.1)``: the rectangular least-squares system [L; 10 S] with L the
  5-point Laplacian and S a seeded selection of unit rows; b = A x_true + 1e-3 noise.
"""
from __future__ import annotations

import numpy as np

__all__ = [
    "advdiff2d", "advdiff3d", "contrast2d", "lsq2d", "rhs_normal", "workload",
    "column_normalize", "to_csr", "write_mm", "read_mm", "default_levels",
]


def _fourier_field(rng, coords, nmodes=8, kmax=4, scale=np.pi):
    """Sum of ``nmodes`` sinusoidal modes with integer frequencies in [0, kmax]
    per coordinate (not all zero), seeded amplitudes and phases."""
    d = len(coords)
    freqs = []
    while len(freqs) < nmodes:
        f = rng.integers(0, kmax + 1, size=d)
        if f.any():
            freqs.append(f)
    amp = rng.normal(0.0, 1.0, size=nmodes) * scale / np.sqrt(nmodes)
    phase = rng.uniform(0.0, 2.0 * np.pi, size=nmodes)
    out = np.zeros_like(coords[0], dtype=np.float64)
    for m in range(nmodes):
        arg = phase[m]
        for c in range(d):
            arg = arg + 2.0 * np.pi * freqs[m][c] * coords[c]
        out += amp[m] * np.sin(arg)
    return out


def _assemble(nrows, ncols, rows, cols, vals):
    """COO -> CSC with sorted row indices (no duplicate entries are produced)."""
    rows = np.asarray(rows, dtype=np.int64)
    cols = np.asarray(cols, dtype=np.int64)
    vals = np.asarray(vals, dtype=np.float64)
    order = np.lexsort((rows, cols))
    rows, cols, vals = rows[order], cols[order], vals[order]
    colptr = np.zeros(ncols + 1, dtype=np.int64)
    np.add.at(colptr, cols + 1, 1)
    colptr = np.cumsum(colptr)
    return (int(nrows), int(ncols), colptr.astype(np.int32), rows.astype(np.int32), vals)


def _stencil_upwind(n, d, vel, h):
    """First-order upwind advection + central diffusion on an n^d grid.
    ``vel`` is a list of d arrays of shape (n,)*d."""
    shape = (n,) * d
    idx = np.arange(n ** d).reshape(shape)
    inv_h2 = 1.0 / (h * h)
    diag = np.full(shape, 2.0 * d * inv_h2)
    rows, cols, vals = [], [], []
    for a in range(d):
        va = vel[a]
        diag += np.abs(va) / h
        for sgn in (-1, 1):
            sl_self = [slice(None)] * d
            sl_nb = [slice(None)] * d
            if sgn < 0:
                sl_self[a] = slice(1, n)
                sl_nb[a] = slice(0, n - 1)
                coef = -inv_h2 - np.maximum(va, 0.0) / h
            else:
                sl_self[a] = slice(0, n - 1)
                sl_nb[a] = slice(1, n)
                coef = -inv_h2 + np.minimum(va, 0.0) / h
            rows.append(idx[tuple(sl_self)].ravel())
            cols.append(idx[tuple(sl_nb)].ravel())
            vals.append(coef[tuple(sl_self)].ravel())
    rows.append(idx.ravel())
    cols.append(idx.ravel())
    vals.append(diag.ravel())
    N = n ** d
    return _assemble(N, N, np.concatenate(rows), np.concatenate(cols), np.concatenate(vals))


def advdiff2d(n=128, vmag=1000.0, seed=1000):
    rng = np.random.default_rng(seed)
    h = 1.0 / (n + 1)
    g = (np.arange(n) + 1) * h
    X, Y = np.meshgrid(g, g, indexing="ij")  # X varies along the slow index i
    theta = _fourier_field(rng, [X, Y])
    vel = [vmag * np.cos(theta), vmag * np.sin(theta)]
    return _stencil_upwind(n, 2, vel, h)


def advdiff3d(n=64, vmag=100.0, seed=1001):
    rng = np.random.default_rng(seed)
    h = 1.0 / (n + 1)
    g = (np.arange(n) + 1) * h
    X, Y, Z = np.meshgrid(g, g, g, indexing="ij")
    az = _fourier_field(rng, [X, Y, Z])
    pol = 0.5 * np.pi + 0.5 * _fourier_field(rng, [X, Y, Z])
    vel = [vmag * np.sin(pol) * np.cos(az), vmag * np.sin(pol) * np.sin(az), vmag * np.cos(pol)]
    return _stencil_upwind(n, 3, vel, h)


def contrast2d(n=512, patches=16, seed=1002):
    rng = np.random.default_rng(seed)
    h = 1.0 / (n + 1)
    logs = rng.uniform(-3.0, 3.0, size=(patches, patches))
    pi = (np.arange(n) * patches) // n
    a = 10.0 ** logs[pi[:, None], pi[None, :]]
    idx = np.arange(n * n).reshape(n, n)
    inv_h2 = 1.0 / (h * h)
    diag = np.zeros((n, n))
    rows, cols, vals = [], [], []
    for axis in (0, 1):
        # interior faces between (.., k) and (.., k+1) along axis
        lo = [slice(None)] * 2
        hi = [slice(None)] * 2
        lo[axis] = slice(0, n - 1)
        hi[axis] = slice(1, n)
        al, ah = a[tuple(lo)], a[tuple(hi)]
        af = 2.0 * al * ah / (al + ah) * inv_h2
        diag[tuple(lo)] += af
        diag[tuple(hi)] += af
        rows += [idx[tuple(lo)].ravel(), idx[tuple(hi)].ravel()]
        cols += [idx[tuple(hi)].ravel(), idx[tuple(lo)].ravel()]
        vals += [-af.ravel(), -af.ravel()]
        # boundary faces use the cell coefficient
        first = [slice(None)] * 2
        last = [slice(None)] * 2
        first[axis] = slice(0, 1)
        last[axis] = slice(n - 1, n)
        diag[tuple(first)] += a[tuple(first)] * inv_h2
        diag[tuple(last)] += a[tuple(last)] * inv_h2
    rows.append(idx.ravel())
    cols.append(idx.ravel())
    vals.append(diag.ravel())
    return _assemble(n * n, n * n, np.concatenate(rows), np.concatenate(cols), np.concatenate(vals))


def lsq2d(n=256, frac=0.1, weight=10.0, noise=1e-3, seed=1003):
    """Returns ``(A, b, x_true)`` for the rectangular system [L; weight*S]."""
    rng = np.random.default_rng(seed)
    h = 1.0 / (n + 1)
    N = n * n
    zero = [np.zeros((n, n)), np.zeros((n, n))]
    m0, n0, cp, ri, va = _stencil_upwind(n, 2, zero, h)
    ksel = int(round(frac * N))
    sel = np.sort(rng.choice(N, size=ksel, replace=False))
    # L in COO
    colsL = np.repeat(np.arange(N), np.diff(cp))
    rows = np.concatenate([ri.astype(np.int64), N + np.arange(ksel)])
    cols = np.concatenate([colsL, sel])
    vals = np.concatenate([va, np.full(ksel, weight)])
    A = _assemble(N + ksel, N, rows, cols, vals)
    g = (np.arange(n) + 1) * h
    X, Y = np.meshgrid(g, g, indexing="ij")
    x_true = _fourier_field(rng, [X, Y], scale=1.0).ravel()
    b = spmv(A, x_true) + noise * rng.normal(0.0, 1.0, size=N + ksel)
    return A, b, x_true


def rhs_normal(m, seed):
    return np.random.default_rng(seed).normal(0.0, 1.0, size=m)


def spmv(A, x):
    m, n, cp, ri, va = A
    y = np.zeros(m)
    cols = np.repeat(np.arange(n), np.diff(cp))
    np.add.at(y, ri, va * x[cols])
    return y


def column_normalize(A):
    """``A <- A * diag(1/||A_j||) * 10`` exactly as ``spaQR.cpp:131-147``:
    sum of squares in stored order, d = 1/sqrt(sum), value = (v*d)*10."""
    m, n, cp, ri, va = A
    cp64 = cp.astype(np.int64)
    cnt = np.diff(cp64)
    acc = np.zeros(n)
    for k in range(int(cnt.max()) if n else 0):  # sequential order within each column
        has = cnt > k
        v = va[np.minimum(cp64[:-1] + k, len(va) - 1)]
        acc += np.where(has, v * v, 0.0)
    d = 1.0 / np.sqrt(acc)
    cols = np.repeat(np.arange(n), cnt)
    out = (va * d[cols]) * 10.0
    return (m, n, cp, ri, out)


def to_csr(A):
    """CSC -> CSR (sorted column indices)."""
    m, n, cp, ri, va = A
    cols = np.repeat(np.arange(n, dtype=np.int64), np.diff(cp))
    order = np.lexsort((cols, ri.astype(np.int64)))
    rp = np.zeros(m + 1, dtype=np.int64)
    np.add.at(rp, ri.astype(np.int64) + 1, 1)
    rp = np.cumsum(rp)
    return (m, n, rp.astype(np.int32), cols[order].astype(np.int32), va[order])


def default_levels(ncols):
    """``nlevels = ceil(log2(ncols/64))`` with the integer division of
    ``spaQR.cpp:112``."""
    return int(np.ceil(np.log2(ncols // 64)))


def workload(name):
    """Named workloads: returns dict(A, b, n, d, levels, tol, skip, res)."""
    if name == "advdiff2d_128":
        A = advdiff2d(128)
        return dict(A=A, b=rhs_normal(A[0], 2000), n=128, d=2, levels=8, tol=1e-3, skip=0, res=1e-12)
    if name == "advdiff3d_64":
        A = advdiff3d(64)
        return dict(A=A, b=rhs_normal(A[0], 2001), n=64, d=3, levels=12, tol=1e-2, skip=2, res=1e-10)
    if name.startswith("advdiff2d_"):
        n = int(name.split("_")[1])
        A = advdiff2d(n, seed=1000 + n)
        return dict(A=A, b=rhs_normal(A[0], 2000 + n), n=n, d=2, levels=default_levels(n * n),
                    tol=1e-3, skip=0, res=1e-12)
    if name.startswith("advdiff3d_"):
        n = int(name.split("_")[1])
        A = advdiff3d(n, seed=1001 + n)
        return dict(A=A, b=rhs_normal(A[0], 2001 + n), n=n, d=3, levels=default_levels(n ** 3),
                    tol=1e-2, skip=2, res=1e-10)
    if name == "contrast2d_512":
        A = contrast2d(512)
        return dict(A=A, b=rhs_normal(A[0], 2002), n=512, d=2, levels=default_levels(512 * 512),
                    tol=1e-2, skip=0, res=1e-10)
    if name == "lsq2d_256":
        A, b, _ = lsq2d(256)
        return dict(A=A, b=b, n=256, d=2, levels=default_levels(256 * 256), tol=1e-2, skip=0, res=1e-10)
    raise KeyError(name)


def diff_batch(count=32, lo=96, hi=256, seed=1004):
    """The differentiation batch: ``count`` independent 2D advection-diffusion
    systems built like advdiff2d_128 (|v| = 1000, 8 seeded Fourier modes) with
    seeded uneven sides in [lo, hi]; system i uses generator seed seed + 7 i,
    right-hand side N(0, 1) and target x* ~ N(0, 1). Returns a list of dicts
    as :func:`workload` plus ``xstar``."""
    rng = np.random.default_rng(seed)
    sides = rng.integers(lo, hi + 1, size=count)
    out = []
    for i, n in enumerate(sides):
        n = int(n)
        A = advdiff2d(n, seed=seed + 7 * i)
        out.append(dict(A=A, b=rhs_normal(A[0], seed + 7 * i + 1), xstar=rhs_normal(n * n, seed + 7 * i + 2), n=n,
                        d=2, levels=default_levels(n * n), tol=1e-3, skip=0, res=1e-12))
    return out


def write_mm(path, A):
    m, n, cp, ri, va = A
    nnz = len(va)
    cols = np.repeat(np.arange(n), np.diff(cp))
    with open(path, "w") as f:
        f.write("%%MatrixMarket matrix coordinate real general\n")
        f.write(f"{m} {n} {nnz}\n")
        for r, c, v in zip(ri, cols, va):
            f.write(f"{int(r) + 1} {int(c) + 1} {float(v)!r}\n")


def read_mm(path):
    with open(path) as f:
        header = f.readline()
        assert header.startswith("%%MatrixMarket")
        line = f.readline()
        while line.startswith("%"):
            line = f.readline()
        m, n, nnz = map(int, line.split())
        data = np.loadtxt(f, ndmin=2)
    rows = data[:, 0].astype(np.int64) - 1
    cols = data[:, 1].astype(np.int64) - 1
    return _assemble(m, n, rows, cols, data[:, 2])
