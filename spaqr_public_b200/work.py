"""Algorithmic work of a factorization, from its event log.

The event log (one record of 8 int64 per task: [type, level, order, a, b, c, d, e])
holds every task shape, so the algorithmic flop count follows from the usual
LAPACK operation counts:

* geqrf m x n:                       2 m n^2 - 2/3 n^3
* larft, k reflectors of length m:   m k^2
* larfb, k reflectors on m x n:      4 m n k - n k^2
* trsm, m x n by n x n:              m n^2
* column-pivoted QR of m x n, stopped after r steps:
                                     4 m n r - 2 r^2 (m + n) + 4/3 r^3

The device RRQR stops at the rank (r steps, plus the last norm test); the
reference's dgeqp3 always runs min(m, n) steps.
"""
from __future__ import annotations

import numpy as np

ELIM, SCALE, SPARS, MERGE, LEVEL, FINAL = 1, 2, 3, 4, 5, 6


def geqrf(m, n):
    return 2.0 * m * n * n - 2.0 / 3.0 * n ** 3


def larft(m, k):
    return float(m) * k * k


def larfb(m, n, k):
    return 4.0 * m * n * k - float(n) * k * k


def rrqr(m, n, r):
    return 4.0 * m * n * r - 2.0 * r * r * (m + n) + 4.0 / 3.0 * r ** 3


def phase_flops(log, reference=False):
    """Flops per phase: dict(elim, scale, sparsify)."""
    log = np.asarray(log).reshape(-1, 8)
    out = dict(elim=0.0, scale=0.0, sparsify=0.0)
    for t, _lvl, _o, a, b, c, d, e in log:
        if t == ELIM and b > 0:
            out["elim"] += geqrf(a, b) + larft(a, b) + larfb(a, e, b)
        elif t == SCALE and b > 0:
            wrow, hcol = divmod(int(e), 100000)
            out["scale"] += geqrf(a, b) + larft(a, b) + larfb(a, wrow, b) + float(hcol) * b * b
        elif t == SPARS and a > 0 and c > 0:
            m, r, n = int(a), int(b), int(c)
            steps = min(m, n) if (reference or r >= m) else r
            out["sparsify"] += rrqr(m, n, steps)
    return out


def total_flops(log, reference=False):
    return sum(phase_flops(log, reference).values())


def factor_bytes(log):
    """nnzR + nnzH + nnzQ of the FINAL record: the factor words one solve reads."""
    log = np.asarray(log).reshape(-1, 8)
    fin = log[log[:, 0] == FINAL]
    if len(fin) == 0:
        return 0
    return int(fin[-1, 4] + fin[-1, 5] + fin[-1, 6])
