"""The oracle's wave-parallel mode (orc_set_threads, used to time the CPU
baseline on all host cores) against its sequential path: with one BLAS thread
the event log, the one-shot solve and the GMRES solution are bitwise the same."""
import numpy as np
import pytest

from oracle import oracle_py as O
from spaqr_public_b200 import matgen


def _run(w, A, threads):
    t = O.OracleTree(w["levels"], w["skip"], w["tol"], 1, 1.0, 1)
    t.set_threads(threads)
    t.set_coords_grid(w["n"], w["d"])
    t.partition(A)
    t.assemble(A)
    t.factorize()
    xs = t.solve(w["b"])
    x, its, res = t.gmres(A, w["b"], iters=100, tol=w["res"])
    return t.log(), xs, x, its, res


@pytest.mark.parametrize("name", ["advdiff2d_32", "advdiff3d_16", "advdiff2d_37"])
def test_parallel_oracle_is_bitwise_sequential(name):
    prev = O.blas_threads(1)
    try:
        w = matgen.workload(name)
        A = matgen.column_normalize(w["A"])
        a = _run(w, A, 1)
        b = _run(w, A, 4)
    finally:
        O.blas_threads(prev)
    assert np.array_equal(a[0], b[0])
    assert np.array_equal(a[1], b[1])
    assert np.array_equal(a[2], b[2])
    assert a[3] == b[3] and a[4] == b[4]
