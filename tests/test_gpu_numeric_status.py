"""Numeric failure detection on the device (a status word the QR and RRQR
kernels set): a NaN in A's values, or an exactly singular block, makes the
factorization return SPQ_ERR_NUMERIC with the cause, instead of a factor full
of NaN. The reference has no such check (Tree::factorize returns 0 always,
src/tree.cpp:1436). The failures are made on the host (the values handed to
the library); no kernel faults."""
import numpy as np
import pytest

from spaqr_public_b200 import FP32, FP64, Tree, matgen
from spaqr_public_b200._abi import SpqError

pytestmark = pytest.mark.gpu


def _tree(w, A, prec):
    t = Tree(w["levels"], w["skip"], precision=prec)
    t.set_tol(w["tol"])
    t.set_scale(1)
    t.set_square(1)
    t.set_coords_grid(w["n"], w["d"])
    t.partition(A)
    t.assemble(A)
    return t


@pytest.mark.parametrize("prec", [FP64, FP32])
@pytest.mark.parametrize("name", ["advdiff2d_32", "advdiff3d_16"])
def test_nan_in_values_is_reported(gpu, prec, name):
    w = matgen.workload(name)
    m, n, cp, ri, va = matgen.column_normalize(w["A"])
    va = va.copy()
    va[len(va) // 3] = np.nan
    t = _tree(w, (m, n, cp, ri, va), prec)
    with pytest.raises(SpqError) as e:
        t.factorize()
    assert e.value.code == 4  # SPQ_ERR_NUMERIC
    assert "NaN or Inf" in str(e.value)


@pytest.mark.parametrize("prec", [FP64, FP32])
def test_zero_column_is_a_zero_pivot(gpu, prec):
    # a column of A that is exactly zero: the elimination of its cluster meets
    # an exactly zero pivot (A is singular). Column 0 is the grid's corner
    # point, inside a leaf interior, eliminated at level 0 before any scaling
    # or sparsification mixes columns.
    w = matgen.workload("advdiff2d_32")
    m, n, cp, ri, va = matgen.column_normalize(w["A"])
    va = va.copy()
    j = 0
    va[cp[j]:cp[j + 1]] = 0.0
    t = _tree(w, (m, n, cp, ri, va), prec)
    with pytest.raises(SpqError) as e:
        t.factorize()
    assert e.value.code == 4
    assert "zero pivot" in str(e.value)


def test_healthy_factorization_has_clean_status(gpu):
    w = matgen.workload("advdiff2d_32")
    A = matgen.column_normalize(w["A"])
    t = _tree(w, A, FP64)
    t.factorize()  # no exception
    x = t.solve(w["b"])
    assert np.all(np.isfinite(x))
