"""Index arrays of the differentiable solve (no GPU): the CSR of A and of A^T
built from A's CSC layout, and the gradient scatter positions."""
import numpy as np
import scipy.sparse as sp

from spaqr_public_b200 import matgen
from spaqr_public_b200.autograd import SparsePattern


def test_pattern_csr_of_a_and_transpose():
    w = matgen.workload("advdiff2d_32")
    m, n, cp, ri, va = w["A"]
    p = SparsePattern(w["A"], device="cpu")
    Acsr = sp.csc_matrix((va, ri, cp), shape=(m, n)).tocsr()
    Acsr.sort_indices()
    assert np.array_equal(p.rp.numpy(), Acsr.indptr)
    assert np.array_equal(p.ci.numpy(), Acsr.indices)
    assert np.array_equal(np.asarray(va)[p.perm.numpy()], Acsr.data)
    # CSR of A^T is the CSC of A: same arrays
    At = sp.csr_matrix((va, ri, cp), shape=(n, m))
    assert np.array_equal(p.rp_t.numpy(), At.indptr) and np.array_equal(p.ci_t.numpy(), At.indices)
    # gradient positions: value k sits at (rows[k], cols[k])
    D = sp.coo_matrix((np.arange(1, len(va) + 1, dtype=float), (p.rows.numpy(), p.cols.numpy())), shape=(m, n))
    assert np.array_equal(D.tocsc().data, np.arange(1, len(va) + 1, dtype=float))
