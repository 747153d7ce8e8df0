"""Ordering without coordinates (CPU only).

The reference orders a matrix without coordinates from a METIS (or PaToH) leaf
part vector: MetisPartition (src/partition.cpp:374-426) turns the parts into
separators, getInterfacesUsingATA (src/partition.cpp:628-675) gives every
separator column its two sides, and Tree::partition sorts and groups them.
METIS is absent, so the library supplies the part vector with its own recursive
bisection of the A^T A graph (or takes one from the caller). Checked here:

* the product's separators, interfaces, permutations and bottom clusters are
  bit-exact with the oracle's restatement of those reference steps, on the
  same part vector (the library's own, and caller-supplied ones);
* the bisection is deterministic, balanced, and its top separator is close to
  the geometric one on a grid; coupled columns never sit in disjoint subtrees;
* the oracle's factorization on this ordering: the reference's numeric fill
  test (src/tree.cpp:857-860) against the library's rule (every candidate that
  passes the separator tests is kept) gives the same ranks and Krylov
  iteration counts;
* argument errors of the C ABI.
"""
import numpy as np
import pytest
import scipy.sparse as sp

from oracle import oracle_py as O
from spaqr_public_b200 import Tree, graph_parts, matgen
from spaqr_public_b200._abi import SpqError


def _compare(A, levels, parts=None, square=1):
    p = graph_parts(A, levels) if parts is None else np.asarray(parts, dtype=np.int32)
    t = Tree(levels, 0)
    t.set_tol(1e-2)
    t.set_scale(1)
    t.set_square(square)
    if parts is not None:
        t.set_parts(p)
    t.partition(A)
    o = O.OracleTree(levels, 0, 1e-2, 1, 1.0, square)
    o.set_parts(p)
    o.partition(A)
    cp, rp = t.perms()
    ocp, orp = o.perms()
    assert np.array_equal(cp, ocp)
    assert np.array_equal(rp, orp)
    assert np.array_equal(t.bottom(), o.bottom())
    return t, p


@pytest.mark.parametrize("n,levels", [(32, 4), (37, 5), (64, 6), (128, 8), (20, 1), (20, 2)])
def test_graph_ordering_2d_matches_oracle(n, levels):
    A = matgen.column_normalize(matgen.advdiff2d(n, seed=7 + n))
    _compare(A, levels)


@pytest.mark.parametrize("n,levels", [(12, 5), (16, 6), (24, 8)])
def test_graph_ordering_3d_matches_oracle(n, levels):
    A = matgen.column_normalize(matgen.advdiff3d(n, seed=11 + n))
    _compare(A, levels)


def test_graph_ordering_least_squares_matches_oracle():
    A, _, _ = matgen.lsq2d(32, seed=37)
    A = matgen.column_normalize(A)
    t, _ = _compare(A, 6, square=0)
    b = t.bottom()
    assert b[:, 3].sum() == A[0]  # every row joins one cluster


def test_graph_ordering_too_many_levels():
    # more leaf parts than unknowns: empty parts must not break the ordering
    A = matgen.column_normalize(matgen.advdiff2d(6, seed=1))
    _compare(A, 7)


def test_caller_supplied_parts():
    # a planted part vector (recursive halving of the grid rows, first cut in
    # the highest bit), as a METIS run would hand it over
    n, levels = 32, 5
    A = matgen.column_normalize(matgen.advdiff2d(n, seed=2))
    rows = np.arange(n * n) // n
    parts = np.minimum(rows * (1 << (levels - 1)) // n, (1 << (levels - 1)) - 1)
    _compare(A, levels, parts=parts)


def test_bisection_deterministic_and_balanced():
    A = matgen.column_normalize(matgen.advdiff3d(16, seed=4))
    p1 = graph_parts(A, 6)
    p2 = graph_parts(A, 6)
    assert np.array_equal(p1, p2)
    counts = np.bincount(p1, minlength=32)
    assert counts.min() > 0
    # every cut keeps its side 0 within |set|/200 + 1 of ceil(|set|/2)
    assert counts.max() - counts.min() <= 0.1 * counts.mean()


def test_bisection_top_separator_near_geometric():
    n, levels = 64, 6
    A = matgen.column_normalize(matgen.advdiff2d(n, seed=5))
    t, _ = _compare(A, levels)
    b = t.bottom()
    top = b[b[:, 4] == levels - 1][:, 1].sum()
    assert top <= 1.1 * (2 * n - 2)  # geometric: two cells thick, 2n - 2 columns


def _oracle_run(A, levels, tol, skip, parts=None, numeric_fill=True, grid=None):
    o = O.OracleTree(levels, skip, tol, 1, 1.0, 1)
    if parts is None:
        o.set_coords_grid(*grid)
    else:
        o.set_parts(parts, numeric_fill)
    o.partition(A)
    o.assemble(A)
    o.factorize()
    b = np.random.default_rng(levels).standard_normal(A[0])
    x, its, res = o.gmres(A, b, tol=1e-12)
    return o.log().reshape(-1, 8), its, res, x


@pytest.mark.parametrize("case", [("2d", 64, 6, 1e-3, 0), ("3d", 16, 6, 1e-2, 1)])
def test_fill_rule_same_ranks_and_iterations(case):
    kind, n, levels, tol, skip = case
    A = matgen.column_normalize(matgen.advdiff2d(n, seed=5) if kind == "2d" else matgen.advdiff3d(n, seed=5))
    p = graph_parts(A, levels)
    lg_ref, its_ref, res_ref, x_ref = _oracle_run(A, levels, tol, skip, parts=p, numeric_fill=True)
    lg, its, res, x = _oracle_run(A, levels, tol, skip, parts=p, numeric_fill=False)
    # records [type, level, order, a, b, c, d, e]: the same eliminations
    # (rows, cols), scalings, merges and sparsifications (cols before, rank,
    # rows); only the updated-cluster counts, RRQR widths and the nnz counters
    # grow by the near-zero fill blocks kept
    assert lg.shape == lg_ref.shape
    body = lg[:, 0] != 6
    assert np.array_equal(lg[body, :5], lg_ref[body, :5])
    spars = lg[:, 0] == 3
    assert np.array_equal(lg[spars, 6], lg_ref[spars, 6])
    assert its == its_ref
    assert np.linalg.norm(x - x_ref) <= 1e-8 * np.linalg.norm(x_ref)
    # the ordering without coordinates converges like the geometric one
    _, its_geo, _, _ = _oracle_run(A, levels, tol, skip, grid=(n, 2 if kind == "2d" else 3))
    assert its <= its_geo + 2


def test_parts_argument_errors():
    A = matgen.column_normalize(matgen.advdiff2d(8, seed=1))
    t = Tree(3, 0)
    with pytest.raises(SpqError):
        t.set_parts(np.full(64, 4))  # 3 levels: parts 0..3
    with pytest.raises(SpqError):
        t.set_parts(np.full(64, -1))
    t.set_parts(np.zeros(63, dtype=np.int32))
    with pytest.raises(SpqError):
        t.partition(A)  # one part per column
    with pytest.raises(SpqError):
        graph_parts(A, 0)


def _ata_pairs(A):
    m, n, cp, ri, _ = A
    S = sp.csc_matrix((np.ones(len(ri)), ri, cp), shape=(m, n))
    G = (S.T @ S).tocoo()
    return G.row, G.col


@pytest.mark.parametrize("kind,n,levels", [("2d", 48, 7), ("3d", 14, 7)])
def test_separators_separate(kind, n, levels):
    # nested-dissection invariant of the ordering: two coupled columns (an
    # A^T A edge) lie on separators in an ancestor/descendant relation of the
    # bisection tree (a leaf is level 0), never in two disjoint subtrees
    A = matgen.column_normalize(matgen.advdiff2d(n, seed=3) if kind == "2d" else matgen.advdiff3d(n, seed=3))
    t, _ = _compare(A, levels)
    cp, _ = t.perms()
    b = t.bottom()
    lvl = np.empty(A[1], dtype=np.int64)
    sep = np.empty(A[1], dtype=np.int64)
    for row in b:
        cols = cp[row[0]:row[0] + row[1]]
        lvl[cols] = row[4]
        sep[cols] = row[5]
    i, j = _ata_pairs(A)
    lo = np.where(lvl[i] <= lvl[j], i, j)
    hi = np.where(lvl[i] <= lvl[j], j, i)
    assert np.all((sep[lo] >> (lvl[hi] - lvl[lo])) == sep[hi])
