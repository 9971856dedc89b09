"""The seeded input builder (host C++): shape properties and determinism."""
import numpy as np
import pytest

from nwgraph_b200 import graphs as G


def check_simple_symmetric(g):
    rp, cl = g.row_ptr, g.col
    assert rp[0] == 0 and int(rp[-1]) == len(cl)
    assert np.all(np.diff(rp.astype(np.int64)) >= 0)
    rows = np.repeat(np.arange(g.n), np.diff(rp))
    assert np.all(cl < g.n)
    assert not np.any(rows == cl), "self loop"
    # sorted, duplicate-free rows
    same_row = rows[1:] == rows[:-1]
    assert np.all(cl[1:][same_row] > cl[:-1][same_row])
    # symmetric: the edge set equals its transpose
    a = rows.astype(np.int64) * g.n + cl
    b = cl.astype(np.int64) * g.n + rows
    assert np.array_equal(np.sort(a), np.sort(b))


@pytest.mark.parametrize("scale", [4, 8, 12])
def test_rmat_properties(scale):
    g = G.rmat(scale, 16, 42)
    assert g.n == 2 ** scale
    check_simple_symmetric(g)


def test_rmat_is_thread_count_independent():
    a = G.rmat(13, 16, 7, nthreads=1)
    b = G.rmat(13, 16, 7, nthreads=8)
    assert np.array_equal(a.row_ptr, b.row_ptr) and np.array_equal(a.col, b.col)
    c = G.rmat(13, 16, 8)
    assert not np.array_equal(a.col[: min(len(a.col), len(c.col))], c.col[: min(len(a.col), len(c.col))])


def test_rmat_skew():
    g = G.rmat(14, 16, 42)
    deg = np.diff(g.row_ptr)
    assert deg.max() > 50 * max(deg.mean(), 1)  # power-law hubs
    assert (deg == 0).sum() > 0                   # isolated vertices


@pytest.mark.parametrize("n,side", [(1000, 31), (1024, 32), (1, 1), (17, 4)])
def test_grid(n, side):
    g = G.grid(n)
    assert g.n == side * side
    if g.n > 1:
        check_simple_symmetric(g)
        deg = np.diff(g.row_ptr)
        assert deg.max() <= 4 and deg.min() >= 2
        assert g.nnz == 4 * side * (side - 1)


def test_from_edges_directed():
    g = G.from_edges([0, 0, 1, 2, 2], [1, 2, 2, 0, 0], 4)
    # adjacency<1>: row = destination
    assert g.row_ptr.tolist() == [0, 1, 2, 4, 4]
    assert g.col.tolist() == [2, 0, 0, 1]
    assert g.out_degree().tolist() == [2, 1, 1, 0]


def test_bad_arguments():
    with pytest.raises(RuntimeError):
        G.rmat(0, 16, 1)
    with pytest.raises(RuntimeError):
        G.from_edges([5], [0], 3)
