"""Graph file readers (nwgpu_edge_file_*), host code: no GPU needed.

Pinned to the reference: tests/golden/loaders.npz holds the edge lists
NWGraph's read_mm<directed> (io/mmio.hpp:86-103, 171-208) reads from the
Matrix Market files in tests/golden/files/, in its order, and
files/general_ref.nw was written by NWGraph's edge_list::serialize
(edge_list.hpp:237-255). The readers must reproduce those edge lists bit for
bit, and the writer must reproduce the reference's file byte for byte. Where
the reference build is present (oracle/_ref), larger files are compared with
it directly.
"""
import ctypes as C
import os

import numpy as np
import pytest

import oracle as O
from nwgraph_b200 import NwgpuError, construct as K
from nwgraph_b200 import _native as N

HERE = os.path.dirname(os.path.abspath(__file__))
FILES = os.path.join(HERE, "golden", "files")


@pytest.fixture(scope="module")
def golden():
    z = np.load(os.path.join(HERE, "golden", "loaders.npz"))
    return {k: z[k] for k in z.files}


@pytest.mark.parametrize("name", ["general_real", "symmetric_pattern", "karate_pattern"])
@pytest.mark.parametrize("threads", [1, 4])
def test_matrix_market_matches_read_mm(golden, name, threads):
    s, d, n = K.read_edges(os.path.join(FILES, name + ".mtx"), nthreads=threads)
    assert n == int(golden[f"{name}/n"][0])
    assert np.array_equal(s, golden[f"{name}/src"]) and np.array_equal(d, golden[f"{name}/dst"])


def test_values_and_probe():
    info = N.EdgeFile()
    N.check(N.lib().nwgpu_edge_file_probe(os.path.join(FILES, "general_real.mtx").encode(), C.byref(info)))
    assert info.format == N.FILE_MATRIX_MARKET and info.n == 50 and info.max_edges == 300 and info.has_values
    s, d, n, v = K.read_edges(os.path.join(FILES, "general_real.mtx"), values=True)
    rows = np.loadtxt(os.path.join(FILES, "general_real.mtx"), comments="%")[1:]  # after the size line
    assert np.array_equal(v, rows[:, 2].astype(np.float32))
    N.check(N.lib().nwgpu_edge_file_probe(os.path.join(FILES, "symmetric_pattern.mtx").encode(), C.byref(info)))
    assert info.max_edges == 300 and not info.has_values


def test_nw_reader_and_writer_match_the_reference(golden, tmp_path):
    ref_file = os.path.join(FILES, "general_ref.nw")
    s, d, n = K.read_edges(ref_file)
    assert n == 50
    assert np.array_equal(s, golden["general_real/src"]) and np.array_equal(d, golden["general_real/dst"])
    ours = str(tmp_path / "ours.nw")
    K.write_nw_edges(ours, s, d, n)
    assert open(ours, "rb").read() == open(ref_file, "rb").read()


def big_mtx(path, n, m, symmetric, seed=0):
    rng = np.random.default_rng(seed)
    i = rng.integers(1, n + 1, m)
    j = rng.integers(1, n + 1, m)
    if symmetric:
        i, j = np.maximum(i, j), np.minimum(i, j)
    with open(path, "w") as f:
        f.write("%%MatrixMarket matrix coordinate pattern " + ("symmetric" if symmetric else "general") + "\n")
        f.write("% a comment\n")
        f.write(f"{n} {n} {m}\n")
        np.savetxt(f, np.stack([i, j], 1), fmt="%d")
    return i, j


@pytest.mark.parametrize("symmetric", [False, True])
def test_large_file_threads_agree(tmp_path, symmetric):
    path = str(tmp_path / "big.mtx")
    i, j = big_mtx(path, 100_000, 400_000, symmetric)
    s1, d1, _ = K.read_edges(path, nthreads=1)
    s8, d8, _ = K.read_edges(path, nthreads=8)
    assert np.array_equal(s1, s8) and np.array_equal(d1, d8)
    if not symmetric:
        assert np.array_equal(s1, i - 1) and np.array_equal(d1, j - 1)
    else:
        off = i != j
        assert len(s1) == len(i) + off.sum()
    if O.ref_available():
        rs, rd, rn = O.ref_read_mm_edges(path, 2 * len(i) + 1)
        assert rn == 100_000 and np.array_equal(rs, s1) and np.array_equal(rd, d1)


def test_load_graph_builds_the_reference_adjacency(golden):
    # load_graph + build_adjacency<1> restated: CSR by target of the file's edges
    s, d, n = K.read_edges(os.path.join(FILES, "karate_pattern.mtx"))
    rp, cl, deg = O.build_csr(s, d, n, 0)
    if O.ref_available():
        rrp, rcl = O.ref_load_mm(os.path.join(FILES, "karate_pattern.mtx"))
        assert np.array_equal(rp, rrp)
        for r in range(n):  # the reference's row order is its unstable sort's; compare rows as sets
            assert np.array_equal(np.sort(rcl[rrp[r]:rrp[r + 1]]), cl[rp[r]:rp[r + 1]])


@pytest.mark.parametrize("text,status", [
    ("%%MatrixMarket matrix array real general\n2 2\n1\n2\n3\n4\n", N.ERR_UNSUPPORTED),
    ("%%MatrixMarket matrix coordinate real hermitian\n2 2 1\n1 1 1\n", N.ERR_UNSUPPORTED),
    ("%%MatrixMarket matrix coordinate pattern general\n3 3 2\n1 2\n", N.ERR_INVALID_GRAPH),
    ("%%MatrixMarket matrix coordinate pattern general\n3 3 1\n4 1\n", N.ERR_INVALID_GRAPH),
    ("hello\n", N.ERR_INVALID_GRAPH),
])
def test_bad_files(tmp_path, text, status):
    path = tmp_path / "bad.mtx"
    path.write_text(text)
    with pytest.raises(NwgpuError) as ei:
        K.read_edges(str(path))
    assert ei.value.status == status


def test_nw_adjacency_file(golden, tmp_path):
    """A serialized adjacency<1> (adjacency.hpp:180-184, compressed.hpp:377-393)
    written by the reference is read back as its CSR."""
    path = os.path.join(FILES, "karate_adj1_ref.nw")
    info = N.EdgeFile()
    N.check(N.lib().nwgpu_edge_file_probe(path.encode(), C.byref(info)))
    assert info.format == N.FILE_NW_ADJACENCY and info.n == 34 and info.max_edges == 156
    g = K.read_adjacency(path)
    assert np.array_equal(g.row_ptr, golden["karate_adj1/row_ptr"]) and np.array_equal(g.col, golden["karate_adj1/col"])
    if O.ref_available():  # larger, straight from the reference
        from nwgraph_b200 import graphs as G
        big = G.rmat(12, 16, 5)
        O.ref_write_adj1(str(tmp_path / "big.nw"), big.row_ptr, big.col)
        r = K.read_adjacency(str(tmp_path / "big.nw"))
        assert np.array_equal(r.row_ptr, big.row_ptr) and np.array_equal(r.col, big.col)
