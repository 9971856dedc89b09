"""Regenerate the golden fixtures in tests/golden/ (run in a container that has
the reference tree; the GPU host only reads the committed .npz files).

    python tests/golden/make_golden.py [--ref <reference tree>]

* ``karate.npz`` -- the karate edge list and the 34 expected values of
  test/page_rank_test.cpp:41-75 (parsed from the test source as text), the
  adjacency<1> CSR the reference's fill builds from it
  (include/nwgraph/build.hpp:209-232), and NWGraph's own outputs on it:
  page_rank_v1<double> at threshold 1e-7 (what the unit test checks) and
  FP32 page_rank_v10 / page_rank at 20 sweeps.
* ``small_graphs.npz`` -- a handful of small graphs (RMAT scale 8 and 10, a
  grid, a star, a path, a directed graph with sinks and sources, isolated
  vertices) with NWGraph's FP32 page_rank_v10 (20 sweeps, threshold 0, and
  threshold 1e-4 with its sweep count and per-sweep errors) and page_rank v11
  on one thread (20 sweeps, 100 sweeps, and threshold 1e-4 with its sweep
  count and per-sweep errors).
* ``csr_build.npz`` -- edge lists with repeated edges, reversed pairs and
  self-loops (and the karate list), and the CSR the reference builds from
  each with every combination of remove_self_loops, lexical sort + uniq, and
  adjacency<0> / adjacency<1> over a directed or undirected edge list
  (build.hpp:58-69, 209-272, 394-410; rows sorted).
* ``files/`` and ``loaders.npz`` -- small Matrix Market files written here
  (general with real values and comments, symmetric pattern with self-loops,
  the karate edge list) with the edge lists NWGraph's read_mm<directed> reads
  from them (io/mmio.hpp:86-103, 171-208), an NW binary edge list written
  by NWGraph's edge_list::serialize (edge_list.hpp:237-255) with its edges,
  and the karate adjacency<1> serialized as adjacency.hpp:180-184 writes it.

* ``c1_rmat16.npz`` (``--only c1``) -- configuration 1 (RMAT scale 16, the
  rows read_mm<directed> builds, sorted): the CSR's SHA-256 and NWGraph's
  page_rank (v11) converged, at threshold 1e-4, and at the configuration's own
  threshold 1e-4 with max_iters 20, with sweep counts.
* ``refdata.npz`` (``--only refdata``) -- the Matrix Market matrices of the
  reference's own test data (test/data/*.mtx in coordinate format), each
  loaded as the reference driver loads a graph (read_mm<directed>, then
  adjacency<1>: io/mmio.hpp:86-103, 171-208; build.hpp:209-232), with its
  build_degrees and NWGraph's FP32 outputs as for small_graphs.npz.

All reference outputs come from oracle/_ref/libnwref.so, built from the
reference headers by oracle/Makefile.
"""
from __future__ import annotations

import argparse
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle as O  # noqa: E402
from nwgraph_b200 import graphs as G  # noqa: E402


def parse_vector(src: str, name: str):
    m = re.search(r"std::vector<\w+>\s*(?:const\s+)?%s\s*=\s*\{([^}]*)\}" % name, src)
    if not m:
        raise ValueError(f"vector {name} not found")
    return [float(x) for x in m.group(1).replace("\n", " ").split(",") if x.strip()]


def ref_runs(rp, cl, deg):
    """NWGraph's FP32 outputs on one graph: page_rank_v10 and page_rank (v11, one thread) at 20 sweeps, v11
    converged (100 sweeps), and the threshold-1e-4 runs of both with their sweep counts and per-sweep errors."""
    out = {}
    r10, it10, _, _ = O.ref_page_rank(10, rp, cl, deg, 0.85, 0.0, 20, 1)
    r11, it11, _, _ = O.ref_page_rank(11, rp, cl, deg, 0.85, 0.0, 20, 1)
    r10t, it10t, e10t, _ = O.ref_page_rank(10, rp, cl, deg, 0.85, 1e-4, 100, 1)
    r11c, _, _, _ = O.ref_page_rank(11, rp, cl, deg, 0.85, 0.0, 100, 1)
    r11t, it11t, e11t, _ = O.ref_page_rank(11, rp, cl, deg, 0.85, 1e-4, 1000, 1)
    out["v10_20"] = r10
    out["v11_20_t1"] = r11
    out["v10_thr"] = r10t
    out["v10_thr_iters"] = np.array([it10t], np.int64)
    out["v10_thr_errors"] = e10t
    out["v11_100_t1"] = r11c
    out["v11_thr"] = r11t
    out["v11_thr_iters"] = np.array([it11t], np.int64)
    out["v11_thr_errors"] = e11t
    return out


def c1_fixture(tmpdir):
    """Configuration 1: RMAT scale 16 (edge factor 16, seed 42), damping 0.85. The reference reads it from
    Matrix Market with read_mm<directed> into adjacency<1>; its fill sorts with an unstable sort, so it builds
    the builder's rows with the entries of each row in another order. The fixture runs NWGraph on the builder's
    CSR (rows sorted, as sort_adjacency leaves them) after checking that the two CSRs hold the same rows; the
    CSR itself is not stored (the builder regenerates it, checked against the SHA-256 kept here). Stored:
    page_rank (v11, one thread) converged at 100 sweeps, its threshold-1e-4 run, the configuration's own run
    (threshold 1e-4, at most 20 sweeps) with sweep counts and per-sweep errors, and page_rank_v10's
    threshold-1e-4 sweep count."""
    import hashlib
    g = G.rmat(16, 16, 42)
    path = os.path.join(tmpdir, "rmat16.mtx")
    rows = np.repeat(np.arange(g.n, dtype=np.int64), np.diff(g.row_ptr))
    with open(path, "w") as f:
        f.write("%%MatrixMarket matrix coordinate pattern general\n")
        f.write(f"{g.n} {g.n} {g.nnz}\n")
        np.savetxt(f, np.stack([g.col.astype(np.int64) + 1, rows + 1], axis=1), fmt="%d")
    rp, cl = O.ref_load_mm(path)
    assert np.array_equal(rp, g.row_ptr)
    for i in range(g.n):
        assert np.array_equal(np.sort(cl[rp[i]:rp[i + 1]]), g.col[g.row_ptr[i]:g.row_ptr[i + 1]]), i
    rp, cl = g.row_ptr, g.col
    deg = O.ref_build_degrees(rp, cl)
    r11c, _, _, _ = O.ref_page_rank(11, rp, cl, deg, 0.85, 0.0, 100, 1)
    _, it11t, e11t, _ = O.ref_page_rank(11, rp, cl, deg, 0.85, 1e-4, 1000, 1)
    r11, it11, e11, _ = O.ref_page_rank(11, rp, cl, deg, 0.85, 1e-4, 20, 1)
    _, it10t, _, _ = O.ref_page_rank(10, rp, cl, deg, 0.85, 1e-4, 1000, 1)
    out = {"csr_sha256": np.array(hashlib.sha256(rp.tobytes() + cl.tobytes()).hexdigest()),
           "v11_100_t1": r11c, "v11_thr_iters": np.array([it11t], np.int64), "v11_thr_errors": e11t,
           "v11_c1": r11, "v11_c1_iters": np.array([it11], np.int64), "v11_c1_errors": e11,
           "v10_thr_iters": np.array([it10t], np.int64)}
    np.savez_compressed(os.path.join(HERE, "c1_rmat16.npz"), **out)
    print("c1: n", g.n, "nnz", g.nnz, "v10 thr iters", it10t, "v11 thr iters", it11t, "v11 (1e-4, 20) iters", it11)


def directed_with_sinks(n=300, m=1500, seed=3):
    rng = np.random.default_rng(seed)
    src = rng.integers(0, n, size=m)
    dst = rng.integers(0, n, size=m)
    # vertices >= n - 20 are sinks (no out-edges); < 10 are sources (no in-edges)
    keep = (src < n - 20) & (dst >= 10) & (src != dst)
    return G.from_edges(src[keep], dst[keep], n, symmetrize=False)


def star(n=1000):
    s = np.zeros(n - 1, np.uint32)
    d = np.arange(1, n, dtype=np.uint32)
    return G.from_edges(s, d, n, symmetrize=True)


def path(n=500):
    s = np.arange(0, n - 1, dtype=np.uint32)
    return G.from_edges(s, s + 1, n, symmetrize=True)


def isolated_mix(n=700, seed=5):
    rng = np.random.default_rng(seed)
    s = rng.integers(0, n // 2, size=900)
    d = rng.integers(0, n // 2, size=900)
    return G.from_edges(s, d, n, symmetrize=True)  # upper half of the ids is isolated


CSR_FLAG_SETS = [f for f in range(0, 0x20, 2)]  # BY_SOURCE | UNDIRECTED | REMOVE_SELF_LOOPS | UNIQUE


def csr_fixtures(karate_i, karate_j):
    rng = np.random.default_rng(2024)
    lists = {"karate": (karate_i, karate_j, 34)}
    for name, n, m in (("small", 12, 60), ("medium", 200, 3000), ("sparse", 1000, 700)):
        s = rng.integers(0, n, m).astype(np.uint32)
        d = rng.integers(0, n, m).astype(np.uint32)
        k = m // 10  # repeated edges, reversed pairs and self-loops
        s[:k], d[:k] = s[k:2 * k], d[k:2 * k]
        s[2 * k:3 * k], d[2 * k:3 * k] = d[3 * k:4 * k], s[3 * k:4 * k]
        d[4 * k:4 * k + k // 2] = s[4 * k:4 * k + k // 2]
        lists[name] = (s, d, n)
    out = {}
    for name, (s, d, n) in lists.items():
        out[f"{name}/src"], out[f"{name}/dst"], out[f"{name}/n"] = s, d, np.array([n], np.int64)
        for f in CSR_FLAG_SETS:
            rp, cl = O.ref_build_csr(s, d, n, f)
            out[f"{name}/{f}/row_ptr"], out[f"{name}/{f}/col"] = rp, cl
            out[f"{name}/{f}/deg"] = O.ref_build_degrees(rp, cl)  # column occurrences
    np.savez_compressed(os.path.join(HERE, "csr_build.npz"), **out)
    print("csr_build:", len(lists), "edge lists x", len(CSR_FLAG_SETS), "flag sets")


def write_mtx(path, header, n, rows, comments=()):
    with open(path, "w") as f:
        f.write(header + "\n")
        for c in comments:
            f.write("%" + c + "\n")
        f.write(f"{n} {n} {len(rows)}\n")
        for r in rows:
            f.write(" ".join(str(x) for x in r) + "\n")


def loader_fixtures(karate_i, karate_j):
    files = os.path.join(HERE, "files")
    os.makedirs(files, exist_ok=True)
    rng = np.random.default_rng(31)
    n = 50
    gi, gj = rng.integers(1, n + 1, 300), rng.integers(1, n + 1, 300)
    gj[:20] = gi[:20]  # self-loops
    gi[20:40], gj[20:40] = gi[40:60], gj[40:60]  # repeats
    vals = np.round(rng.uniform(-2, 2, 300), 4)
    write_mtx(os.path.join(files, "general_real.mtx"), "%%MatrixMarket matrix coordinate real general", n,
              [(a, b, v) for a, b, v in zip(gi, gj, vals)], comments=(" written by make_golden.py", ""))
    si, sj = rng.integers(1, 41, 150), rng.integers(1, 41, 150)
    si, sj = np.maximum(si, sj), np.minimum(si, sj)  # lower triangle, diagonal included
    write_mtx(os.path.join(files, "symmetric_pattern.mtx"), "%%MatrixMarket matrix coordinate pattern symmetric", 40,
              list(zip(si, sj)))
    write_mtx(os.path.join(files, "karate_pattern.mtx"), "%%MatrixMarket matrix coordinate pattern symmetric", 34,
              list(zip(np.maximum(karate_i, karate_j) + 1, np.minimum(karate_i, karate_j) + 1)))
    out = {}
    for name in ("general_real", "symmetric_pattern", "karate_pattern"):
        s, d, nn = O.ref_read_mm_edges(os.path.join(files, name + ".mtx"), 1000)
        out[f"{name}/src"], out[f"{name}/dst"], out[f"{name}/n"] = s, d, np.array([nn], np.int64)
    s, d = out["general_real/src"], out["general_real/dst"]
    O.ref_write_nw_edges(os.path.join(files, "general_ref.nw"), s, d, n)
    # the reference's adjacency<1> of the karate edge list, serialized by the reference
    rp, cl = O.ref_fill_adj1(karate_i, karate_j, 34)
    O.ref_write_adj1(os.path.join(files, "karate_adj1_ref.nw"), rp, cl)
    out["karate_adj1/row_ptr"], out["karate_adj1/col"] = rp, cl
    np.savez_compressed(os.path.join(HERE, "loaders.npz"), **out)
    print("loaders:", sorted({k.split("/")[0] for k in out}), "+ general_ref.nw")


def refdata_fixtures(ref_root):
    data = os.path.join(ref_root, "test", "data")
    out, names = {}, []
    for fname in sorted(os.listdir(data)):
        path = os.path.join(data, fname)
        if not fname.endswith(".mtx") or "coordinate" not in open(path, errors="replace").readline():
            continue
        name = fname[:-4]
        rp, cl = O.ref_load_mm(path)
        if len(rp) < 3:
            continue
        deg = O.ref_build_degrees(rp, cl)
        out[f"{name}/row_ptr"], out[f"{name}/col"], out[f"{name}/deg"] = rp, cl, deg
        for key, val in ref_runs(rp, cl, deg).items():
            out[f"{name}/{key}"] = val
        names.append(name)
        print(name, "n", len(rp) - 1, "nnz", len(cl), "v10 thr iters", int(out[f"{name}/v10_thr_iters"][0]))
    out["names"] = np.array(names)
    np.savez_compressed(os.path.join(HERE, "refdata.npz"), **out)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("NWGRAPH_REF") or O.default_reference_root(),
                    help="the reference tree (default: $NWGRAPH_REF, else a directory named reference beside "
                         "this repository)")
    ap.add_argument("--only", choices=["csr", "loaders", "refdata", "c1"], default=None,
                    help="regenerate csr_build.npz, files/ and loaders.npz, refdata.npz or c1_rmat16.npz alone")
    args = ap.parse_args()
    if not os.path.isdir(os.path.join(args.ref, "include", "nwgraph")):
        ap.error(f"no reference tree at {args.ref} (set --ref or NWGRAPH_REF)")
    os.environ["NWGRAPH_REF"] = args.ref
    O.build(with_reference=True)
    if args.only == "refdata":
        refdata_fixtures(args.ref)
        return
    if args.only == "c1":
        import tempfile
        with tempfile.TemporaryDirectory() as d:
            c1_fixture(d)
        return
    if args.only:
        src = open(os.path.join(args.ref, "test", "page_rank_test.cpp")).read()
        ki, kj = np.array(parse_vector(src, "i"), np.uint32), np.array(parse_vector(src, "j"), np.uint32)
        (csr_fixtures if args.only == "csr" else loader_fixtures)(ki, kj)
        return

    src = open(os.path.join(args.ref, "test", "page_rank_test.cpp")).read()
    i = np.array(parse_vector(src, "i"), np.uint32)
    j = np.array(parse_vector(src, "j"), np.uint32)
    answer = np.array(parse_vector(src, "answer"), np.float64)
    rp, cl = O.ref_fill_adj1(i, j, 34)
    deg = O.ref_build_degrees(rp, cl)
    v1 = O.ref_page_rank_v1_f64(rp, cl, deg, 0.85, 1e-7, 100)
    k = {"edge_i": i, "edge_j": j, "answer": answer, "row_ptr": rp, "col": cl, "deg": deg, "v1_f64": v1}
    k.update(ref_runs(rp, cl, deg))
    np.savez_compressed(os.path.join(HERE, "karate.npz"), **k)
    print("karate: max rel err of reference v1 vs golden", float(np.max(np.abs(v1 - answer) / answer)))

    graphs = {
        "rmat8": G.rmat(8, 16, 42),
        "rmat10": G.rmat(10, 16, 42),
        "grid": G.grid(1024),
        "star": star(),
        "path": path(),
        "directed": directed_with_sinks(),
        "isolated": isolated_mix(),
    }
    out = {}
    for name, g in graphs.items():
        deg = O.ref_build_degrees(g.row_ptr, g.col)
        out[f"{name}/row_ptr"] = g.row_ptr
        out[f"{name}/col"] = g.col
        out[f"{name}/deg"] = deg
        for key, val in ref_runs(g.row_ptr, g.col, deg).items():
            out[f"{name}/{key}"] = val
        print(name, "n", g.n, "nnz", g.nnz, "v10 thr iters", int(out[f"{name}/v10_thr_iters"][0]))
    np.savez_compressed(os.path.join(HERE, "small_graphs.npz"), **out)
    csr_fixtures(i, j)
    loader_fixtures(i, j)
    refdata_fixtures(args.ref)
    import tempfile
    with tempfile.TemporaryDirectory() as d:
        c1_fixture(d)


if __name__ == "__main__":
    main()
