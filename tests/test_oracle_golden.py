"""Pins the CPU oracle (oracle/oracle.c): against the golden fixtures made by
the reference's own CPU code (tests/golden/make_golden.py), against the
known answers of the reference's example graph, and, where the compiled
reference is present, against it directly on fresh seeded graphs."""
import glob
import os

import numpy as np
import pytest

import oracle as O
from conftest import GOLDEN

FIXTURES = sorted(glob.glob(os.path.join(GOLDEN, "*.npz")))


def load_fixture(path):
    z = np.load(path)
    n = int(z["n"])
    directed = bool(int(z["directed"]))
    if "edge_src" in z:
        g = O.make_graph(n, z["edge_src"], z["edge_dst"], directed, w=z["edge_w"])
    elif "scale" in z:
        g = O.rmat_graph(int(z["scale"]), int(z["edge_factor"]), int(z["seed"]), directed=directed)
    elif "rows" in z:
        g = O.grid_graph(int(z["rows"]), int(z["cols"]), weight_seed=int(z["seed"]))
    else:
        s, d = O.er_edges(int(z["er_n"]), int(z["er_m"]), int(z["seed"]))
        g = O.make_graph(n, s, d, False, weight_mode=1, weight_seed=int(z["seed"]))
    return z, g


@pytest.mark.parametrize("path", FIXTURES, ids=[os.path.basename(p)[:-4] for p in FIXTURES])
def test_builder_reproduces_fixture_csr(path):
    z, g = load_fixture(path)
    assert np.array_equal(g.rowptr, z["rowptr"])
    assert np.array_equal(g.col, z["col"])
    if z["w"].size:
        assert np.array_equal(g.w, z["w"])
    assert np.array_equal(g.in_rowptr, z["in_rowptr"])
    assert np.array_equal(g.in_col, z["in_col"])


@pytest.mark.parametrize("path", FIXTURES, ids=[os.path.basename(p)[:-4] for p in FIXTURES])
def test_oracle_matches_reference_outputs(path):
    z, g = load_fixture(path)
    src = int(z["src"])
    assert np.array_equal(O.bfs(g, src), z["bfs"])
    assert np.array_equal(O.sssp(g, src), z["sssp"])  # bit-exact FP64
    assert np.array_equal(O.wcc(g), z["wcc"])
    pr = O.pagerank(g, 10, 0.85)
    assert np.abs(pr - z["pagerank"]).sum() <= 1e-12 * np.abs(z["pagerank"]).sum()
    assert np.array_equal(O.cdlp(g, 10), z["cdlp"])
    assert np.array_equal(O.tc(g), z["tc"])


def test_reference_example_known_answers():
    """GPU_csr_example.cu's graph, source "one" (ids one=0 .. six=5)."""
    z = np.load(os.path.join(GOLDEN, "toy_example_directed.npz"))
    assert z["bfs"].tolist() == [0, 1, 1, 1, 2, 1]
    assert z["sssp"].tolist() == [0.0, 0.8, 1.0, 1.0, 2.0, 1.0]
    assert z["wcc"].tolist() == [0] * 6
    assert z["cdlp"].tolist() == [0] * 6
    expect = [0.11221769699688859, 0.13606398563018426, 0.30954548324429865, 0.13606398563018426,
              0.17004486286826004, 0.13606398563018426]
    assert np.allclose(z["pagerank"], expect, rtol=0, atol=1e-15)
    t = np.load(os.path.join(GOLDEN, "triangle_pendant_isolated.npz"))
    assert t["tc"].tolist() == [6, 6, 6, 0, 0]
    assert t["cdlp"].tolist() == [0, 0, 0, 0, 4]
    assert t["wcc"].tolist() == [0, 0, 0, 0, 4]


@pytest.mark.skipif(not O.ref_available(), reason="compiled reference (oracle/_ref) not built")
@pytest.mark.parametrize("directed", [False, True])
def test_oracle_matches_compiled_reference_rmat12(directed):
    g = O.rmat_graph(12, 16, 7, directed=directed)
    r = O.Ref().load(g)
    src = int(np.argmax(np.diff(g.rowptr)))
    assert np.array_equal(O.bfs(g, src), r.bfs(src))
    assert np.array_equal(O.bfs(g, src, 2), r.bfs(src, 2))
    assert np.array_equal(O.sssp(g, src), r.sssp(src))
    assert np.array_equal(O.wcc(g), r.wcc())
    assert np.array_equal(O.pagerank(g, 10, 0.85), r.pagerank(10, 0.85))
    assert np.array_equal(O.cdlp(g, 10), r.cdlp(10))
    assert np.array_equal(O.tc(g), r.tc())


def test_oracle_planted_mistake_is_caught():
    """A wrong answer planted in the oracle's output must fail the comparison."""
    z, g = load_fixture(os.path.join(GOLDEN, "rmat10_seed42_undirected.npz"))
    d = O.bfs(g, int(z["src"]))
    d[np.argmax(d < 2**31 - 1)] += 1
    assert not np.array_equal(d, z["bfs"])


@pytest.mark.skipif(not O.ref_available(), reason="compiled reference (oracle/_ref) not built")
def test_oracle_matches_compiled_reference_on_hub_rows():
    """CDLP and TC on rows at the GPU kernels' class edges (1024 | 1025,
    2048 | 2049, 4096 | 4097 entries) and on hubs of 9,000 and 20,000 entries,
    each hub a vertex of its own joined to distinct RMAT vertices: the oracle
    the GPU parity tests use agrees with the reference's CPU code there."""
    scale = 15
    base = 1 << scale
    s, d = O.rmat_edges(scale, 4 << scale, 13)
    rng = np.random.default_rng(17)
    degs = (1024, 1025, 2048, 2049, 4096, 4097, 9000, 20000)
    hs, hd = [s], [d]
    for k, deg in enumerate(degs):
        hs.append(np.full(deg, base + k, np.int32))
        hd.append(rng.choice(base, size=deg, replace=False).astype(np.int32))
    g = O.make_graph(base + len(degs), np.concatenate(hs), np.concatenate(hd), False, weight_mode=0)
    assert np.diff(g.rowptr)[base:].tolist() == list(degs)
    r = O.Ref().load(g)
    for iters in (1, 2, 10):
        assert np.array_equal(O.cdlp(g, iters), r.cdlp(iters)), iters
    assert np.array_equal(O.tc(g), r.tc())


def _wrap32(c64):
    return (np.asarray(c64, np.int64) & 0xFFFFFFFF).astype(np.uint32).view(np.int32)


@pytest.mark.parametrize("path", [p for p in FIXTURES if "undirected" in p or "er3000" in p or "grid" in p],
                         ids=lambda p: os.path.basename(p)[:-4])
def test_oriented_tc_checker_matches_fixtures(path):
    """The oriented CPU triangle count (the checker used where the
    reference's quadratic merge does not finish) gives the reference's
    per-vertex counts on the symmetric golden fixtures."""
    z, g = load_fixture(path)
    c, tri = O.tc_oriented(g)
    assert np.array_equal(_wrap32(c), z["tc"])
    assert int(c.sum()) == 18 * tri


@pytest.mark.skipif(not O.ref_available(), reason="compiled reference (oracle/_ref) not built")
@pytest.mark.parametrize("scale,seed", [(12, 7), (14, 42)])
def test_oriented_tc_checker_matches_compiled_reference(scale, seed):
    """Against the reference's Tri_Counting (CPU_TC.hpp:31-60) itself, on
    RMAT graphs with hubs (all counts well inside int32 here)."""
    g = O.rmat_graph(scale, 16, seed, directed=False, weight_mode=0)
    c, tri = O.tc_oriented(g)
    r = O.Ref().load(g)
    ref = r.tc()
    r.close()
    assert c.max() < 2**31
    assert np.array_equal(c.astype(np.int32), ref)
    assert np.array_equal(c.astype(np.int32), O.tc(g))


def test_oriented_tc_checker_planted_mistake_is_caught():
    z, g = load_fixture(os.path.join(GOLDEN, "rmat10_seed42_undirected.npz"))
    c, _ = O.tc_oriented(g)
    c[np.argmax(c > 0)] += 6
    assert not np.array_equal(_wrap32(c), z["tc"])
