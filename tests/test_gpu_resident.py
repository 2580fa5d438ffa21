"""Resident (degree-relabelled) graph handle: every ghb_graph_* entry point
against the CPU oracle, with the same bars as the raw-CSR entry points
(bit-exact; PageRank within 1e-6 relative L1 of FP64)."""
import numpy as np
import pytest
import torch

import oracle as O

pytestmark = pytest.mark.gpu

PR_TOL = 1e-6


@pytest.fixture(scope="module")
def G():
    import graphhet_b200 as G
    G.lib()
    return G


def to_gpu(G, og):
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    g = G.CSRGraph(n=og.n, rowptr=t(og.rowptr), col=t(og.col), w=t(og.w) if og.w is not None else None,
                   directed=og.directed)
    if og.directed:
        g.in_rowptr, g.in_col = t(og.in_rowptr), t(og.in_col)
        g.in_w = t(og.in_w) if og.in_w is not None else None
    return g


def rel_l1(a, b):
    return float(np.abs(a - b).sum() / np.abs(b).sum())


def check_resident(G, og, srcs):
    rg = G.ResidentGraph(to_gpu(G, og))
    assert rg.m == og.m
    deg = np.diff(og.rowptr) + (np.diff(og.in_rowptr) if og.directed else 0)
    assert rg.n_active == int((deg > 0).sum())
    for s in srcs:
        ref = O.bfs(og, s)
        for pol in (G.POLICY_HEURISTIC, G.POLICY_PUSH, G.POLICY_PULL):
            assert np.array_equal(rg.bfs(s, policy=pol)[0].cpu().numpy(), ref), f"bfs {pol}"
        if og.w is not None:
            assert np.array_equal(rg.sssp(s)[0].cpu().numpy(), O.sssp(og, s)), "sssp"
    assert np.array_equal(rg.wcc().cpu().numpy(), O.wcc(og)), "wcc"
    ref_pr = O.pagerank(og, 10, 0.85)
    for prec in (G.PR_FP64, G.PR_FP32_KAHAN):
        pr, _, _ = rg.pagerank(10, 0.85, precision=prec)
        assert rel_l1(pr.cpu().numpy(), ref_pr) <= PR_TOL, f"pagerank {prec}"
    assert np.array_equal(rg.cdlp(10).cpu().numpy(), O.cdlp(og, 10)), "cdlp"
    assert np.array_equal(rg.tc()[1].cpu().numpy(), O.tc(og)), "tc"
    d, _ = rg.msbfs(srcs)
    for i, s in enumerate(srcs):
        assert np.array_equal(d[i].cpu().numpy(), O.bfs(og, s)), "msbfs"
    return rg


@pytest.mark.parametrize("directed", [False, True])
def test_resident_rmat16_config0(G, directed):
    og = O.rmat_graph(16, 16, 42, directed=directed)
    src = int(np.argmax(np.diff(og.rowptr)))
    check_resident(G, og, [src, 3, 12345])


def test_resident_grid_and_er(G):
    check_resident(G, O.grid_graph(64, 48, weight_seed=2), [0, 1500])
    s, d = O.er_edges(9000, 7000, 17)
    og = O.make_graph(9000, s, d, False, weight_mode=1, weight_seed=17)
    check_resident(G, og, [0, int(np.argmax(np.diff(og.rowptr)))])


def test_resident_isolated_source_and_predecessors(G):
    og = O.rmat_graph(12, 8, 23)
    deg = np.diff(og.rowptr)
    iso = int(np.nonzero(deg == 0)[0][0])
    rg = check_resident(G, og, [iso, int(np.argmax(deg))])
    src = int(np.argmax(deg))
    depth, pred = rg.bfs_pred(src)
    depth, pred = depth.cpu().numpy(), pred.cpu().numpy()
    for v in range(og.n):
        p = pred[v]
        if v == src or depth[v] == 2**31 - 1:
            assert p == -1
        else:
            assert depth[p] == depth[v] - 1 and v in og.col[og.rowptr[p]:og.rowptr[p + 1]]
    dist, pr = rg.sssp_pred(src)
    dist, pr = dist.cpu().numpy(), pr.cpu().numpy()
    for v in range(og.n):
        p = pr[v]
        if v == src or dist[v] == O.DBL_MAX:
            assert p == -1
            continue
        lo, hi = og.rowptr[p], og.rowptr[p + 1]
        j = lo + np.searchsorted(og.col[lo:hi], v)
        assert og.col[j] == v and dist[p] + og.w[j] == dist[v]


def test_resident_sssp_light_heavy_deltas(G):
    """Delta-stepping with the light/heavy split: bit-exact for any delta,
    including deltas below every weight, above every weight, and a finite inf."""
    for directed in (False, True):
        og = O.rmat_graph(13, 12, 29, directed=directed)
        rg = G.ResidentGraph(to_gpu(G, og))
        src = int(np.argmax(np.diff(og.rowptr)))
        ref = O.sssp(og, src)
        for delta in (1e-7, 0.003, 0.03, 0.25, 1.0, 50.0):
            assert np.array_equal(rg.sssp(src, delta=delta)[0].cpu().numpy(), ref), delta
        exp = np.where(ref < 0.5, ref, 0.5)
        assert np.array_equal(rg.sssp(src, inf=0.5, delta=0.1)[0].cpu().numpy(), exp)
    og = O.grid_graph(40, 30, weight_seed=6)
    rg = G.ResidentGraph(to_gpu(G, og))
    for delta in (1.0, 37.0, 150.0, 5000.0):
        assert np.array_equal(rg.sssp(77, delta=delta)[0].cpu().numpy(), O.sssp(og, 77))
