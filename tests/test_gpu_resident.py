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


def test_sssp_one_launch_matches_host_rounds_and_oracle(G):
    """The whole-traversal SSSP launch against the host-driven rounds and the
    oracle: hubs whose light and heavy ranges span many 1024-entry chunks,
    widths from below every weight (a split per settled distance) to above
    all of them, raw CSR and resident graph, and its pass counters."""
    scale = 14
    base = 1 << scale
    s, d = O.rmat_edges(scale, 8 << scale, 23)
    rng = np.random.default_rng(5)
    hs, hd = [s], [d]
    for k, deg in enumerate((1023, 1025, 3000, 9000)):
        hs.append(np.full(deg, base + k, np.int32))
        hd.append(rng.choice(base, size=deg, replace=False).astype(np.int32))
    og = O.make_graph(base + 4, np.concatenate(hs), np.concatenate(hd), False, weight_mode=1, weight_seed=8)
    g = to_gpu(G, og)
    ws = G.Workspace()
    rg = G.ResidentGraph(g, ws=ws)
    for src in (base + 3, base + 1, int(np.argmax(np.diff(og.rowptr)))):
        ref = O.sssp(og, src)
        for delta in (1e-6, 0.02, 0.4, 3.0):
            d1, st1 = rg.sssp(src, delta=delta, ws=ws)
            assert np.array_equal(d1.cpu().numpy(), ref), (src, delta)
            d2, _ = G.sssp(g, src, delta=delta, ws=ws)
            assert np.array_equal(d2.cpu().numpy(), ref), (src, delta)
            assert st1["levels"] >= 1 and st1["edges_examined"] >= st1["edges_reached"]
        G.tune_set("sssp_persistent", 0, ws=ws)
        d3, _ = rg.sssp(src, ws=ws)
        d4, _ = G.sssp(g, src, ws=ws)
        G.tune_set("sssp_persistent", 1, ws=ws)
        assert np.array_equal(d3.cpu().numpy(), ref) and np.array_equal(d4.cpu().numpy(), ref)
    rg.close()


def test_sssp_adaptive_widths_match_oracle(G):
    """Bucket widths that move from bucket to bucket (sssp_adapt = 1) on the
    one-launch SSSP, widths far below and far above the light/heavy split:
    distances equal the oracle's on the resident graph (split rows) and the
    raw CSR (no split), RMAT with U(0,1] weights and a grid with integer
    weights."""
    for og in (O.rmat_graph(14, 16, 31, directed=False), O.grid_graph(60, 70, 9)):
        g = to_gpu(G, og)
        ws = G.Workspace()
        rg = G.ResidentGraph(g, ws=ws)
        G.tune_set("sssp_adapt", 1, ws=ws)
        deg = np.diff(og.rowptr)
        for src in (int(np.argmax(deg)), int(np.nonzero(deg)[0][-1])):
            ref = O.sssp(og, src)
            for delta in (0.0, 1e-4, 0.05, 2.0, 500.0):
                d1, _ = rg.sssp(src, delta=delta, ws=ws)
                assert np.array_equal(d1.cpu().numpy(), ref), (src, delta)
                d2, _ = G.sssp(g, src, delta=delta, ws=ws)
                assert np.array_equal(d2.cpu().numpy(), ref), (src, delta)
        G.tune_set("sssp_adapt", 0, ws=ws)
        assert G.tune_get("sssp_adapt", ws=ws) == 0
        rg.close()


def test_bfs_many_host_matches_oracle(G):
    """Many BFS into a host array (GPU traversal, byte copies, host
    widening, pipelined): every row equals the oracle's depths.  A 600-vertex
    path beside an RMAT component makes some traversals run over 255 levels
    (their int32 depths are copied instead), in both pipeline slots; also a
    depth limit, one host thread, a repeated and an isolated source, and the
    error for a source outside [0, n)."""
    s, d = O.rmat_edges(12, 8 << 12, 41)
    base, plen = 1 << 12, 600
    ps = np.arange(base, base + plen - 1, dtype=np.int32)
    og = O.make_graph(base + plen, np.concatenate([s, ps]), np.concatenate([d, ps + 1]), False, weight_mode=0)
    rg = G.ResidentGraph(to_gpu(G, og))
    deg = np.diff(og.rowptr)
    hub = int(np.argmax(deg))
    iso = int(np.nonzero(deg == 0)[0][0])
    srcs = [hub, base, base + 300, iso, hub, base + plen - 1, 17]
    out, st = rg.bfs_many_host(srcs)
    assert out.shape == (len(srcs), og.n)
    for i, x in enumerate(srcs):
        assert np.array_equal(out[i], O.bfs(og, x)), i
    assert st["edges_reached"] == sum(rg.bfs(x)[1]["edges_reached"] for x in srcs)
    assert st["levels"] >= plen - 1
    out3, _ = rg.bfs_many_host(srcs, max_depth=3, host_threads=1)
    for i, x in enumerate(srcs):
        assert np.array_equal(out3[i], O.bfs(og, x, 3)), i
    empty, _ = rg.bfs_many_host([])
    assert empty.shape == (0, og.n)
    with pytest.raises(G.GhbError):
        rg.bfs_many_host([0, og.n])
    rg.close()


def test_msbfs_forced_schedules_and_trace(G):
    """The one-launch multi-source pass under forced directions (all push,
    all pull, alternating): depths equal the oracle's in every case, the
    trace's direction column is the schedule, and its counts are the
    frontier sizes; the rule-steered run matches too."""
    og = O.rmat_graph(13, 16, 19, directed=False)
    rg = G.ResidentGraph(to_gpu(G, og))
    deg = np.diff(og.rowptr)
    srcs = [int(np.argmax(deg)), 3, 77, int(np.nonzero(deg)[0][-1])] + list(range(100, 160))
    refs = [O.bfs(og, x) for x in srcs]
    d0, st0, tr0 = rg.msbfs_ex(srcs, trace_cap=64)
    levels = st0["levels"]
    assert tr0.shape == (levels, G.MS_TRACE_COLS)
    for sched in (None, [0] * 64, [1] * 64, [k & 1 for k in range(64)]):
        d, st, tr = rg.msbfs_ex(srcs, schedule=sched, trace_cap=64)
        for i, ref in enumerate(refs):
            assert np.array_equal(d[i].cpu().numpy(), ref), (sched and sched[:4], i)
        assert st["levels"] == levels
        if sched is not None:
            assert tr[:, 0].astype(int).tolist() == sched[:levels]
        # The frontier a level finds is the next level's frontier.
        assert np.array_equal(tr[1:, 2], tr[:-1, 4]) and np.array_equal(tr[1:, 3], tr[:-1, 5])
        assert np.all(tr[:, 1] >= 0)
    # The learned direction model (the shipped weights) steering the pass.
    from graphhet_b200 import policy as P
    P.ms_install()
    G.tune_set("ms_learned", 1)
    try:
        d, st, tr = rg.msbfs_ex(srcs, trace_cap=64)
        d2, _ = rg.msbfs(srcs)
    finally:
        G.tune_set("ms_learned", 0)
        G.lib().ghb_ms_policy_load(None, 0)
    for i, ref in enumerate(refs):
        assert np.array_equal(d[i].cpu().numpy(), ref) and np.array_equal(d2[i].cpu().numpy(), ref), i
    rg.close()


def test_resident_cdlp_and_wcc_with_repeated_entries(G):
    """A symmetric CSR whose rows repeat some entries (so label counts of 2
    occur in the first CDLP iteration) and a directed graph: CDLP and WCC on
    the handle equal the oracle's."""
    rng = np.random.default_rng(4)
    n = 300
    s = rng.integers(0, n, 1200)
    d = rng.integers(0, n, 1200)
    keep = s != d
    s, d = s[keep], d[keep]
    # Symmetric rows with repeats: each undirected pair listed 1 or 2 times.
    rows = [[] for _ in range(n)]
    for a, b in zip(s, d):
        k = 2 if (a + b) % 5 == 0 else 1
        rows[a] += [b] * k
        rows[b] += [a] * k
    rp = np.zeros(n + 1, np.int32)
    rp[1:] = np.cumsum([len(r) for r in rows])
    col = np.concatenate([np.sort(np.array(r, np.int32)) for r in rows if r]).astype(np.int32)
    og = O.Graph(n=n, rowptr=rp, col=col, w=None, directed=False, in_rowptr=rp, in_col=col, in_w=None)
    rg = G.ResidentGraph(to_gpu(G, og))
    assert np.array_equal(rg.cdlp(10).cpu().numpy(), O.cdlp(og, 10))
    assert np.array_equal(rg.wcc().cpu().numpy(), O.wcc(og))
    og2 = O.rmat_graph(10, 8, 77, directed=True)
    rg2 = G.ResidentGraph(to_gpu(G, og2))
    assert np.array_equal(rg2.cdlp(10).cpu().numpy(), O.cdlp(og2, 10))
    assert np.array_equal(rg2.wcc().cpu().numpy(), O.wcc(og2))


def test_cdlp_rows_beyond_4096_entries(G):
    """Rows of the global-table class (> 4096 entries): two star hubs of 6,000
    and 9,000 leaves on an RMAT graph, raw CSR and handle, 10 iterations."""
    s, d = O.rmat_edges(14, 8 << 14, 31)
    s = np.concatenate([s, np.zeros(6000, np.int32), np.full(9000, 7, np.int32)])
    d = np.concatenate([d, np.arange(100, 6100, dtype=np.int32), np.arange(3000, 12000, dtype=np.int32)])
    og = O.make_graph(1 << 14, s, d, False, weight_mode=0)
    assert np.diff(og.rowptr).max() > 4096
    ref = O.cdlp(og, 10)
    assert np.array_equal(G.cdlp(to_gpu(G, og), 10).cpu().numpy(), ref)
    rg = G.ResidentGraph(to_gpu(G, og))
    assert np.array_equal(rg.cdlp(10).cpu().numpy(), ref)
    assert np.array_equal(rg.cdlp(3).cpu().numpy(), O.cdlp(og, 3))


def test_cdlp_class_edges_and_many_chunks(G):
    """Rows at each class edge (1024 | 1025, 2048 | 2049 and 4096 | 4097
    entries, the last the first chunked row), rows of four and five chunks
    of 2048 (8192 | 8193) and hubs of 20,000 and 45,000 entries (10 and 22
    chunks), each hub a vertex of its own joined to distinct RMAT vertices;
    raw CSR and handle, 1, 2 and 10 iterations."""
    scale = 16
    base = 1 << scale
    s, d = O.rmat_edges(scale, 8 << scale, 11)
    rng = np.random.default_rng(5)
    degs = (1024, 1025, 2048, 2049, 4096, 4097, 8192, 8193, 20000, 45000)
    hs, hd = [s], [d]
    for k, deg in enumerate(degs):
        hs.append(np.full(deg, base + k, np.int32))
        hd.append(rng.choice(base, size=deg, replace=False).astype(np.int32))
    og = O.make_graph(base + len(degs), np.concatenate(hs), np.concatenate(hd), False, weight_mode=0)
    assert np.diff(og.rowptr)[base:].tolist() == list(degs)
    g = to_gpu(G, og)
    rg = G.ResidentGraph(to_gpu(G, og))
    for iters in (1, 2, 10):
        ref = O.cdlp(og, iters)
        assert np.array_equal(G.cdlp(g, iters).cpu().numpy(), ref), iters
        assert np.array_equal(rg.cdlp(iters).cpu().numpy(), ref), iters
