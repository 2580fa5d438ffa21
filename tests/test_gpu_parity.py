"""GPU parity: every algorithm through the C ABI against the CPU oracle
(oracle/oracle.c, itself pinned to the reference) and the golden fixtures.
Integer outputs and SSSP distances must match bit for bit; PageRank within
1e-6 relative L1 of the FP64 oracle."""
import glob
import os

import numpy as np
import pytest
import torch

import oracle as O
from conftest import GOLDEN

pytestmark = pytest.mark.gpu

PR_TOL = 1e-6  # relative L1 vs FP64

FIXTURES = sorted(glob.glob(os.path.join(GOLDEN, "*.npz")))


@pytest.fixture(scope="module")
def G():
    import graphhet_b200 as G
    assert torch.cuda.is_available()
    G.lib()
    return G


def to_gpu(G, og: O.Graph):
    dev = torch.device("cuda")
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    g = G.CSRGraph(n=og.n, rowptr=t(og.rowptr), col=t(og.col), w=t(og.w) if og.w is not None else None,
                   directed=og.directed)
    if og.directed:
        g.in_rowptr, g.in_col = t(og.in_rowptr), t(og.in_col)
        g.in_w = t(og.in_w) if og.in_w is not None else None
    return g


def rel_l1(a, b):
    return float(np.abs(a - b).sum() / np.abs(b).sum())


def check_all(G, g, og, src, pr_tol=PR_TOL):
    d, st = G.bfs(g, src)
    assert np.array_equal(d.cpu().numpy(), O.bfs(og, src)), "bfs"
    for pol in (G.POLICY_PUSH, G.POLICY_PULL):
        d2, _ = G.bfs(g, src, policy=pol)
        assert np.array_equal(d2.cpu().numpy(), O.bfs(og, src)), f"bfs policy {pol}"
    dist, _ = G.sssp(g, src)
    assert np.array_equal(dist.cpu().numpy(), O.sssp(og, src)), "sssp"
    assert np.array_equal(G.wcc(g).cpu().numpy(), O.wcc(og)), "wcc"
    ref_pr = O.pagerank(og, 10, 0.85)
    for prec in (G.PR_FP64, G.PR_FP32_KAHAN):
        pr, _, _ = G.pagerank(g, 10, 0.85, precision=prec)
        assert rel_l1(pr.cpu().numpy(), ref_pr) <= pr_tol, f"pagerank precision {prec}"
    assert np.array_equal(G.cdlp(g, 10).cpu().numpy(), O.cdlp(og, 10)), "cdlp"
    c64, c32, total = G.tc(g)
    ref_tc = O.tc(og)
    assert np.array_equal(c32.cpu().numpy(), ref_tc), "tc int32"


@pytest.mark.parametrize("path", FIXTURES, ids=[os.path.basename(p)[:-4] for p in FIXTURES])
def test_golden_fixtures(G, path):
    z = np.load(path)
    n = int(z["n"])
    og = O.Graph(n, z["rowptr"], z["col"], z["w"] if z["w"].size else None, bool(int(z["directed"])),
                 z["in_rowptr"], z["in_col"], None)
    g = to_gpu(G, og)
    src = int(z["src"])
    assert np.array_equal(G.bfs(g, src)[0].cpu().numpy(), z["bfs"])
    if og.w is not None:
        assert np.array_equal(G.sssp(g, src)[0].cpu().numpy(), z["sssp"])
    assert np.array_equal(G.wcc(g).cpu().numpy(), z["wcc"])
    pr, _, _ = G.pagerank(g, 10, 0.85)
    assert rel_l1(pr.cpu().numpy(), z["pagerank"]) <= PR_TOL
    assert np.array_equal(G.cdlp(g, 10).cpu().numpy(), z["cdlp"])
    assert np.array_equal(G.tc(g)[1].cpu().numpy(), z["tc"])


@pytest.mark.parametrize("directed", [False, True])
def test_gpu_builder_matches_cpu_builder(G, directed):
    src, dst = G.gen_rmat(12, 16 << 12, 42)
    s_cpu, d_cpu = O.rmat_edges(12, 16 << 12, 42)
    assert np.array_equal(src.cpu().numpy(), s_cpu) and np.array_equal(dst.cpu().numpy(), d_cpu)
    g = G.make_graph(1 << 12, src, dst, directed, weight_seed=42)
    og = O.make_graph(1 << 12, s_cpu, d_cpu, directed, weight_seed=42)
    assert np.array_equal(g.rowptr.cpu().numpy(), og.rowptr)
    assert np.array_equal(g.col.cpu().numpy(), og.col)
    assert np.array_equal(g.w.cpu().numpy(), og.w)
    if directed:
        assert np.array_equal(g.in_rowptr.cpu().numpy(), og.in_rowptr)
        assert np.array_equal(g.in_col.cpu().numpy(), og.in_col)
        assert np.array_equal(g.in_w.cpu().numpy(), og.in_w)


def test_builder_duplicates_last_weight_wins(G):
    s = torch.tensor([0, 0, 1, 2, 1, 3, 1], dtype=torch.int32, device="cuda")
    d = torch.tensor([1, 1, 0, 2, 2, 1, 2], dtype=torch.int32, device="cuda")
    w = torch.tensor([0.5, 0.25, 0.75, 1.0, 0.125, 2.0, 0.0625], dtype=torch.float64, device="cuda")
    rp, col, wt = G.build_csr(5, s, d, w=w, symmetrize=False)
    orp, ocol, ow = O.build_csr(5, s.cpu().numpy(), d.cpu().numpy(), w=w.cpu().numpy())
    assert np.array_equal(rp.cpu().numpy(), orp) and np.array_equal(col.cpu().numpy(), ocol)
    assert np.array_equal(wt.cpu().numpy(), ow)


def test_builder_rejects_bad_endpoint(G):
    s = torch.tensor([0, 5], dtype=torch.int32, device="cuda")
    d = torch.tensor([1, 1], dtype=torch.int32, device="cuda")
    with pytest.raises(G.GhbError):
        G.build_csr(5, s, d)


@pytest.mark.parametrize("directed", [False, True])
def test_rmat16_config0_all_algorithms(G, directed):
    """RMAT seed 42, scale 16, edge factor 16, sources = highest degree vertex."""
    g = G.rmat_graph(16, 16, 42, directed=directed)
    og = O.rmat_graph(16, 16, 42, directed=directed)
    assert np.array_equal(g.col.cpu().numpy(), og.col)
    deg = np.diff(og.rowptr)
    src = int(np.argmax(deg))  # first maximum = smallest id among ties
    check_all(G, g, og, src)


def test_grid_high_diameter(G):
    g = G.grid_graph(96, 80, weight_seed=3)
    og = O.grid_graph(96, 80, weight_seed=3)
    assert np.array_equal(g.w.cpu().numpy(), og.w)
    check_all(G, g, og, 0)
    check_all(G, g, og, 96 * 80 // 2 + 7)


def test_er_sparse_many_components(G):
    s, d = O.er_edges(20000, 12000, 11)
    og = O.make_graph(20000, s, d, False, weight_mode=1, weight_seed=11)
    g = to_gpu(G, og)
    check_all(G, g, og, int(np.argmax(np.diff(og.rowptr))))
    check_all(G, g, og, 5)


def test_edge_cases(G):
    # no edges at all
    og = O.make_graph(7, np.zeros(0, np.int32), np.zeros(0, np.int32), False)
    g = to_gpu(G, og)
    assert G.bfs(g, 3)[0].cpu().tolist() == [2**31 - 1] * 3 + [0] + [2**31 - 1] * 3
    assert G.wcc(g).cpu().tolist() == list(range(7))
    assert G.cdlp(g, 5).cpu().tolist() == list(range(7))
    assert G.tc(g)[1].cpu().tolist() == [0] * 7
    pr, _, _ = G.pagerank(g, 10, 0.85)
    assert rel_l1(pr.cpu().numpy(), O.pagerank(og, 10, 0.85)) <= PR_TOL
    dist = G.sssp(g, 2)[0].cpu().numpy()
    assert dist[2] == 0 and np.all(np.delete(dist, 2) == O.DBL_MAX)
    # single vertex
    og1 = O.make_graph(1, np.zeros(0, np.int32), np.zeros(0, np.int32), False)
    g1 = to_gpu(G, og1)
    assert G.bfs(g1, 0)[0].cpu().tolist() == [0]
    # star: hub row far longer than a warp
    hub = np.zeros(9000, np.int32)
    leaves = np.arange(1, 9001, dtype=np.int32)
    og2 = O.make_graph(9001, hub, leaves, False, weight_mode=1, weight_seed=2)
    check_all(G, to_gpu(G, og2), og2, 17)
    # max_depth
    og3 = O.rmat_graph(12, 8, 5)
    g3 = to_gpu(G, og3)
    for md in (0, 1, 2, 3):
        assert np.array_equal(G.bfs(g3, 1, max_depth=md)[0].cpu().numpy(), O.bfs(og3, 1, md))
    # invalid source is an error, not a fault
    with pytest.raises(G.GhbError):
        G.bfs(g3, og3.n)
    with pytest.raises(G.GhbError):
        G.sssp(g3, -1)


def test_sssp_custom_inf_and_delta(G):
    og = O.rmat_graph(13, 8, 9, directed=True)
    g = to_gpu(G, og)
    ref = O.sssp(og, 0)
    for delta in (0.01, 0.3, 5.0):
        dist, _ = G.sssp(g, 0, delta=delta)
        assert np.array_equal(dist.cpu().numpy(), ref)
    # finite inf: vertices at distance >= inf stay at inf (reference semantics)
    dist, _ = G.sssp(g, 0, inf=1.0)
    exp = np.where(ref < 1.0, ref, 1.0)
    assert np.array_equal(dist.cpu().numpy(), exp)


def test_bfs_schedule_and_trace(G):
    og = O.rmat_graph(14, 16, 4)
    g = to_gpu(G, og)
    ref = O.bfs(og, 10)
    d, st, tr = G.bfs(g, 10, trace_cap=64, oracle_timing=True)
    assert np.array_equal(d.cpu().numpy(), ref)
    assert tr.shape[0] == st["levels"] and tr.shape[1] == G.TRACE_COLS
    assert np.all(tr[:, 14] >= 0) and np.all(tr[:, 15] >= 0)
    sched = [0, 1, 0, 1, 1, 0, 0, 1, 0, 1, 1, 1, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0]
    d2, _ = G.bfs(g, 10, policy=G.POLICY_SCHEDULE, schedule=sched)
    assert np.array_equal(d2.cpu().numpy(), ref)


def test_bfs_and_sssp_predecessors(G):
    for directed in (False, True):
        og = O.rmat_graph(12, 16, 21, directed=directed)
        g = to_gpu(G, og)
        src = int(np.argmax(np.diff(og.rowptr)))
        depth, pred = G.bfs_pred(g, src)
        depth, pred = depth.cpu().numpy(), pred.cpu().numpy()
        assert np.array_equal(depth, O.bfs(og, src))
        for v in range(og.n):
            p = pred[v]
            if v == src or depth[v] == 2**31 - 1:
                assert p == -1
                continue
            row = og.col[og.rowptr[p]:og.rowptr[p + 1]]
            assert depth[p] == depth[v] - 1 and v in row
        dist, pr = G.sssp_pred(g, src)
        dist, pr = dist.cpu().numpy(), pr.cpu().numpy()
        assert np.array_equal(dist, O.sssp(og, src))
        for v in range(og.n):
            p = pr[v]
            if v == src or dist[v] == O.DBL_MAX:
                assert p == -1
                continue
            lo, hi = og.rowptr[p], og.rowptr[p + 1]
            j = lo + np.searchsorted(og.col[lo:hi], v)
            assert og.col[j] == v and dist[p] + og.w[j] == dist[v]


def test_msbfs_matches_single_source(G):
    og = O.rmat_graph(13, 16, 8)
    g = to_gpu(G, og)
    rng = np.random.default_rng(0)
    srcs = rng.integers(0, og.n, 70).astype(np.int32)
    srcs[3] = srcs[4]  # duplicate source
    d = torch.empty(len(srcs) * og.n, dtype=torch.int32, device="cuda")
    st = G.TraversalStats()
    import ctypes
    G._check(G.lib().ghb_msbfs(G._ws(None), og.n, G._ptr(g.rowptr), G._ptr(g.col), G._ptr(g.rowptr),
                               G._ptr(g.col), G._ptr(torch.from_numpy(srcs).cuda()), len(srcs), G._ptr(d),
                               ctypes.byref(st)), "ghb_msbfs")
    d = d.cpu().numpy().reshape(len(srcs), og.n)
    for i in range(0, len(srcs), 7):
        assert np.array_equal(d[i], O.bfs(og, int(srcs[i])))
    assert np.array_equal(d[4], O.bfs(og, int(srcs[4])))
    assert np.array_equal(d[69], O.bfs(og, int(srcs[69])))


def test_batch_wcc_and_tc(G):
    import ctypes
    rng = np.random.default_rng(5)
    graphs = []
    for i in range(12):
        n = int(rng.integers(50, 3000))
        m = int(rng.integers(n // 2, 6 * n))
        s, d = O.er_edges(n, m, 100 + i)
        graphs.append(O.make_graph(n, s, d, False, weight_mode=0))
    vbase = np.zeros(len(graphs) + 1, np.int64)
    ebase = np.zeros(len(graphs) + 1, np.int64)
    for i, og in enumerate(graphs):
        vbase[i + 1] = vbase[i] + og.n
        ebase[i + 1] = ebase[i] + og.m
    rp = torch.from_numpy(np.concatenate([og.rowptr for og in graphs])).cuda()
    col = torch.from_numpy(np.concatenate([og.col for og in graphs])).cuda()
    lab = torch.empty(int(vbase[-1]), dtype=torch.int32, device="cuda")
    P = ctypes.POINTER(ctypes.c_int64)
    G._check(G.lib().ghb_batch_wcc(G._ws(None), len(graphs), vbase.ctypes.data_as(ctypes.c_void_p),
                                   ebase.ctypes.data_as(ctypes.c_void_p), G._ptr(rp), G._ptr(col), G._ptr(lab)),
             "ghb_batch_wcc")
    c64 = torch.empty(int(vbase[-1]), dtype=torch.int64, device="cuda")
    totals = np.zeros(len(graphs), np.int64)
    G._check(G.lib().ghb_batch_tc(G._ws(None), len(graphs), vbase.ctypes.data_as(ctypes.c_void_p),
                                  ebase.ctypes.data_as(ctypes.c_void_p), G._ptr(rp), G._ptr(col), G._ptr(c64),
                                  totals.ctypes.data_as(ctypes.c_void_p)), "ghb_batch_tc")
    lab, c64 = lab.cpu().numpy(), c64.cpu().numpy()
    for i, og in enumerate(graphs):
        a, b = vbase[i], vbase[i + 1]
        assert np.array_equal(lab[a:b], O.wcc(og))
        ref = O.tc(og)
        assert np.array_equal(c64[a:b].astype(np.int32), ref)
        assert totals[i] == int(ref.astype(np.int64).sum()) // 18


@pytest.mark.parametrize("count", [1, 64, 65, 130, 256, 300])
def test_msbfs_word_widths(G, count):
    """Passes of 64, 128 and 256 sources (1, 2 and 4 words per vertex), a
    second pass past 256, duplicates and isolated sources; raw CSR and the
    relabelled handle, directed and undirected; a star hub so that pull rows
    go to the block-per-row path."""
    import ctypes
    for directed in (False, True):
        og = O.rmat_graph(11, 8, 13 + count, directed=directed)
        if not directed:
            # Add a hub adjacent to 1500 vertices (rows of > 256 entries).
            s, d = O.rmat_edges(11, 8 << 11, 13 + count)
            hub = np.full(1500, 5, np.int32)
            leaves = np.arange(200, 1700, dtype=np.int32)
            og = O.make_graph(1 << 11, np.concatenate([s, hub]), np.concatenate([d, leaves]), False)
        g = to_gpu(G, og)
        rng = np.random.default_rng(count)
        srcs = rng.integers(0, og.n, count).astype(np.int32)
        if count > 2:
            srcs[1] = srcs[0]
        deg = np.diff(og.rowptr) + (np.diff(og.in_rowptr) if directed else 0)
        iso = np.nonzero(deg == 0)[0]
        if iso.size and count > 3:
            srcs[2] = iso[0]
        d = torch.empty(count * og.n, dtype=torch.int32, device="cuda")
        st = G.TraversalStats()
        irp, icol = (g.in_rowptr, g.in_col) if directed else (g.rowptr, g.col)
        G._check(G.lib().ghb_msbfs(G._ws(None), og.n, G._ptr(g.rowptr), G._ptr(g.col), G._ptr(irp), G._ptr(icol),
                                   G._ptr(torch.from_numpy(srcs).cuda()), count, G._ptr(d), ctypes.byref(st)),
                 "ghb_msbfs")
        d = d.cpu().numpy().reshape(count, og.n)
        rg = G.ResidentGraph(g)
        dr, _ = rg.msbfs(srcs)
        dr = dr.cpu().numpy()
        check = set(range(0, count, 17)) | {0, 1, 2, count - 1}
        if count > 255:
            check |= {63, 64, 127, 128, 255, 256}
        for i in sorted(check):
            if i < count:
                ref = O.bfs(og, int(srcs[i]))
                assert np.array_equal(d[i], ref), (directed, i)
                assert np.array_equal(dr[i], ref), (directed, i)
        rg.close()


@pytest.mark.parametrize("count", [3, 100, 200])
def test_msbfs_long_diameter(G, count):
    """A grid (about 70 levels): depths leave the kept level words in many
    chunks, on the raw CSR and on the relabelled handle."""
    import ctypes
    og = O.grid_graph(30, 40, 1)
    g = to_gpu(G, og)
    srcs = np.random.default_rng(count).integers(0, og.n, count).astype(np.int32)
    d = torch.empty(count * og.n, dtype=torch.int32, device="cuda")
    st = G.TraversalStats()
    G._check(G.lib().ghb_msbfs(G._ws(None), og.n, G._ptr(g.rowptr), G._ptr(g.col), G._ptr(g.rowptr), G._ptr(g.col),
                               G._ptr(torch.from_numpy(srcs).cuda()), count, G._ptr(d), ctypes.byref(st)), "ghb_msbfs")
    d = d.cpu().numpy().reshape(count, og.n)
    rg = G.ResidentGraph(g)
    dr = rg.msbfs(srcs)[0].cpu().numpy()
    for i in sorted({0, count // 2, count - 1}):
        ref = O.bfs(og, int(srcs[i]))
        assert np.array_equal(d[i], ref)
        assert np.array_equal(dr[i], ref)
    rg.close()


def test_msbfs_one_launch_pass_and_graph_replay(G):
    """A 256-source pass as one cooperative launch: equal to the host-driven
    levels and to single-source runs, with a hub of 5,000 leaves (push rows
    cut into chunks) and isolated / duplicate sources; then the launch-only
    entry recorded in a CUDA graph and replayed twice, bit-exact."""
    scale = 13
    s, d = O.rmat_edges(scale, 8 << scale, 77)
    hub = np.full(5000, 9, np.int32)
    leaves = np.arange(100, 5100, dtype=np.int32)
    og = O.make_graph(1 << scale, np.concatenate([s, hub]), np.concatenate([d, leaves]), False)
    g = to_gpu(G, og)
    rng = np.random.default_rng(11)
    srcs = rng.integers(0, og.n, 256).astype(np.int32)
    srcs[1] = srcs[0]
    srcs[2] = 9
    iso = np.nonzero(np.diff(og.rowptr) == 0)[0]
    if iso.size:
        srcs[3] = iso[0]
    ws = G.Workspace()
    rg = G.ResidentGraph(g, ws=ws)
    one, st1 = rg.msbfs(srcs, ws=ws)
    one = one.cpu().numpy()
    G.tune_set("ms_persistent", 0, ws=ws)
    host = rg.msbfs(srcs, ws=ws)[0].cpu().numpy()
    G.tune_set("ms_persistent", 1, ws=ws)
    assert np.array_equal(one, host)
    assert st1["levels"] >= 1
    for i in (0, 1, 2, 3, 64, 128, 200, 255):
        assert np.array_equal(one[i], O.bfs(og, int(srcs[i]))), i
    # Launch-only entry, captured in a CUDA graph on a side stream.
    sd = torch.from_numpy(srcs).cuda()
    out = torch.full((256 * og.n,), -5, dtype=torch.int32, device="cuda")
    rg.msbfs_reserve(256, ws=ws)
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.stream(side):
        with torch.cuda.graph(graph, stream=side):
            rg.msbfs_launch(sd, out, ws=ws)
    for _ in range(2):
        out.fill_(-5)
        graph.replay()
        torch.cuda.synchronize()
        assert np.array_equal(out.cpu().numpy().reshape(256, og.n), one)
    del graph
    rg.close()


def test_union_batch_wcc_tc_and_graph_capture(G):
    """Many ER graphs as one disjoint-union CSR: WCC labels and triangle
    counts equal the oracle's per graph; the launch-only call recorded in a
    CUDA graph and replayed gives the same arrays."""
    b = G.er_batch(25, 7, n_lo=50, n_hi=3000, deg_lo=1.0, deg_hi=12.0)
    ws = G.Workspace()
    b.reserve(ws)
    N = b.g.n
    lab = torch.empty(N, dtype=torch.int32, device="cuda")
    c64 = torch.empty(N, dtype=torch.int64, device="cuda")
    tri = torch.empty(b.n_graphs, dtype=torch.int64, device="cuda")
    b.wcc_tc(lab, c64, tri, ws=ws)
    torch.cuda.synchronize()
    rp, col = b.g.rowptr.cpu().numpy(), b.g.col.cpu().numpy()
    lab_h, c64_h, tri_h = lab.cpu().numpy(), c64.cpu().numpy(), tri.cpu().numpy()
    vb = b.vbase_host
    for g in range(b.n_graphs):
        lo, hi = int(vb[g]), int(vb[g + 1])
        lrp = (rp[lo:hi + 1] - rp[lo]).astype(np.int32)
        lcol = (col[rp[lo]:rp[hi]] - lo).astype(np.int32)
        og = O.Graph(n=hi - lo, rowptr=lrp, col=lcol, w=None, directed=False, in_rowptr=lrp, in_col=lcol, in_w=None)
        assert np.array_equal(lab_h[lo:hi], O.wcc(og)), g
        ref_tc = O.tc(og)
        assert np.array_equal(c64_h[lo:hi].astype(np.int32), ref_tc), g
        assert tri_h[g] * 18 == int(ref_tc.astype(np.int64).sum()), g
    # Record the launch-only call in a CUDA graph and replay it twice.
    lab2 = torch.full_like(lab, -1)
    c642 = torch.full_like(c64, -1)
    tri2 = torch.full_like(tri, -1)
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.stream(side):
        with torch.cuda.graph(graph, stream=side):
            b.wcc_tc(lab2, c642, tri2, ws=ws)
    for _ in range(2):
        lab2.fill_(-1)
        graph.replay()
        torch.cuda.synchronize()
        assert torch.equal(lab2, lab) and torch.equal(c642, c64) and torch.equal(tri2, tri)
    del graph
    ws.close()


def test_dangling_selection_matches_oracle_and_pagerank(G):
    """The seeded dangling-vertex selection (PageRank precision workload) is
    the same on the GPU and in the oracle, and PageRank on such a directed
    graph meets the 1e-6 relative-L1 bar in both precisions."""
    import ctypes
    s, d = O.rmat_edges(12, 16 << 12, 11)
    keep = torch.empty(len(s), dtype=torch.uint8, device="cuda")
    G._check(G.lib().ghb_gen_dangling_keep(G._ws(None), len(s), G._ptr(torch.from_numpy(s).cuda()), 11, 0.1,
                                           G._ptr(keep)), "ghb_gen_dangling_keep")
    ref_keep = O.dangling_keep(s, 11, 0.1)
    assert np.array_equal(keep.cpu().numpy(), ref_keep)
    og = O.make_graph(1 << 12, s[ref_keep == 1], d[ref_keep == 1], True, weight_mode=0)
    ref = O.pagerank(og, 20, 0.85)
    g = G.rmat_dangling_graph(12, 16, 11, 0.1)
    assert g.m == og.m
    for prec in (G.PR_FP64, G.PR_FP32_KAHAN):
        pr, _, _ = G.pagerank(g, 20, 0.85, precision=prec)
        pr = pr.cpu().numpy()
        assert np.abs(pr - ref).sum() / np.abs(ref).sum() <= 1e-6


@pytest.mark.parametrize("count", [1, 5, 64, 100, 256, 300])
def test_mssssp_matches_single_source(G, count):
    """Multi-source SSSP (one bucketed traversal per 256 sources): every row
    equals the oracle's Dijkstra bit for bit, on the raw CSR and the
    relabelled handle, RMAT with U(0,1] weights (one with a 1,585-entry
    row, relaxed as 256-entry chunks) and a grid with integer weights;
    duplicate and isolated sources included."""
    import ctypes
    graphs = [O.rmat_graph(11, 8, 3 + count), O.grid_graph(20, 30, count)]
    if count in (64, 300):
        graphs.append(O.rmat_graph(12, 24, 5))
    for og in graphs:
        g = to_gpu(G, og)
        rng = np.random.default_rng(count)
        srcs = rng.integers(0, og.n, count).astype(np.int32)
        if count > 2:
            srcs[1] = srcs[0]
        iso = np.nonzero(np.diff(og.rowptr) == 0)[0]
        if iso.size and count > 3:
            srcs[2] = iso[0]
        outs = {}
        for one_launch in (1, 0):
            G.tune_set("mssp_persistent", one_launch)
            try:
                d = torch.empty(count * og.n, dtype=torch.float64, device="cuda")
                st = G.TraversalStats()
                G._check(G.lib().ghb_mssssp(G._ws(None), og.n, G._ptr(g.rowptr), G._ptr(g.col), G._ptr(g.w),
                                            G._ptr(torch.from_numpy(srcs).cuda()), count, G.DBL_MAX, G._ptr(d),
                                            ctypes.byref(st)), "ghb_mssssp")
                assert st.levels >= 1 and st.edges_examined >= 0
                rg = G.ResidentGraph(g)
                outs[one_launch] = (d.cpu().numpy().reshape(count, og.n), rg.mssssp(srcs)[0].cpu().numpy())
                rg.close()
            finally:
                G.tune_set("mssp_persistent", 1)
        # Both drivers (one cooperative launch per pass, host-driven rounds)
        # give the same bits on every row.
        assert np.array_equal(outs[1][0], outs[0][0]) and np.array_equal(outs[1][1], outs[0][1])
        d, dr = outs[1]
        check = sorted({0, 1, 2, count // 2, count - 1} | set(range(0, count, 37)))
        for i in check:
            if i < count:
                ref = O.sssp(og, int(srcs[i]))
                assert np.array_equal(d[i], ref), i
                assert np.array_equal(dr[i], ref), i


def test_tc_complete_graph_long_oriented_rows(G):
    """K_1060: oriented rows of 0..1059 entries, so every hash path runs
    (warp hash up to 128 entries, block hash above), and with the block
    path capped at 200 entries the longest rows take the galloping walk;
    every vertex is in C(1059, 2) triangles (the reference counts 6x)."""
    n = 1060
    iu = torch.triu_indices(n, n, 1)
    src, dst = iu[0].int().cuda(), iu[1].int().cuda()
    g = G.make_graph(n, src, dst, False, weight_mode=G.WEIGHT_NONE)
    per_vertex = 6 * (n - 1) * (n - 2) // 2
    triangles = n * (n - 1) * (n - 2) // 6
    c64, c32, total = G.tc(g)
    assert total == triangles
    assert bool((c32 == per_vertex).all())
    rg = G.ResidentGraph(g)
    c64, c32, total = rg.tc()
    assert total == triangles and bool((c32 == per_vertex).all())
    ws = G.Workspace()
    for knob, value in (("tc_block_row", 200), ("tc_hash", 0)):
        G.tune_set(knob, value, ws=ws)
        c64, c32, total = G.tc(g, ws=ws)
        assert total == triangles and bool((c32 == per_vertex).all()), knob


def test_tc_hash_paths_match_oracle(G):
    """Oriented hash-probe TC against the oracle on RMAT (hub rows over the
    warp hash's 128 entries, rows over 4,096 entries oriented by the
    long-row kernel) and a sparse ER graph, with the range trim on every
    list, on lists over 32 entries and on none, with and without the block
    path, and against the galloping path."""
    for og in (O.rmat_graph(14, 16, 3, directed=False, weight_mode=0),
               O.make_graph(20000, *O.er_edges(20000, 60000, 8), False, weight_mode=0)):
        g = to_gpu(G, og)
        ref = O.tc(og)
        ws = G.Workspace()
        for knob, value in ((None, None), ("tc_slice_blocks", 1), ("tc_trim_min", 32), ("tc_trim_min", 1 << 20),
                            ("tc_block_row", 128), ("tc_hash", 0)):
            if knob:
                G.tune_set(knob, value, ws=ws)
            c64, c32, total = G.tc(g, ws=ws)
            assert np.array_equal(c32.cpu().numpy(), ref), knob
            assert int(c64.sum()) == 18 * total
