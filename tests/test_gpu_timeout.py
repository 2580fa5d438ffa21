"""The bounded grid barrier's timeout path.

Every wait of a persistent kernel on its grid barrier gives up after the
workspace's "barrier_limit_us"; the kernel then leaves and the call returns
GHB_ERR_TIMEOUT, with the device still usable.  The test knob
"barrier_extra" makes every barrier wait for one arrival more than there are
blocks, a wait that nothing ends, so the limit is what ends it.  Nothing
faults or hangs: each block's wait ends on its own clock after about a
millisecond.  The same workspace then runs a normal traversal, checked
against the oracle."""
import ctypes

import numpy as np
import pytest
import torch

import oracle as O

pytestmark = pytest.mark.gpu

GHB_ERR_TIMEOUT = 4


@pytest.fixture(scope="module")
def G():
    import graphhet_b200 as G
    G.lib()
    return G


def test_bfs_barrier_timeout_then_recovers(G):
    og = O.rmat_graph(12, 16, 42, directed=False)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    g = G.CSRGraph(n=og.n, rowptr=t(og.rowptr), col=t(og.col), w=None, directed=False)
    ws = G.Workspace()
    rg = G.ResidentGraph(g, ws=ws)
    src = int(np.argmax(np.diff(og.rowptr)))
    L = G.lib()
    depth = torch.empty(og.n, dtype=torch.int32, device="cuda")
    st = G.TraversalStats()
    opt = G.BfsOptions(policy=G.POLICY_HEURISTIC)

    G.tune_set("barrier_limit_us", 1000, ws=ws)
    G.tune_set("barrier_extra", 1, ws=ws)
    rc = L.ghb_graph_bfs(ws.handle, rg._h, src, G.INT32_MAX, G._ptr(depth), ctypes.byref(opt), ctypes.byref(st))
    assert rc == GHB_ERR_TIMEOUT
    assert "timed out" in L.ghb_last_error().decode()
    assert L.ghb_status_string(rc).decode() == "device wait timed out"
    torch.cuda.synchronize()  # the context is intact: no sticky error

    G.tune_set("barrier_extra", 0, ws=ws)
    G.tune_set("barrier_limit_us", 2000000, ws=ws)
    rc = L.ghb_graph_bfs(ws.handle, rg._h, src, G.INT32_MAX, G._ptr(depth), ctypes.byref(opt), ctypes.byref(st))
    assert rc == 0, L.ghb_last_error().decode()
    assert np.array_equal(depth.cpu().numpy(), O.bfs(og, src))
    rg.close()


def test_barrier_knobs_are_range_checked(G):
    ws = G.Workspace()
    with pytest.raises(G.GhbError):
        G.tune_set("barrier_extra", 2, ws=ws)
    with pytest.raises(G.GhbError):
        G.tune_set("barrier_limit_us", 10, ws=ws)
    assert G.tune_get("barrier_limit_us", ws=ws) == 2000000
    assert G.tune_get("barrier_extra", ws=ws) == 0


def test_sssp_barrier_timeout_then_recovers(G):
    og = O.rmat_graph(12, 16, 42, directed=False)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    g = G.CSRGraph(n=og.n, rowptr=t(og.rowptr), col=t(og.col), w=t(og.w), directed=False)
    ws = G.Workspace()
    rg = G.ResidentGraph(g, ws=ws)
    src = int(np.argmax(np.diff(og.rowptr)))
    G.tune_set("barrier_limit_us", 1000, ws=ws)
    G.tune_set("barrier_extra", 1, ws=ws)
    for call in (lambda: rg.sssp(src, ws=ws), lambda: G.sssp(g, src, ws=ws)):
        with pytest.raises(G.GhbError, match="timed out"):
            call()
    torch.cuda.synchronize()
    G.tune_set("barrier_extra", 0, ws=ws)
    G.tune_set("barrier_limit_us", 2000000, ws=ws)
    ref = O.sssp(og, src)
    assert np.array_equal(rg.sssp(src, ws=ws)[0].cpu().numpy(), ref)
    assert np.array_equal(G.sssp(g, src, ws=ws)[0].cpu().numpy(), ref)
    rg.close()


def test_multi_source_barrier_timeout_then_recovers(G):
    """The one-launch multi-source BFS and SSSP passes give up on the same
    bounded barrier, return GHB_ERR_TIMEOUT, and the workspace runs the
    next pass normally."""
    og = O.rmat_graph(12, 16, 42, directed=False)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    g = G.CSRGraph(n=og.n, rowptr=t(og.rowptr), col=t(og.col), w=t(og.w), directed=False)
    ws = G.Workspace()
    rg = G.ResidentGraph(g, ws=ws)
    srcs = np.array([0, 5, 17, 300, 4095], dtype=np.int32)
    G.tune_set("barrier_limit_us", 1000, ws=ws)
    G.tune_set("barrier_extra", 1, ws=ws)
    for call in (lambda: rg.msbfs(srcs, ws=ws), lambda: rg.mssssp(srcs, ws=ws)):
        with pytest.raises(G.GhbError, match="timed out"):
            call()
    torch.cuda.synchronize()
    G.tune_set("barrier_extra", 0, ws=ws)
    G.tune_set("barrier_limit_us", 2000000, ws=ws)
    depth = rg.msbfs(srcs, ws=ws)[0].cpu().numpy().reshape(len(srcs), og.n)
    dist = rg.mssssp(srcs, ws=ws)[0].cpu().numpy().reshape(len(srcs), og.n)
    for i, s in enumerate(srcs):
        assert np.array_equal(depth[i], O.bfs(og, int(s)))
        assert np.array_equal(dist[i], O.sssp(og, int(s)))
    rg.close()
