"""Dynamic graph (ghb_gpma_*, the reference's GPMA update path): the device
structure after every batch against the oracle's update_gpma restatement,
bit-exact (rows, columns and weights), on the reference-made fixture, on
random batches large enough to move rows and repack the arena, from an
empty graph up and back down; then every analytic on the updated graph."""
import os

import numpy as np
import pytest
import torch

import oracle as O
from conftest import GOLDEN

pytestmark = pytest.mark.gpu

FIX = os.path.join(GOLDEN, "gpma", "rmat9_seed42_batches.npz")


@pytest.fixture(scope="module")
def G():
    import graphhet_b200 as G
    G.lib()
    return G


def t(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def assert_state(dg, n, keys, vals):
    cg = dg.csr_graph(weights=True)
    rp, col, w = O.gpma_to_csr(n, keys, vals)
    assert np.array_equal(cg.rowptr.cpu().numpy(), rp)
    assert np.array_equal(cg.col.cpu().numpy(), col)
    assert np.array_equal(cg.w.cpu().numpy(), w)
    assert dg.m == len(keys)
    # the cached snapshot without weights agrees as well
    cg2 = dg.csr_graph(weights=False)
    assert np.array_equal(cg2.col.cpu().numpy(), col)


def update(dg, keys, vals, bk, bv):
    got = dg.update(t(bk), t(bv))
    keys, vals, counts = O.gpma_update(keys, vals, bk, bv)
    assert (got["inserted"], got["deleted"], got["modified"], got["ignored"]) == counts
    return keys, vals


def test_load_export_roundtrip(G):
    og = O.rmat_graph(12, 16, 3, directed=True)
    dg = G.DynamicGraph.from_csr(t(og.rowptr), t(og.col), t(og.w))
    keys, vals = O.gpma_from_csr(og.rowptr, og.col, og.w)
    assert_state(dg, og.n, keys, vals)
    dg1 = G.DynamicGraph.from_csr(t(og.rowptr), t(og.col))  # weight 1
    assert_state(dg1, og.n, keys, np.ones(len(keys)))


def test_reference_fixture_batches(G):
    z = np.load(FIX)
    n = int(z["n"])
    dg = G.DynamicGraph.from_csr(t(z["rowptr"]), t(z["col"]), t(z["w"]))
    keys, vals = O.gpma_from_csr(z["rowptr"], z["col"], z["w"])
    for i in range(4):
        keys, vals = update(dg, keys, vals, O.gpma_keys(z[f"b{i}_src"], z[f"b{i}_dst"]), z[f"b{i}_w"])
        cg = dg.csr_graph(weights=True)
        assert np.array_equal(cg.rowptr.cpu().numpy(), z[f"a{i}_rowptr"])
        assert np.array_equal(cg.col.cpu().numpy(), z[f"a{i}_col"])
        assert np.array_equal(cg.w.cpu().numpy(), z[f"a{i}_w"])


def random_batch(rng, n, keys, size, hubs=None):
    k_present = keys[rng.integers(len(keys), size=size // 4)] if len(keys) else np.zeros(0, np.int64)
    src = rng.integers(n, size=size // 2)
    if hubs is not None:  # pile inserts onto a few rows so they outgrow their slack
        src[: size // 4] = rng.choice(hubs, size=size // 4)
    fresh = O.gpma_keys(src, rng.integers(n, size=size // 2))
    bk = np.concatenate([k_present, fresh, k_present[: size // 8]])
    bv = np.where(rng.random(len(bk)) < 0.3, 0.0, rng.uniform(0.1, 3.0, len(bk)))
    perm = rng.permutation(len(bk))
    return bk[perm], bv[perm]


def test_random_batches_move_rows_and_repack(G):
    og = O.rmat_graph(14, 8, 11, directed=True)
    n = og.n
    dg = G.DynamicGraph.from_csr(t(og.rowptr), t(og.col), t(og.w))
    keys, vals = O.gpma_from_csr(og.rowptr, og.col, og.w)
    rng = np.random.default_rng(5)
    hubs = np.argsort(-np.diff(og.rowptr))[:16]
    for size in [1, 7, 1000, 50000, 3, 200000, 120000, 0, 400000, 64]:
        bk, bv = random_batch(rng, n, keys, size, hubs=hubs)
        keys, vals = update(dg, keys, vals, bk, bv)
        assert_state(dg, n, keys, vals)
    st = dg.stats()
    assert st["rows_moved"] > 0 and st["repacks"] >= 1, st
    assert st["slots_used"] <= st["slots"]
    # lookups
    probe = np.concatenate([keys[:: max(1, len(keys) // 1000)], O.gpma_keys([0, 1, n - 1], [n - 1, 0, 5])])
    expect = dict(zip(keys.tolist(), vals.tolist()))
    got = dg.find(t(probe)).cpu().numpy()
    assert np.array_equal(got, np.array([expect.get(k, 0.0) for k in probe.tolist()]))


def test_grow_from_empty_and_delete_all(G):
    og = O.rmat_graph(12, 16, 9, directed=True)
    n = og.n
    keys_all, vals_all = O.gpma_from_csr(og.rowptr, og.col, og.w)
    dg = G.DynamicGraph(n)
    keys, vals = np.zeros(0, np.int64), np.zeros(0)
    assert_state(dg, n, keys, vals)
    for part in np.array_split(np.random.default_rng(1).permutation(len(keys_all)), 3):
        keys, vals = update(dg, keys, vals, keys_all[part], vals_all[part])
        assert_state(dg, n, keys, vals)
    assert np.array_equal(keys, keys_all)
    keys, vals = update(dg, keys, vals, keys_all, np.zeros(len(keys_all)))
    assert len(keys) == 0
    assert_state(dg, n, keys, vals)
    assert dg.csr_graph().rowptr.cpu().numpy().tolist() == [0] * (n + 1)


def test_invalid_key_rejected_without_change(G):
    og = O.rmat_graph(10, 8, 2, directed=True)
    dg = G.DynamicGraph.from_csr(t(og.rowptr), t(og.col), t(og.w))
    keys, vals = O.gpma_from_csr(og.rowptr, og.col, og.w)
    version = dg.info()[3]
    bad = O.gpma_keys([1, og.n], [2, 3])  # row n is outside [0, n)
    with pytest.raises(G.GhbError):
        dg.update(t(bad), t(np.array([1.0, 1.0])))
    bad = O.gpma_keys([1, 2], [2, og.n + 5])
    with pytest.raises(G.GhbError):
        dg.update(t(bad), t(np.array([1.0, 1.0])))
    assert dg.info()[3] == version
    assert_state(dg, og.n, keys, vals)
    with pytest.raises(G.GhbError):  # unsorted rows are refused by the loader
        G.DynamicGraph.from_csr(t(np.array([0, 2], np.int32)), t(np.array([0, 0], np.int32)))
    with pytest.raises(G.GhbError):  # a weight of 0 would mark a deleted entry
        G.DynamicGraph.from_csr(t(np.array([0, 1, 1], np.int32)), t(np.array([1], np.int32)),
                                t(np.array([0.0])))


def test_clone_is_independent(G):
    og = O.rmat_graph(11, 8, 4, directed=True)
    dg = G.DynamicGraph.from_csr(t(og.rowptr), t(og.col), t(og.w))
    keys, vals = O.gpma_from_csr(og.rowptr, og.col, og.w)
    cl = dg.clone()
    rng = np.random.default_rng(8)
    bk, bv = random_batch(rng, og.n, keys, 5000)
    k2, v2 = update(cl, keys, vals, bk, bv)
    assert_state(dg, og.n, keys, vals)
    assert_state(cl, og.n, k2, v2)
    dg.close()
    assert_state(cl, og.n, k2, v2)


def test_batch_larger_than_one_pass(G):
    """More than 2^25 updates in one call run as consecutive passes; repeats
    across the pass boundary keep the last value."""
    n = 1 << 20
    rng = np.random.default_rng(12)
    size = (1 << 25) + 1_000_000
    bk = O.gpma_keys(rng.integers(n, size=size), rng.integers(n, size=size))
    bk[-500_000:] = bk[:500_000]  # repeats straddling the boundary
    bv = rng.uniform(0.1, 3.0, size)
    bv[-100_000:] = 0.0
    dg = G.DynamicGraph(n)
    got = dg.update(t(bk), t(bv))
    keys, vals, _ = O.gpma_update(np.zeros(0, np.int64), np.zeros(0), bk, bv)
    assert_state(dg, n, keys, vals)
    # Passes count their own effects (a repeat in the second pass modifies or
    # deletes what the first inserted); the net count is the same.
    assert got["inserted"] - got["deleted"] == len(keys)
    assert sum(got.values()) == len(bk)


def symmetric_batch(rng, n, keys, size):
    """Updates of undirected edges, both directions with the same value, no
    self-loops."""
    und = keys[(keys >> 32) < (keys & 0xFFFFFFFF)]
    old = und[rng.integers(len(und), size=size // 2)]
    u, v = rng.integers(n, size=size), rng.integers(n, size=size)
    keep = u != v
    new = O.gpma_keys(np.minimum(u, v)[keep], np.maximum(u, v)[keep])
    k = np.concatenate([old, new])
    w = np.where(rng.random(len(k)) < 0.5, 0.0, rng.uniform(0.1, 2.0, len(k)))
    rev = ((k & 0xFFFFFFFF) << 32) | (k >> 32)
    return np.concatenate([k, rev]), np.concatenate([w, w])


def test_analytics_after_updates(G):
    og = O.rmat_graph(12, 16, 21, directed=False)
    n = og.n
    dg = G.DynamicGraph.from_csr(t(og.rowptr), t(og.col), t(og.w))
    keys, vals = O.gpma_from_csr(og.rowptr, og.col, og.w)
    rng = np.random.default_rng(3)
    for _ in range(3):
        bk, bv = symmetric_batch(rng, n, keys, 6000)
        keys, vals = update(dg, keys, vals, bk, bv)
    rp, col, w = O.gpma_to_csr(n, keys, vals)
    upd = O.Graph(n, rp, col, w, False, rp, col, w)
    g = dg.csr_graph(weights=True)
    src = int(np.argmax(np.diff(rp)))
    assert np.array_equal(G.bfs(g, src)[0].cpu().numpy(), O.bfs(upd, src))
    assert np.array_equal(G.sssp(g, src)[0].cpu().numpy(), O.sssp(upd, src))
    assert np.array_equal(G.wcc(g).cpu().numpy(), O.wcc(upd))
    pr, _, _ = G.pagerank(g, 10, 0.85)
    ref = O.pagerank(upd, 10, 0.85)
    assert float(np.abs(pr.cpu().numpy() - ref).sum() / np.abs(ref).sum()) <= 1e-6
    assert np.array_equal(G.cdlp(g, 10).cpu().numpy(), O.cdlp(upd, 10))
    assert np.array_equal(G.tc(g)[1].cpu().numpy(), O.tc(upd))
    rg = G.ResidentGraph(g)
    assert np.array_equal(rg.bfs(src)[0].cpu().numpy(), O.bfs(upd, src))


def test_directed_out_and_in_graphs(G):
    """The reference's pair of GPMAs for a directed graph (out rows keyed
    (u, v), in rows keyed (v, u), LDBC_GPU_gpma.cu:155-211): both take the same
    edits, and the analytics read them as one directed CSRGraph."""
    og = O.rmat_graph(12, 16, 31, directed=True)
    n = og.n
    out_g = G.DynamicGraph.from_csr(t(og.rowptr), t(og.col), t(og.w))
    in_g = G.DynamicGraph.from_csr(t(og.in_rowptr), t(og.in_col), t(og.in_w))
    keys, vals = O.gpma_from_csr(og.rowptr, og.col, og.w)
    rng = np.random.default_rng(17)
    for _ in range(3):
        bk, bv = random_batch(rng, n, keys, 8000)
        keep = (bk >> 32) != (bk & 0xFFFFFFFF)  # no self-loops
        bk, bv = bk[keep], bv[keep]
        keys, vals = update(out_g, keys, vals, bk, bv)
        rev = ((bk & 0xFFFFFFFF) << 32) | (bk >> 32)
        in_g.update(t(rev), t(bv))
    rp, col, w = O.gpma_to_csr(n, keys, vals)
    rk = ((keys & 0xFFFFFFFF) << 32) | (keys >> 32)
    o = np.argsort(rk)
    irp, icol, iw = O.gpma_to_csr(n, rk[o], vals[o])
    upd = O.Graph(n, rp, col, w, True, irp, icol, iw)
    for g in (out_g.csr_graph(directed=True, in_graph=in_g), out_g.csr_graph(directed=True)):
        assert np.array_equal(g.in_rowptr.cpu().numpy(), irp) and np.array_equal(g.in_col.cpu().numpy(), icol)
        src = int(np.argmax(np.diff(rp)))
        assert np.array_equal(G.bfs(g, src)[0].cpu().numpy(), O.bfs(upd, src))
        assert np.array_equal(G.sssp(g, src)[0].cpu().numpy(), O.sssp(upd, src))
        assert np.array_equal(G.wcc(g).cpu().numpy(), O.wcc(upd))
        pr, _, _ = G.pagerank(g, 10, 0.85)
        ref = O.pagerank(upd, 10, 0.85)
        assert float(np.abs(pr.cpu().numpy() - ref).sum() / np.abs(ref).sum()) <= 1e-6
        assert np.array_equal(G.cdlp(g, 10).cpu().numpy(), O.cdlp(upd, 10))


def test_long_rows_take_the_flattened_path(G):
    """Rows with more than 4,096 existing entries + updates are rebuilt by the
    grid-wide kernels: a star whose centre row grows, shrinks and moves."""
    n = 50000
    hub_cols = np.arange(1, 30001)
    rp = np.zeros(n + 1, np.int32)
    rp[1:] = len(hub_cols)
    dg = G.DynamicGraph.from_csr(t(rp), t(hub_cols.astype(np.int32)))
    keys, vals = O.gpma_from_csr(rp, hub_cols)
    rng = np.random.default_rng(4)
    for _ in range(4):
        c = rng.integers(n, size=20000)
        bk = O.gpma_keys(np.zeros(len(c), np.int64), c)
        bv = np.where(rng.random(len(c)) < 0.45, 0.0, rng.uniform(0.5, 1.5, len(c)))
        keys, vals = update(dg, keys, vals, bk, bv)
        assert_state(dg, n, keys, vals)
