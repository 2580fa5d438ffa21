"""Seeded inputs and the CPU CSR builder: determinism and invariants."""
import numpy as np

import oracle as O


def test_rmat_is_deterministic_and_seed_dependent():
    a = O.rmat_edges(12, 1 << 14, 42)
    b = O.rmat_edges(12, 1 << 14, 42)
    c = O.rmat_edges(12, 1 << 14, 43)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    assert not np.array_equal(a[0], c[0])
    assert a[0].min() >= 0 and a[0].max() < 4096


def test_rmat_skew_follows_parameters():
    s, d = O.rmat_edges(14, 1 << 18, 3, permute=False)
    # quadrant a = 0.57: the top bit of both endpoints is 0 for ~57% of edges
    top = ((s >> 13) == 0) & ((d >> 13) == 0)
    assert abs(top.mean() - 0.57) < 0.01


def test_permutation_is_a_bijection():
    s, _ = O.rmat_edges(10, 1 << 16, 9, permute=False)
    sp, _ = O.rmat_edges(10, 1 << 16, 9, permute=True)
    # same multiset sizes per vertex after relabelling
    assert np.array_equal(np.sort(np.bincount(s, minlength=1024)), np.sort(np.bincount(sp, minlength=1024)))


def test_symmetric_csr_invariants():
    g = O.rmat_graph(11, 16, 1, directed=False)
    rp, col = g.rowptr, g.col
    rows = np.repeat(np.arange(g.n), np.diff(rp))
    assert np.all(rows != col), "self-loop left"
    for u in range(0, g.n, 97):
        r = col[rp[u]:rp[u + 1]]
        assert np.all(np.diff(r) > 0), "row not strictly increasing"
    key = rows.astype(np.int64) << 32 | col
    rkey = col.astype(np.int64) << 32 | rows
    assert np.array_equal(np.sort(key), np.sort(rkey)), "not symmetric"
    # one weight per undirected pair
    wk = dict(zip(key.tolist(), g.w.tolist()))
    for k, w in list(wk.items())[:2000]:
        u, v = k >> 32, k & 0xFFFFFFFF
        assert wk[(v << 32) | u] == w
    assert np.all((g.w > 0) & (g.w <= 1))


def test_directed_in_csr_is_transpose():
    g = O.rmat_graph(10, 8, 2, directed=True)
    rows = np.repeat(np.arange(g.n), np.diff(g.rowptr))
    irows = np.repeat(np.arange(g.n), np.diff(g.in_rowptr))
    a = np.sort(rows.astype(np.int64) << 32 | g.col)
    b = np.sort(g.in_col.astype(np.int64) << 32 | irows)
    assert np.array_equal(a, b)


def test_grid_shape_and_weights():
    g = O.grid_graph(8, 5, weight_seed=4)
    assert g.n == 40 and g.m == 2 * (8 * 4 + 7 * 5)
    assert np.all(g.w == np.round(g.w)) and g.w.min() >= 1 and g.w.max() <= 100
