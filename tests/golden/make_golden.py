"""Regenerates the golden fixtures in this folder.

Every expected output here comes from the reference's own CPU algorithms
(GraphHET include/CPU_adj_list/algorithm/*.hpp), compiled from the reference
tree by oracle/Makefile into oracle/_ref/libref.so and run on the graphs
below.  Run from the repository root, where the reference tree is present:

    make -C oracle && python tests/golden/make_golden.py

Each fixture stores the input edge list, the CSR built from it (the layout
the reference's toCSR produces from graph_structure's sorted rows) and the
reference outputs: BFS depths and SSSP distances from `src`, WCC labels,
PageRank (10 iterations, d = 0.85), CDLP labels (10 iterations) and the
per-vertex triangle counts.  gpma/ holds dynamic-graph fixtures: a graph,
update batches, and the reference's rows after each batch.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.abspath(os.path.join(HERE, "..", "..")))

import oracle as O  # noqa: E402


def run_ref(name, g, src, extra=None):
    r = O.Ref().load(g)
    out = dict(
        n=np.int64(g.n), directed=np.int64(g.directed), src=np.int64(src),
        rowptr=g.rowptr, col=g.col, w=g.w if g.w is not None else np.zeros(0),
        in_rowptr=g.in_rowptr, in_col=g.in_col,
        bfs=r.bfs(src), sssp=r.sssp(src), wcc=r.wcc(), pagerank=r.pagerank(10, 0.85),
        cdlp=r.cdlp(10), tc=r.tc(),
    )
    if extra:
        out.update(extra)
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
    print(name, "n", g.n, "m", g.m)


def from_edges(name, n, edges, directed, src):
    src_a = np.array([e[0] for e in edges], np.int32)
    dst_a = np.array([e[1] for e in edges], np.int32)
    w = np.array([e[2] for e in edges], np.float64)
    g = O.make_graph(n, src_a, dst_a, directed, w=w)
    run_ref(name, g, src, dict(edge_src=src_a, edge_dst=dst_a, edge_w=w))


def main():
    # The graph of the reference's GPU_csr_example.cu after its removals and
    # re-insertions: one=0 two=1 three=2 four=3 five=4 six=5 (six reuses R's id).
    toy = [(0, 1, 0.8), (1, 2, 1.0), (0, 2, 1.0), (0, 3, 1.0), (3, 2, 1.0), (3, 4, 1.0), (0, 5, 1.0)]
    from_edges("toy_example_directed", 6, toy, True, 0)
    # One triangle {0,1,2}, a pendant 3 and an isolated 4 (undirected).
    tri = [(0, 1, 1.0), (1, 2, 1.0), (0, 2, 1.0), (2, 3, 1.0)]
    from_edges("triangle_pendant_isolated", 5, tri, False, 0)
    # Duplicates, a self-loop and both directions of one pair in a directed
    # edge list: the builder merges pairs (last weight wins) and drops loops.
    dup = [(0, 1, 0.5), (0, 1, 0.25), (1, 0, 0.75), (2, 2, 1.0), (1, 2, 0.125), (3, 1, 2.0), (1, 2, 0.0625)]
    from_edges("duplicates_directed", 5, dup, True, 0)
    # Path and star (undirected).
    from_edges("path_undirected", 9, [(i, i + 1, 1.0 + i) for i in range(8)], False, 0)
    from_edges("star_undirected", 17, [(0, i, 0.5 * i) for i in range(1, 17)], False, 3)
    # Seeded synthetic graphs (include/ghb_gen.h), small enough to commit.
    for directed in (False, True):
        g = O.rmat_graph(10, 16, 42, directed=directed)
        deg = np.diff(g.rowptr)
        src = int(np.argmax(deg))
        run_ref(f"rmat10_seed42_{'directed' if directed else 'undirected'}", g, src,
                dict(scale=np.int64(10), edge_factor=np.int64(16), seed=np.int64(42)))
    g = O.grid_graph(16, 16, weight_seed=1)
    run_ref("grid16x16", g, 0, dict(rows=np.int64(16), cols=np.int64(16), seed=np.int64(1)))
    s, d = O.er_edges(3000, 9000, 5)
    g = O.make_graph(3000, s, d, False, weight_mode=1, weight_seed=5)
    run_ref("er3000_seed5", g, 0, dict(er_n=np.int64(3000), er_m=np.int64(9000), seed=np.int64(5)))
    gpma_fixture()


def gpma_batches(rowptr, col, n, n_batches, size, seed):
    """Seeded update batches over a graph: new edges, weight changes and
    deletes of present edges, deletes of absent ones, self-loops, and repeats
    of keys inside a batch (the later value must win)."""
    rng = np.random.default_rng(seed)
    rows = np.repeat(np.arange(n), np.diff(rowptr))
    present = list(zip(rows.tolist(), np.asarray(col).tolist()))
    out = []
    for _ in range(n_batches):
        q = size // 8
        s, d, w = [], [], []
        for _ in range(2 * q):  # inserts (or overwrites when present)
            s.append(int(rng.integers(n))); d.append(int(rng.integers(n))); w.append(float(rng.uniform(0.25, 2.0)))
        for i in rng.integers(len(present), size=2 * q):  # deletes of present edges
            s.append(present[i][0]); d.append(present[i][1]); w.append(0.0)
        for _ in range(q):  # deletes of (mostly) absent edges
            s.append(int(rng.integers(n))); d.append(int(rng.integers(n))); w.append(0.0)
        for i in rng.integers(len(present), size=q):  # weight changes
            s.append(present[i][0]); d.append(present[i][1]); w.append(float(rng.uniform(0.25, 2.0)))
        for _ in range(q // 4):  # self-loops
            v = int(rng.integers(n)); s.append(v); d.append(v); w.append(1.5)
        perm = rng.permutation(len(s))
        s, d, w = np.array(s, np.int32)[perm], np.array(d, np.int32)[perm], np.array(w)[perm]
        rep = rng.integers(len(s), size=q)  # repeats with a new value (a third of them deletes)
        rw = np.where(rng.random(q) < 1 / 3, 0.0, rng.uniform(0.25, 2.0, q))
        s = np.concatenate([s, s[rep]]); d = np.concatenate([d, d[rep]]); w = np.concatenate([w, rw])
        out.append((s, d, w))
    return out


def gpma_fixture():
    """Dynamic-graph updates: the directed RMAT-9 graph (seed 42) edited by
    four seeded batches through the reference's graph_structure::add_edge /
    remove_edge (the edits the GPMA drivers mirror, LDBC_GPU_gpma.cu:124-148),
    with the reference's out-rows after every batch."""
    g = O.rmat_graph(9, 16, 42, directed=True)
    r = O.Ref().load(g)
    batches = gpma_batches(g.rowptr, g.col, g.n, 4, 2048, 2024)
    out = dict(n=np.int64(g.n), rowptr=g.rowptr, col=g.col, w=g.w)
    for i, (s, d, w) in enumerate(batches):
        r.apply_updates(s, d, w)
        rp, c, ww = r.export_out()
        out.update({f"b{i}_src": s, f"b{i}_dst": d, f"b{i}_w": w, f"a{i}_rowptr": rp, f"a{i}_col": c, f"a{i}_w": ww})
    os.makedirs(os.path.join(HERE, "gpma"), exist_ok=True)
    np.savez_compressed(os.path.join(HERE, "gpma", "rmat9_seed42_batches.npz"), **out)
    print("gpma rmat9_seed42_batches", [int(out[f"a{i}_rowptr"][-1]) for i in range(4)])


if __name__ == "__main__":
    main()
