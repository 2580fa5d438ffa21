"""ghb_ldbc_load: LDBC .v/.e text straight into device CSRs, with the
reference loader's rules (include/LDBC/ldbc.hpp:181-253 and
graph_structure::add_vertice / add_edge, CPU_adj_list.hpp:75-122): ids by
first appearance (.v lines, then names first met in .e, a before b), weight =
third field else 1, both directions when undirected, last weight wins for a
repeated ordered pair, self-loops kept.  The expected CSR is built here by
restating those rules and the oracle's CSR builder."""
import numpy as np
import pytest
import torch

import oracle as O

pytestmark = pytest.mark.gpu


def write_files(tmp, rng, weighted):
    names = ["n%d" % i for i in rng.permutation(400)]
    v_lines = names[:300] + [names[5], names[17]]          # repeated names keep their first id
    lines = []
    for _ in range(3000):
        a = names[int(rng.integers(0, 400))]             # names 300..399 appear first in .e
        b = names[int(rng.integers(0, 400))] if rng.random() > 0.02 else a   # self-loops
        if weighted:
            lines.append("%s %s %.17g" % (a, b, rng.uniform(0.001, 1.0)))
        else:
            lines.append("%s %s" % (a, b))
    lines += lines[:50]                                   # repeated pairs (same weights)
    if weighted:
        lines += ["%s %.17g" % (" ".join(l.split()[:2]), 7.5) for l in lines[100:120]]  # last weight wins
    lines.append("lonely")                                # fewer than two fields: skipped
    (tmp / "g.v").write_text("\n".join(v_lines) + "\n")
    (tmp / "g.e").write_text("\n".join(lines) + "\n")
    return v_lines, lines


def expected(v_lines, lines, directed, weighted):
    ids, order = {}, []
    def add(nm):
        if nm not in ids:
            ids[nm] = len(order)
            order.append(nm)
        return ids[nm]
    for nm in v_lines:
        add(nm)
    src, dst, w = [], [], []
    for l in lines:
        f = l.split(" ")
        if len(f) < 2:
            continue
        a, b = add(f[0]), add(f[1])
        src.append(a)
        dst.append(b)
        w.append(float(f[2]) if len(f) > 2 else 1.0)
    n = len(order)
    rp, col, wt = O.build_csr(n, np.array(src, np.int32), np.array(dst, np.int32), w=np.array(w),
                              symmetrize=not directed, drop_self_loops=False)
    return n, order, rp, col, wt


@pytest.mark.parametrize("directed", [False, True])
@pytest.mark.parametrize("weighted", [False, True])
def test_ldbc_loader_matches_reference_rules(tmp_path, directed, weighted):
    import graphhet_b200 as G
    rng = np.random.default_rng(3 + 2 * directed + weighted)
    v_lines, lines = write_files(tmp_path, rng, weighted)
    g, names = G.load_ldbc(str(tmp_path / "g.v"), str(tmp_path / "g.e"), directed)
    n, order, rp, col, wt = expected(v_lines, lines, directed, weighted)
    assert names == order and g.n == n
    assert np.array_equal(g.rowptr.cpu().numpy(), rp)
    assert np.array_equal(g.col.cpu().numpy(), col)
    assert np.array_equal(g.w.cpu().numpy(), wt)
    if directed:
        t_rp, t_col, t_w = G.transpose_csr(n, torch.from_numpy(rp).cuda(), torch.from_numpy(col).cuda(),
                                           torch.from_numpy(wt).cuda())
        assert torch.equal(g.in_rowptr, t_rp) and torch.equal(g.in_col, t_col) and torch.equal(g.in_w, t_w)


def test_loaded_graph_results_round_trip_through_validation_files(tmp_path):
    """Load an LDBC dataset, run BFS / SSSP / WCC / PR / CDLP on it, write
    LDBC validation files, and check them against the oracle's results with
    the reference checkers' rules (graphhet_b200.validation)."""
    import graphhet_b200 as G
    from graphhet_b200 import validation as V
    rng = np.random.default_rng(9)
    v_lines, lines = write_files(tmp_path, rng, True)
    g, names = G.load_ldbc(str(tmp_path / "g.v"), str(tmp_path / "g.e"), False)
    n, order, rp, col, wt = expected(v_lines, lines, False, True)
    og = O.Graph(n=n, rowptr=rp, col=col, w=wt, directed=False, in_rowptr=rp, in_col=col, in_w=wt)
    src = 3
    res = {
        "bfs": (G.bfs(g, src)[0].cpu().numpy(), O.bfs(og, src)),
        "sssp": (G.sssp(g, src)[0].cpu().numpy(), O.sssp(og, src)),
        "wcc": (G.wcc(g).cpu().numpy(), O.wcc(og)),
        "pr": (G.pagerank(g, 10, 0.85)[0].cpu().numpy(), O.pagerank(og, 10, 0.85)),
        "cdlp": (G.cdlp(g, 10).cpu().numpy(), O.cdlp(og, 10)),
    }
    for kind, (ours, ref) in res.items():
        path = str(tmp_path / ("ref." + kind))
        V.write(path, kind, names, ref)
        ok, msg = V.check(path, kind, names, ours)
        assert ok, (kind, msg)
