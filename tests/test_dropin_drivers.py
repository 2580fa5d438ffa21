"""The reference's own GPU drivers, compiled unchanged against this
repository's include/GPU_csr and include/GPU_gpma headers and linked to
libghb.so (make dropin):

* GPU_csr_example and GPU_gpma_example print the known answers of their
  6-vertex graph;
* LDBC_GPU_csr and LDBC_GPU_gpma load an LDBC Graphalytics dataset written
  here, run BFS, SSSP (+ SSSP with predecessors on the CSR path), WCC,
  PageRank and CDLP through the drop-in entry points and validate them with
  the reference's own checkers (include/LDBC/checker.hpp) against expected
  outputs from the CPU oracle.  The GPMA driver builds its graphs with
  update_gpma, so this also runs the dynamic graph's batch path.
"""
import os
import re
import subprocess

import numpy as np
import pytest

import oracle as O
from conftest import ROOT

pytestmark = pytest.mark.gpu

DROPIN = os.path.join(ROOT, "build", "dropin")
EXAMPLE = os.path.join(DROPIN, "GPU_csr_example")
LDBC = os.path.join(DROPIN, "LDBC_GPU_csr")
GPMA_EXAMPLE = os.path.join(DROPIN, "GPU_gpma_example")
GPMA_LDBC = os.path.join(DROPIN, "LDBC_GPU_gpma")

needs_example = pytest.mark.skipif(not os.path.exists(EXAMPLE), reason="drop-in drivers not built (make dropin)")
needs_ldbc = pytest.mark.skipif(not os.path.exists(LDBC), reason="drop-in drivers not built (make dropin)")


def sections(text):
    out, cur = {}, None
    for line in text.splitlines():
        if line.endswith("result:"):
            cur = line[: -len(" result:")]
            out[cur] = {}
        elif line.startswith("Running"):
            cur = None
        elif cur and len(line.split()) == 2:
            k, v = line.split()
            out[cur][k] = v
    return out


@pytest.mark.parametrize("binary", [EXAMPLE, GPMA_EXAMPLE], ids=["csr", "gpma"])
def test_gpu_example_known_answers(binary):
    if not os.path.exists(binary):
        pytest.skip("drop-in drivers not built (make dropin)")
    r = subprocess.run([binary], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    s = sections(r.stdout)
    assert s["BFS"] == {"one": "0", "two": "1", "three": "1", "four": "1", "five": "2", "six": "1"}
    assert s["Connected Components"] == {k: "one" for k in ["one", "two", "three", "four", "five", "six"]}
    assert s["SSSP"] == {"one": "0", "two": "0.8", "three": "1", "four": "1", "five": "2", "six": "1"}
    pr = {k: float(v) for k, v in s["PageRank"].items()}
    exp = {"one": 0.112218, "two": 0.136064, "three": 0.309545, "four": 0.136064, "five": 0.170045, "six": 0.136064}
    assert all(abs(pr[k] - exp[k]) < 1e-6 for k in exp)
    assert s["Community Detection"] == {k: "one" for k in ["one", "two", "three", "four", "five", "six"]}


def write_dataset(tmp, name, og: O.Graph, directed: bool, names, src):
    """LDBC files for graph og (ids = graph_structure ids = .v line order)."""
    d = os.path.join(tmp, name)
    n = og.n
    with open(os.path.join(tmp, name + ".v"), "w") as f:
        f.write("\n".join(names) + "\n")
    rows = np.repeat(np.arange(n), np.diff(og.rowptr))
    with open(os.path.join(tmp, name + ".e"), "w") as f:
        for u, v, w in zip(rows, og.col, og.w):
            if directed or u < v:
                f.write(f"{names[u]} {names[v]} {float(w)!r}\n")
    m = og.m if directed else og.m // 2
    props = {
        "vertex-file": name + ".v", "edge-file": name + ".e", "vertices": n, "edges": m,
        "directed": "true" if directed else "false", "edge-properties.names": "weight",
        "algorithms": "bfs, cdlp, pr, sssp, wcc", "bfs.source-vertex": names[src],
        "cdlp.max-iterations": 10, "pr.damping-factor": 0.85, "pr.num-iterations": 10,
        "sssp.weight-property": "weight", "sssp.source-vertex": names[src],
    }
    with open(os.path.join(tmp, name + ".properties"), "w") as f:
        for k, v in props.items():
            f.write(f"graph.{name}.{k} = {v}\n")
    bfs = O.bfs(og, src)
    with open(d + "-BFS", "w") as f:
        for i in range(n):
            f.write(f"{names[i]} {bfs[i] if bfs[i] != 2**31 - 1 else 9223372036854775807}\n")
    sssp = O.sssp(og, src)
    with open(d + "-SSSP", "w") as f:
        for i in range(n):
            f.write(f"{names[i]} {'infinity' if sssp[i] == O.DBL_MAX else repr(float(sssp[i]))}\n")
    wcc = O.wcc(og)
    with open(d + "-WCC", "w") as f:
        for i in range(n):
            f.write(f"{names[i]} {names[wcc[i]]}\n")
    pr = O.pagerank(og, 10, 0.85)
    with open(d + "-PR", "w") as f:
        for i in range(n):
            f.write(f"{names[i]} {float(pr[i])!r}\n")
    cd = O.cdlp(og, 10)
    with open(d + "-CDLP", "w") as f:
        for i in range(n):
            f.write(f"{names[i]} {names[cd[i]]}\n")


@pytest.mark.parametrize("binary,csv,n_results", [(LDBC, "result-gpu-csr.csv", 5),
                                                   (GPMA_LDBC, "result-gpu-gpma.csv", 5)], ids=["csr", "gpma"])
@pytest.mark.parametrize("directed", [True, False])
def test_ldbc_driver_validates_with_reference_checkers(tmp_path, directed, binary, csv, n_results):
    if not os.path.exists(binary):
        pytest.skip("drop-in drivers not built (make dropin)")
    og = O.rmat_graph(10, 8, 13, directed=directed)
    n = og.n
    names = [str(1000003 + 7919 * i) for i in range(n)]
    src = int(np.argmax(np.diff(og.rowptr)))
    name = "rmat10" + ("d" if directed else "u")
    write_dataset(str(tmp_path), name, og, directed, names, src)
    r = subprocess.run([binary], input=f"{tmp_path}/\n{name}\n", capture_output=True, text=True, timeout=600,
                       cwd=str(tmp_path))
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    for what in ["BFS", "SSSP", "WCC", "PageRank", "CDLP"]:
        assert f"{what} results are correct!" in r.stdout, r.stdout[-3000:]
    assert "Error: pre_v is wrong" not in r.stdout and "Not found!" not in r.stdout
    row = open(os.path.join(str(tmp_path), csv)).read().strip().split(",")
    assert len(row) == n_results and all(re.fullmatch(r"[0-9.]+", x) for x in row), row
