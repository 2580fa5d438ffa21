"""Autotuner for libghb's launch shapes and thresholds (the workspace
tunables of ghb_tune_set): PageRank's hub-cache size, persistent block shape
and row split, and the multi-source BFS's block-row threshold and direction
switch.  None of them changes a result (PageRank stays within its 1e-6 bar,
every depth stays bit-exact; `tune` checks both), only the time.

The search is coordinate descent over a small grid per parameter, starting
from the current values: each candidate is timed with CUDA events (median of
`reps` calls after one warm-up call) on the caller's graph, the best value of
one parameter is kept before the next is tried, and the sweep runs twice.
Infeasible shapes (more than 2,048 threads or 224 KB of shared memory per SM)
are skipped.  `save` / `load` keep the chosen values as JSON.
"""
from __future__ import annotations

import json
import statistics
from typing import Callable, Dict, List, Optional, Sequence, Tuple

SPACES: Dict[str, Dict[str, List[int]]] = {
    "pagerank": {
        "pr_cache_kb": [0, 48, 96, 144, 192, 200],
        "pr_threads": [256, 512, 1024],
        "pr_blocks_per_sm": [1, 2, 4],
        "pr_short": [8, 16, 32, 64],
        "pr_chunk": [128, 256, 512, 1024],
    },
    "msbfs": {
        "ms_warp_rest": [64, 128, 256, 512, 2048],
        "ms_pull_div": [2, 4, 8, 16, 32],
    },
}


def feasible(cfg: Dict[str, int]) -> bool:
    threads = cfg.get("pr_threads", 1024) * cfg.get("pr_blocks_per_sm", 1)
    smem = cfg.get("pr_cache_kb", 192) * cfg.get("pr_blocks_per_sm", 1)
    return threads <= 2048 and smem <= 224


def _timer(fn: Callable[[], object], reps: int) -> float:
    import torch
    fn()
    times = []
    for _ in range(reps):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        s.record()
        fn()
        e.record()
        torch.cuda.synchronize()
        times.append(s.elapsed_time(e))
    return statistics.median(times)


def _workload(rg, algo: str, sources: Sequence[int], iterations: int):
    """(run, check) for one algorithm on a resident graph: run() launches it,
    check() compares its output with the first run's."""
    import torch
    import graphhet_b200 as G
    if algo == "pagerank":
        out = torch.empty(rg.n, dtype=torch.float64, device="cuda")
        ref = rg.pagerank(iterations, 0.85, precision=G.PR_FP32_KAHAN)[0].clone()

        def run():
            rg.pagerank(iterations, 0.85, precision=G.PR_FP32_KAHAN, out=out)

        def check():
            return float((out - ref).abs().sum() / ref.abs().sum()) <= 1e-6
        return run, check
    if algo == "msbfs":
        out = torch.empty(len(sources) * rg.n, dtype=torch.int32, device="cuda")
        ref = rg.msbfs(sources)[0].clone()

        def run():
            rg.msbfs(sources, out=out)

        def check():
            return bool(torch.equal(out[: len(sources) * rg.n].view(len(sources), rg.n), ref))
        return run, check
    raise ValueError("unknown algorithm %r" % algo)


def tune(rg, algo: str, sources: Sequence[int] = (), iterations: int = 10, reps: int = 3, rounds: int = 2,
         space: Optional[Dict[str, List[int]]] = None, ws=None, log=print) -> Tuple[Dict[str, int], List[dict]]:
    """Search the tunables of `algo` on resident graph `rg`; leaves the best
    values set on the workspace and returns them with the timing table."""
    import graphhet_b200 as G
    space = space or SPACES[algo]
    cfg = {k: G.tune_get(k, ws=ws) for k in space}
    run, check = _workload(rg, algo, list(sources), iterations)
    table = []

    def measure(c):
        for k, v in c.items():
            G.tune_set(k, v, ws=ws)
        ms = _timer(run, reps)
        ok = check()
        table.append(dict(c, ms=round(ms, 4), ok=ok))
        if log:
            log("%s %s %.4f ms%s" % (algo, c, ms, "" if ok else "  RESULT CHANGED"))
        if not ok:
            raise RuntimeError("tunable changed the result: %r" % c)
        return ms

    best_ms = measure(cfg)
    for _ in range(rounds):
        for k, values in space.items():
            for v in values:
                if v == cfg[k]:
                    continue
                trial = dict(cfg, **{k: v})
                if not feasible(trial):
                    continue
                ms = measure(trial)
                if ms < best_ms:
                    best_ms, cfg = ms, trial
    for k, v in cfg.items():
        G.tune_set(k, v, ws=ws)
    return cfg, table


def save(path: str, results: Dict[str, Dict[str, int]]) -> None:
    with open(path, "w") as f:
        json.dump(results, f, indent=1, sort_keys=True)


def load(path: str, ws=None) -> Dict[str, Dict[str, int]]:
    """Apply saved values (every algorithm's) to the workspace."""
    import graphhet_b200 as G
    with open(path) as f:
        results = json.load(f)
    for cfg in results.values():
        for k, v in cfg.items():
            G.tune_set(k, v, ws=ws)
    return results


def main(argv=None) -> int:
    import argparse

    import graphhet_b200 as G
    ap = argparse.ArgumentParser(description="search libghb's launch shapes and thresholds on an RMAT graph")
    ap.add_argument("--algo", choices=sorted(SPACES), action="append")
    ap.add_argument("--scale", type=int, default=22)
    ap.add_argument("--edge-factor", type=int, default=16)
    ap.add_argument("--seed", type=int, default=7)
    ap.add_argument("--sources", type=int, default=256)
    ap.add_argument("--out", default=None, help="write the chosen values as JSON")
    a = ap.parse_args(argv)
    g = G.rmat_graph(a.scale, a.edge_factor, a.seed)
    rg = G.ResidentGraph(g)
    import numpy as np
    deg = (g.rowptr[1:] - g.rowptr[:-1]).cpu().numpy()
    cand = np.nonzero(deg > 0)[0]
    srcs = [int(x) for x in np.random.default_rng(a.seed).choice(cand, size=min(a.sources, cand.size), replace=False)]
    del g
    results = {}
    for algo in a.algo or sorted(SPACES):
        cfg, table = tune(rg, algo, sources=srcs)
        default_ms, best_ms = table[0]["ms"], min(t["ms"] for t in table)
        results[algo] = cfg
        print(json.dumps({"algo": algo, "scale": a.scale, "best": cfg, "default_ms": default_ms, "best_ms": best_ms}))
    if a.out:
        save(a.out, results)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
